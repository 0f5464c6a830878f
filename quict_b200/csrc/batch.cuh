// Persistent batch kernel: device code shared by the generic kernel
// (batch.cu) and the relocatable kernel linked with generated register-stage
// functions (rdc/batch_dev.cu).  See batch.cu for the design.
#pragma once

#include "common.cuh"
#include "regtile.cuh"

namespace qs {
namespace {

enum : int32_t { BI_FWD = 0, BI_HAM = 1, BI_BWD = 2, BI_FIN = 3 };

struct __align__(16) BItem {
    int32_t kind;     // BI_*
    int32_t inst;     // instance
    int32_t stage;    // FWD / BWD: index of the stage's BArgs; HAM: index of the item within the HAM stage
    int32_t fresh;    // FWD: the pass reads |0...0> instead of psi
    int64_t need;     // items of this instance that finish before this one starts
    uint64_t t0, t1;  // FWD / BWD: tile range; HAM: amplitude range of psi
};

struct __align__(16) BInst {
    int32_t n, nslots, nparams, nham;
    int32_t term_begin, nterms, tiles_bwd, pad;
    int64_t state_off;  // elements: the pair vector (psi: 2^n amplitudes, then lam)
    int64_t part_off;   // doubles: EXPECT partials (2 nslots tiles_bwd), then HAM partials (2 nham)
    int64_t w_off;      // doubles of the blob's weight array: W (nparams x nslots, row-major)
    int64_t grad_off;   // doubles of the gradient output
};

struct __align__(16) BTerm {  // an instance's terms are sorted (stably) by x
    uint64_t x, z;
    double cre, cim;  // coefficient times i^popc(x & z)
};

struct __align__(16) BArgs {  // a planned register pass; its arrays sit elsewhere in the blob
    RegHead h;
    int64_t off_st, off_ops, off_cp, off_es;  // byte offsets in the blob
    int32_t jit_fn;      // generated device function of the linked kernel (-1: the generic body)
    int32_t pad;
    int64_t off_params;  // byte offset of that function's parameter block
};

struct __align__(16) BHead {
    int32_t ninst, nitems, nstages, dtype;
    int32_t threads, big, pad0, pad1;
    int64_t off_items, off_inst, off_args, off_terms, off_w;
    int64_t smem;
};

// control words (ctrl): [0] next item, [1] error (0, or (1 << 32) | item whose
// wait timed out), [2], [3] unused, [4 + i] items of instance i done
constexpr int kCtrlHead = 4;

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Block sum of (a, b) in a fixed order; the result is valid in thread 0.
__device__ __forceinline__ double2 block_sum(double a, double b) {
    __shared__ double2 red[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = make_double2(a, b);
    __syncthreads();
    double2 s = make_double2(0.0, 0.0);
    if (threadIdx.x == 0)
        for (int w = 0; w < int(blockDim.x >> 5); ++w) {
            s.x += red[w].x;
            s.y += red[w].y;
        }
    return s;
}

// lam[j] = sum_t c_t (-1)^popc(z_t & (j ^ x_t)) psi[j ^ x_t] for j in [j0, j1),
// and the FP64 partial of <psi|lam> over the range (lam as stored).  psi was
// written by other CTAs of this launch: it is read through L2 (ld.cg).
template <typename V>
__device__ void ham_range(V* __restrict__ pl, const BInst& I, const BTerm* __restrict__ tm, uint64_t j0, uint64_t j1,
                          double* __restrict__ out) {
    const uint64_t N = uint64_t(1) << I.n;
    const V* psi = pl;
    V* lam = pl + N;
    double er = 0.0, ei = 0.0;
    for (uint64_t j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
        double re = 0.0, im = 0.0;
        int t = 0;
        while (t < I.nterms) {
            const uint64_t x = tm[t].x;
            const uint64_t src = j ^ x;
            const V a = __ldcg(psi + src);
            double sr = 0.0, si = 0.0;
            for (; t < I.nterms && tm[t].x == x; ++t) {
                const bool neg = __popcll(tm[t].z & src) & 1;
                sr += neg ? -tm[t].cre : tm[t].cre;
                si += neg ? -tm[t].cim : tm[t].cim;
            }
            const double ar = double(a.x), ai = double(a.y);
            re += sr * ar - si * ai;
            im += sr * ai + si * ar;
        }
        const V lv = mk<V>(re, im);
        lam[j] = lv;
        const V u = __ldcg(psi + j);
        er += double(u.x) * double(lv.x) + double(u.y) * double(lv.y);
        ei += double(u.x) * double(lv.y) - double(u.y) * double(lv.x);
    }
    const double2 s = block_sum(er, ei);
    if (threadIdx.x == 0) {
        out[0] = s.x;
        out[1] = s.y;
    }
}

// energy (re, im) = sum of the HAM partials; gradient[k] = sum_s W[k, s] *
// Im(sum over tiles of slot s's EXPECT partials).  `scratch`: nslots doubles
// of shared memory.
__device__ void finish(const BInst& I, const double* __restrict__ parts, const double* __restrict__ W,
                       double* __restrict__ energy, double* __restrict__ grads, double* __restrict__ scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const double* ep = parts + I.part_off + 2 * int64_t(I.nslots) * I.tiles_bwd;
    if (warp == 0) {
        double r = 0.0, i = 0.0;
        for (int t = lane; t < I.nham; t += 32) {
            r += __ldcg(ep + 2 * t);
            i += __ldcg(ep + 2 * t + 1);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            r += __shfl_xor_sync(0xffffffffu, r, o);
            i += __shfl_xor_sync(0xffffffffu, i, o);
        }
        if (lane == 0) {
            energy[0] = r;
            energy[1] = i;
        }
    }
    for (int s = warp; s < I.nslots; s += nw) {
        const double* sp = parts + I.part_off + 2 * int64_t(s) * I.tiles_bwd;
        double im = 0.0;
        for (int t = lane; t < I.tiles_bwd; t += 32) im += __ldcg(sp + 2 * t + 1);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) im += __shfl_xor_sync(0xffffffffu, im, o);
        if (lane == 0) scratch[s] = im;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < I.nparams; k += blockDim.x) {
        const double* w = W + I.w_off + int64_t(k) * I.nslots;
        double g = 0.0;
        for (int s = 0; s < I.nslots; ++s) g += w[s] * scratch[s];
        grads[I.grad_off + k] = g;
    }
}

// One register stage's tiles [t0, t1); a call (not inlined), so that each
// body is optimised on its own.
template <typename V, int R, bool EXP>
__device__ __noinline__ void batch_pass(V* __restrict__ vec, const RegHead& h, const KStage* __restrict__ st,
                                        const KOp* __restrict__ ops, const KCopy* __restrict__ cp,
                                        const int* __restrict__ es, const V* __restrict__ mats,
                                        double* __restrict__ partials, uint64_t t0, uint64_t t1, bool fresh) {
    reg_tiles<V, R, EXP, false>(vec, h, st, ops, cp, es, mats, partials, t0, t1, 1, fresh);
}

// The generated-function dispatcher of a linked batch kernel (generated with
// the plan, compiled at link time): runs register stage function `fn`;
// returns 0 for an unknown index.
extern "C" __device__ int qs_batch_jit(int fn, void* vec, const void* params, const void* mats, double* partials,
                                       unsigned long long t0, unsigned long long t1, unsigned zero_in);

// The persistent loop.  LINKED: register stages with a generated function
// (BArgs.jit_fn >= 0) call it through qs_batch_jit; otherwise (and always
// when !LINKED) they run the generic register body.
template <typename V, int R, bool LINKED>
__device__ __forceinline__ void batch_loop(const unsigned char* __restrict__ blob, V* __restrict__ states,
                                           const V* __restrict__ mats, double* __restrict__ parts,
                                           double* __restrict__ energies, double* __restrict__ grads,
                                           unsigned long long* __restrict__ ctrl, uint64_t timeout_ns) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const BHead& hd = *reinterpret_cast<const BHead*>(blob);
    const BItem* items = reinterpret_cast<const BItem*>(blob + hd.off_items);
    const BInst* insts = reinterpret_cast<const BInst*>(blob + hd.off_inst);
    const BArgs* args = reinterpret_cast<const BArgs*>(blob + hd.off_args);
    const BTerm* terms = reinterpret_cast<const BTerm*>(blob + hd.off_terms);
    const double* W = reinterpret_cast<const double*>(blob + hd.off_w);
    unsigned long long* next = ctrl;
    unsigned long long* err = ctrl + 1;
    unsigned long long* done = ctrl + kCtrlHead;
    __shared__ long long s_item;
    for (;;) {
        if (threadIdx.x == 0) {
            long long it = (long long)atomicAdd(next, 1ull);
            if (it < hd.nitems) {
                const BItem& I = items[it];
                const unsigned long long need = (unsigned long long)I.need;
                if (need > 0 && ld_acquire(done + I.inst) < need) {
                    const uint64_t start = global_ns();
                    while (ld_acquire(done + I.inst) < need) {
                        if (*reinterpret_cast<volatile unsigned long long*>(err) != 0ull) {
                            it = -1;
                            break;
                        }
                        if (global_ns() - start > timeout_ns) {
                            atomicCAS(err, 0ull, (1ull << 32) | (unsigned long long)it);
                            it = -1;
                            break;
                        }
                        __nanosleep(256);
                    }
                }
                __threadfence();
            }
            s_item = it;
        }
        __syncthreads();
        const long long it = s_item;
        if (it < 0 || it >= hd.nitems) return;
        const BItem& I = items[it];
        const BInst& S = insts[I.inst];
        V* pl = states + S.state_off;
        if (I.kind == BI_FWD || I.kind == BI_BWD) {
            const BArgs& A = args[I.stage];
            const KStage* st = reinterpret_cast<const KStage*>(blob + A.off_st);
            const KOp* ops = reinterpret_cast<const KOp*>(blob + A.off_ops);
            const KCopy* cp = reinterpret_cast<const KCopy*>(blob + A.off_cp);
            const int* es = reinterpret_cast<const int*>(blob + A.off_es);
            double* pp = I.kind == BI_BWD ? parts + S.part_off : nullptr;
            int ran = 0;
            if constexpr (LINKED) {
                if (A.jit_fn >= 0)
                    ran = qs_batch_jit(A.jit_fn, pl, blob + A.off_params, mats, pp, I.t0, I.t1, unsigned(I.fresh));
            }
            if (!ran) {
                if (I.kind == BI_FWD) batch_pass<V, R, false>(pl, A.h, st, ops, cp, es, mats, pp, I.t0, I.t1, I.fresh != 0);
                else batch_pass<V, R, true>(pl, A.h, st, ops, cp, es, mats, pp, I.t0, I.t1, false);
            }
        } else if (I.kind == BI_HAM) {
            ham_range<V>(pl, S, terms + S.term_begin, I.t0, I.t1,
                         parts + S.part_off + 2 * int64_t(S.nslots) * S.tiles_bwd + 2 * int64_t(I.stage));
        } else {
            finish(S, parts, W, energies + 2 * int64_t(I.inst), grads, reinterpret_cast<double*>(smem_raw));
        }
        __syncthreads();  // the item's stores are done; shared memory is free again
        if (threadIdx.x == 0) {
            __threadfence();
            atomicAdd(done + I.inst, 1ull);
        }
    }
}

}  // namespace
}  // namespace qs
