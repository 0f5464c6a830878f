// Fused passes: one launch streams the state through on-chip tiles once and
// applies every op of the pass to each tile.
//
// A tile holds 2^k amplitudes: vector bits 0..nlow-1 (contiguous, so each
// warp moves 2^nlow consecutive amplitudes) plus k-nlow chosen higher bits.
// Ops whose non-diagonal targets lie in the tile run on chip; diagonal factors
// and controls on bits outside the tile are resolved per tile from the tile's
// base index, so they fuse into any pass.
//
// Register-resident kernel (k_fused_reg, tiles of 2^(R+5..R+8)):
//   each thread owns 2^R amplitudes in registers.  A "layout" assigns R tile
//   bits to register-slot bits and the remaining tile bits to the thread index
//   (lanes first).  Ops whose dense targets are slot bits run as fully
//   unrolled register code (one template per slot mask, no shared memory, no
//   barriers); between groups of ops ("stages") the tile is re-laid-out
//   through shared memory under a per-relayout XOR address map that keeps
//   both sides free of bank conflicts.  Loads and stores use a layout whose
//   lanes are tile bits 0..4, i.e. warp-contiguous global runs.  The host
//   (this file) plans the stages, translates each op into slot / thread /
//   outside-tile terms and permutes its matrix to the slot order.
// Shared-memory kernel (k_fused_smem): tiles too small for that layout.
//
// The reference has no fusion: one kernel and one full HBM pass per gate
// (statevector_simulator.py:155-164, gate_function.py:31-1031).
#include <algorithm>
#include <array>
#include <cstdarg>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <type_traits>
#include <unordered_map>
#include <utility>
#include <vector>

#include "common.cuh"
#include "jit.h"
#include "regtile.cuh"

namespace qs {
namespace {

constexpr int kFT = 256;

// =============================================================== shared-memory kernel
struct PassArgs {
    int n, k, nlow, nops, inst_shift;
    int hi[QS_MAX_TILE_BITS];
    qs_op ops[QS_MAX_PASS_OPS];
};

template <int M>
__device__ __forceinline__ void sort_bits(const int* t, int* s) {
#pragma unroll
    for (int i = 0; i < M; ++i) s[i] = t[i];
#pragma unroll
    for (int i = 0; i < M; ++i)
#pragma unroll
        for (int j = 0; j + 1 < M - i; ++j)
            if (s[j] > s[j + 1]) { int x = s[j]; s[j] = s[j + 1]; s[j + 1] = x; }
}

template <typename V, int M>
__device__ __forceinline__ void tile_mat(V* __restrict__ tile, int K, const qs_op& op, const V* __restrict__ mat) {
    constexpr int D = 1 << M;
    int t[M], s[M];
#pragma unroll
    for (int j = 0; j < M; ++j) t[j] = op.tgt[j];
    sort_bits<M>(t, s);
    uint32_t spread[D];
#pragma unroll
    for (int r = 0; r < D; ++r) {
        uint32_t o = 0;
#pragma unroll
        for (int j = 0; j < M; ++j)
            if ((r >> (M - 1 - j)) & 1) o |= 1u << t[j];
        spread[r] = o;
    }
    const uint32_t lctrl = op.lctrl;
    const uint32_t groups = 1u << (K - M);
    for (uint32_t g = threadIdx.x; g < groups; g += kFT) {
        uint32_t i0 = g;
#pragma unroll
        for (int j = 0; j < M; ++j) i0 = ins0(i0, s[j]);
        if ((i0 & lctrl) != lctrl) continue;
        V x[D];
#pragma unroll
        for (int r = 0; r < D; ++r) x[r] = tile[i0 | spread[r]];
#pragma unroll
        for (int r = 0; r < D; ++r) {
            V acc = cmul(__ldg(&mat[r * D]), x[0]);
#pragma unroll
            for (int c = 1; c < D; ++c) acc = cfma(__ldg(&mat[r * D + c]), x[c], acc);
            tile[i0 | spread[r]] = acc;
        }
    }
}

template <typename V>
__device__ __forceinline__ void tile_diag(V* __restrict__ tile, int K, uint64_t base, const qs_op& op,
                                          const V* __restrict__ mat) {
    const int m = op.m;
    uint32_t ext = 0;
    int lpos[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        lpos[j] = -1;
        if (j < m) {
            if (op.tgt[j] < 0) ext |= uint32_t((base >> op.gbit[j]) & 1) << (m - 1 - j);
            else lpos[j] = op.tgt[j];
        }
    }
    const uint32_t lctrl = op.lctrl;
    const uint32_t T = 1u << K;
    for (uint32_t e = threadIdx.x; e < T; e += kFT) {
        if ((e & lctrl) != lctrl) continue;
        uint32_t sidx = ext;
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (j < m && lpos[j] >= 0) sidx |= ((e >> lpos[j]) & 1u) << (m - 1 - j);
        tile[e] = cmul(tile[e], __ldg(&mat[sidx]));
    }
}

// <lam| G |psi> over the tile for a generator on m <= 2 tile bits (dense) or
// a diagonal on bits anywhere (QS_OPF_DIAG); thread-partial sum returned.
template <typename V, int M>
__device__ __forceinline__ double2 tile_expect_dense(const V* __restrict__ psi, const V* __restrict__ lam, int K,
                                                     const qs_op& op, const V* __restrict__ g) {
    constexpr int D = 1 << M;
    int t[M], s[M];
#pragma unroll
    for (int j = 0; j < M; ++j) t[j] = op.tgt[j];
    sort_bits<M>(t, s);
    uint32_t spread[D];
#pragma unroll
    for (int r = 0; r < D; ++r) {
        uint32_t o = 0;
#pragma unroll
        for (int j = 0; j < M; ++j)
            if ((r >> (M - 1 - j)) & 1) o |= 1u << t[j];
        spread[r] = o;
    }
    double re = 0.0, im = 0.0;
    const uint32_t groups = 1u << (K - M);
    for (uint32_t gi = threadIdx.x; gi < groups; gi += blockDim.x) {
        uint32_t i0 = gi;
#pragma unroll
        for (int j = 0; j < M; ++j) i0 = ins0(i0, s[j]);
        if ((i0 & op.lctrl) != op.lctrl) continue;
        V x[D];
#pragma unroll
        for (int r = 0; r < D; ++r) x[r] = psi[i0 | spread[r]];
#pragma unroll
        for (int r = 0; r < D; ++r) {
            V acc = cmul(g[r * D], x[0]);
#pragma unroll
            for (int c = 1; c < D; ++c) acc = cfma(g[r * D + c], x[c], acc);
            const V l = lam[i0 | spread[r]];
            re += double(l.x) * double(acc.x) + double(l.y) * double(acc.y);
            im += double(l.x) * double(acc.y) - double(l.y) * double(acc.x);
        }
    }
    return make_double2(re, im);
}

template <typename V>
__device__ __forceinline__ double2 tile_expect_diag(const V* __restrict__ psi, const V* __restrict__ lam, int K,
                                                    uint64_t base, const qs_op& op, const V* __restrict__ d) {
    const int m = op.m;
    uint32_t ext = 0;
    int lpos[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        lpos[j] = -1;
        if (j < m) {
            if (op.tgt[j] < 0) ext |= uint32_t((base >> op.gbit[j]) & 1) << (m - 1 - j);
            else lpos[j] = op.tgt[j];
        }
    }
    double re = 0.0, im = 0.0;
    for (uint32_t e = threadIdx.x; e < (1u << K); e += blockDim.x) {
        if ((e & op.lctrl) != op.lctrl) continue;
        uint32_t sidx = ext;
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (j < m && lpos[j] >= 0) sidx |= ((e >> lpos[j]) & 1u) << (m - 1 - j);
        const V acc = cmul(d[sidx], psi[e]);
        const V l = lam[e];
        re += double(l.x) * double(acc.x) + double(l.y) * double(acc.y);
        im += double(l.x) * double(acc.y) - double(l.y) * double(acc.x);
    }
    return make_double2(re, im);
}

// Shared-memory tile kernel.  ADJ: two vectors (psi, lam) move through the
// same tiles; apply-ops act on both and EXPECT ops write per-tile partials.
template <typename V, bool ADJ>
__global__ void __launch_bounds__(kFT) k_fused_smem(V* __restrict__ vec, V* __restrict__ vec2,
                                                     const __grid_constant__ PassArgs p, const V* __restrict__ mats,
                                                     double* __restrict__ partials) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double2 red[kFT / 32];
    const int K = p.k, L = p.nlow, H = K - L;
    const uint32_t T = 1u << K;
    V* tile = reinterpret_cast<V*>(smem_raw);
    V* tile2 = tile + (ADJ ? T : 0);
    uint64_t* hoff = reinterpret_cast<uint64_t*>(smem_raw + sizeof(V) * T * (ADJ ? 2 : 1));
    for (uint32_t j = threadIdx.x; j < (1u << H); j += kFT) {
        uint64_t o = 0;
        for (int t = 0; t < H; ++t)
            if ((j >> t) & 1) o |= uint64_t(1) << p.hi[t];
        hoff[j] = o;
    }
    __syncthreads();
    const uint32_t lmask = (1u << L) - 1u;
    const uint64_t ntiles = uint64_t(1) << (p.n - K);
    for (uint64_t tid = blockIdx.x; tid < ntiles; tid += gridDim.x) {
        uint64_t base = tid << L;
        for (int t = 0; t < H; ++t) base = insert0(base, p.hi[t]);
        const uint64_t inst = p.inst_shift > 0 ? (base >> p.inst_shift) : 0;
        for (uint32_t e = threadIdx.x; e < T; e += kFT) {
            const uint64_t gi = base | hoff[e >> L] | (e & lmask);
            tile[e] = vec[gi];
            if (ADJ) tile2[e] = vec2[gi];
        }
        __syncthreads();
        for (int o = 0; o < p.nops; ++o) {
            const qs_op& op = p.ops[o];
            const bool on = (base & op.gctrl) == op.gctrl;  // CTA-uniform
            const V* mat = mats + op.mat + int64_t(inst) * op.mat_stride;
            if (ADJ && op.kind == QS_OP_EXPECT) {
                double2 v = make_double2(0.0, 0.0);
                if (on) {
                    if (op.flags & QS_OPF_DIAG) v = tile_expect_diag<V>(tile, tile2, K, base, op, mat);
                    else if (op.m == 1) v = tile_expect_dense<V, 1>(tile, tile2, K, op, mat);
                    else v = tile_expect_dense<V, 2>(tile, tile2, K, op, mat);
                }
                // block reduction in a fixed order (deterministic)
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) {
                    v.x += __shfl_xor_sync(0xffffffffu, v.x, off);
                    v.y += __shfl_xor_sync(0xffffffffu, v.y, off);
                }
                if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
                __syncthreads();
                if (threadIdx.x == 0) {
                    double2 s2 = make_double2(0.0, 0.0);
                    for (int w = 0; w < kFT / 32; ++w) { s2.x += red[w].x; s2.y += red[w].y; }
                    const uint64_t at = 2 * (uint64_t(op.slot) * ntiles + tid);
                    partials[at] = s2.x;
                    partials[at + 1] = s2.y;
                }
                __syncthreads();
                continue;
            }
            if (!on) continue;
            if (op.kind == QS_OP_DIAG) {
                tile_diag<V>(tile, K, base, op, mat);
                if (ADJ) tile_diag<V>(tile2, K, base, op, mat);
            } else {
                switch (op.m) {
                    case 1: tile_mat<V, 1>(tile, K, op, mat); if (ADJ) tile_mat<V, 1>(tile2, K, op, mat); break;
                    case 2: tile_mat<V, 2>(tile, K, op, mat); if (ADJ) tile_mat<V, 2>(tile2, K, op, mat); break;
                    case 3: tile_mat<V, 3>(tile, K, op, mat); if (ADJ) tile_mat<V, 3>(tile2, K, op, mat); break;
                    default: tile_mat<V, 4>(tile, K, op, mat); if (ADJ) tile_mat<V, 4>(tile2, K, op, mat); break;
                }
            }
            __syncthreads();
        }
        for (uint32_t e = threadIdx.x; e < T; e += kFT) {
            const uint64_t gi = base | hoff[e >> L] | (e & lmask);
            vec[gi] = tile[e];
            if (ADJ) vec2[gi] = tile2[e];
        }
        __syncthreads();
    }
}

// One register pass over the whole vector.  Tile order: strided over the
// grid; batched passes take contiguous runs of tiles instead, so that a CTA
// restages per-instance matrices once per instance rather than once per tile.
template <typename V, int R, bool EXP, bool BIG>
__global__ void __launch_bounds__(256, 1) k_fused_reg(V* __restrict__ vec, const __grid_constant__ RegArgs p,
                                                      const V* __restrict__ mats, double* __restrict__ partials) {
    const uint64_t ntiles = uint64_t(1) << (p.n - p.K);
    uint64_t tile = blockIdx.x, tend = ntiles, tstep = gridDim.x;
    if (p.batched) {
        const uint64_t chunk = (ntiles + gridDim.x - 1) / gridDim.x;
        tile = uint64_t(blockIdx.x) * chunk;
        tend = tile + chunk < ntiles ? tile + chunk : ntiles;
        tstep = 1;
    }
    // one call: the body is inlined once
    reg_tiles<V, R, EXP, BIG>(vec, p, p.st, p.ops, p.cp, p.eslot, mats, partials, tile, tend, tstep, false);
}

template <typename V, bool ADJ>
int launch_smem(V* vec, V* vec2, int n, const qs_pass& ps, const qs_op* ops, const V* mats, double* partials,
                cudaStream_t st) {
    static thread_local PassArgs args;
    args.n = n; args.k = ps.k; args.nlow = ps.nlow; args.nops = ps.op_count; args.inst_shift = ps.inst_shift;
    for (int t = 0; t < QS_MAX_TILE_BITS; ++t) args.hi[t] = t < ps.k - ps.nlow ? ps.hi[t] : 0;
    for (int i = 0; i < ps.op_count; ++i) args.ops[i] = ops[ps.op_begin + i];
    size_t smem = sizeof(V) * (size_t(1) << ps.k) * (ADJ ? 2 : 1) + sizeof(uint64_t) * (size_t(1) << (ps.k - ps.nlow));
    config_smem((const void*)k_fused_smem<V, ADJ>);
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_fused_smem<V, ADJ>, kFT, smem);
    if (occ < 1) occ = 1;
    uint64_t ntiles = uint64_t(1) << (n - ps.k);
    uint64_t cap = uint64_t(sm_count()) * occ;
    k_fused_smem<V, ADJ><<<unsigned(ntiles < cap ? ntiles : cap), kFT, smem, st>>>(vec, vec2, args, mats, partials);
    QS_CHECK_LAUNCH(ADJ ? "qs_adjoint_fused" : "qs_apply_fused(smem)");
    return QS_OK;
}

// ------------------------------------------------------- run-time compiled passes
// A register pass planned by build_reg can also run as a kernel generated for
// it alone: every op, slot mask, control and relayout address is a constant
// of the generated code, so there is no per-op dispatch, plain exchanges
// (X, CX, SWAP without outside controls) become register renamings, zero and
// unit matrix entries drop out of the arithmetic, and the matrices are read
// as constant-bank operands from the launch's parameter block.  The source
// depends on the pass's structure and on which matrix entries are exactly
// 0, 1 or -1, not on the other matrix values, so passes of the same shape
// share one compiled kernel (jit.cu caches by source text).
// Single-buffered generated kernels (see gen_reg_pass): QS_JIT_SINGLE_BUFFER=0 / 1,
// else complex128 only.
inline bool jit_single_buffer(bool c128) {
    static const int env = [] {
        const char* e = getenv("QS_JIT_SINGLE_BUFFER");
        return e && (*e == '0' || *e == '1') ? *e - '0' : -1;
    }();
    return env >= 0 ? env == 1 : c128;
}

struct JitPass {
    std::string src;
    std::vector<uint64_t> params;  // the kernel's parameter block (16-byte multiple)
    std::vector<uint8_t> classes;  // value class of every matrix entry (what the source depends on)
    int threads = 0;
    size_t smem = 0;
};

constexpr size_t kJitMaxParamBytes = 32000;  // below the 32764-byte kernel parameter limit

struct SrcBuf {
    std::string s;
    bool truncated = false;  // a formatted piece did not fit: the source is not used
    void add(const char* fmt, ...) __attribute__((format(printf, 2, 3))) {
        char tmp[1024];
        va_list ap;
        va_start(ap, fmt);
        int k = vsnprintf(tmp, sizeof(tmp), fmt, ap);
        va_end(ap);
        if (k >= int(sizeof(tmp))) {
            truncated = true;
            k = int(sizeof(tmp)) - 1;
        }
        s.append(tmp, size_t(k));
    }
};

// XOR of per-thread-bit images over the set bits of threadIdx.x, as an expression
std::string thread_xor_expr(const uint32_t* img, int nT) {
    std::string e;
    for (int i = 0; i < nT; ++i) {
        if (!img[i]) continue;
        char t[64];
        snprintf(t, sizeof(t), "%s(((tid >> %d) & 1u) * %uu)", e.empty() ? "" : " ^ ", i, img[i]);
        e += t;
    }
    return e.empty() ? std::string("0u") : e;
}

// devfn != nullptr: emit the pass as `extern "C" __device__ void <devfn>(vec,
// params, mats, partials, tile, tend, zero_in)` for the persistent batch
// kernel instead of a kernel: it runs tiles [tile, tend) of the calling CTA,
// reads its parameter block from global memory (params), may run in a CTA
// wider than its own thread count (the other threads share the loads, repeat
// the register work of thread tid mod threads, and store nothing), and with
// zero_in != 0 reads |0...0> instead of the vector.
template <typename V>
bool gen_reg_pass(const RegArgs& a, int R, const V* hm, JitPass& out, bool with_source = true,
                  const char* devfn = nullptr) {
    constexpr bool C128 = sizeof(V) == 16;
    const int E = 1 << R, nT = a.nT, K = a.K, L = a.L, H = a.H;
    const int threads = 1 << nT, nwarps = threads / 32;
    const int NM = a.nmats > 0 ? a.nmats : 1;
    const int NOPS = a.nops > 0 ? a.nops : 1;
    const int NEXP = a.nexp > 0 ? a.nexp : 1;
    const bool batched = a.batched != 0;
    // ---- parameter block (all fields 8-byte aligned, V first):
    //   V m[NM]; u64 ntiles, gthr[8], gslot[E], hibit[16], gctrl[NOPS], hsh[4 NOPS],
    //   mgoff[NOPS], mstride[NOPS], eslot[NEXP], misc[2]; u32 pe[NM]
    // m holds every op's matrix in slot order; for a batched pass the ops with
    // per-instance tables (stride != 0) are staged into shared memory per
    // instance instead: pe[g] = (op << 16) | offset within the instance block
    const size_t o_ntiles = sizeof(V) * size_t(NM), o_gthr = o_ntiles + 8, o_gslot = o_gthr + 64,
                 o_hibit = o_gslot + 8 * size_t(E), o_gctrl = o_hibit + 128, o_hsh = o_gctrl + 8 * size_t(NOPS),
                 o_mgoff = o_hsh + 32 * size_t(NOPS), o_mstride = o_mgoff + 8 * size_t(NOPS),
                 o_eslot = o_mstride + 8 * size_t(NOPS), o_misc = o_eslot + 8 * size_t(NEXP), o_pe = o_misc + 16;
    size_t bytes = o_pe + (batched ? 4 * size_t(NM) : 0);
    bytes = (bytes + 15) & ~size_t(15);
    if (bytes > kJitMaxParamBytes) return false;
    out.params.assign(bytes / 8, 0);
    unsigned char* pb = reinterpret_cast<unsigned char*>(out.params.data());
    auto put64 = [&](size_t off, uint64_t v) { memcpy(pb + off, &v, 8); };
    V* pm = reinterpret_cast<V*>(pb);
    std::vector<char> strided(size_t(NOPS), 0);
    for (int o = 0; o < a.nops; ++o) {
        const KCopy& c = a.cp[o];
        const int D = 1 << c.m;
        const int cnt = c.diag ? D : D * D;
        strided[o] = batched && c.stride != 0;
        put64(o_mgoff + 8 * size_t(o), uint64_t(c.goff));
        put64(o_mstride + 8 * size_t(o), uint64_t(c.stride));
        for (int e = 0; e < cnt; ++e) {
            const int kr = c.diag ? e : e / D, kc = c.diag ? 0 : e % D;
            int sr = 0, sc = 0;
            for (int i = 0; i < c.m; ++i) {
                sr |= ((kr >> i) & 1) << c.perm[i];
                sc |= ((kc >> i) & 1) << c.perm[i];
            }
            const int src = c.diag ? sr : sr * D + sc;
            if (strided[o]) {  // bit 31 marks a staged entry
                const uint32_t v = (1u << 31) | (uint32_t(o) << 16) | uint32_t(src);
                memcpy(pb + o_pe + 4 * size_t(c.soff + e), &v, 4);
            } else {
                pm[c.soff + e] = hm[c.goff + src];
            }
        }
    }
    if (a.nops > 32767) return false;
    // tile position of the psi/lam pair bit (adjoint pair passes)
    int pair_tile = -1;
    for (int b = 0; b < 64 && a.pairmask; ++b)
        if ((a.pairmask >> b) & 1) {
            if (b < L) pair_tile = b;
            for (int t = 0; t < H; ++t)
                if (a.hi[t] == b) pair_tile = L + t;
        }
    auto gbit = [&](int b) -> uint64_t { return uint64_t(1) << (b < L ? b : a.hi[b - L]); };
    const KStage& SL = a.st[a.nstages - 1];
    put64(o_ntiles, uint64_t(1) << (a.n - K));
    for (int i = 0; i < nT; ++i) put64(o_gthr + 8 * i, gbit(SL.T[i]));
    for (int s = 0; s < E; ++s) {
        uint64_t v = 0;
        for (int j = 0; j < R; ++j)
            if ((s >> j) & 1) v |= gbit(SL.R[j]);
        put64(o_gslot + 8 * s, v);
    }
    for (int t = 0; t < H; ++t) put64(o_hibit + 8 * t, uint64_t(1) << a.hi[t]);
    for (int o = 0; o < a.nops; ++o) {
        put64(o_gctrl + 8 * o, a.ops[o].gctrl);
        for (int q = 0; q < a.ops[o].nh; ++q)
            put64(o_hsh + 32 * o + 8 * q, a.ops[o].hsrc[q] >= 64 ? uint64_t(a.ops[o].hsrc[q] - 64) : 0);
    }
    for (int e = 0; e < a.nexp; ++e) put64(o_eslot + 8 * e, uint64_t(a.eslot[e]));
    put64(o_misc, ~a.pairmask);
    put64(o_misc + 8, uint64_t(a.inst_shift));
    // value class of a matrix entry: 0, 1, -1, general (3), real (4), imaginary
    // (5).  An entry of a per-instance table gets the class that holds for
    // every instance's value (e.g. real for the entries of Ry tables, imaginary
    // for the off-diagonal entries of Rx tables); the value itself is read from
    // the staged table at run time.
    auto value_class = [](const V v) -> int {
        if (v.y == 0) {
            if (v.x == 0) return 0;
            if (v.x == 1) return 1;
            if (v.x == -1) return 2;
            return 4;
        }
        return v.x == 0 ? 5 : 3;
    };
    auto join_class = [](int c1, int c2) -> int {
        if (c1 == c2) return c1;
        const bool r1 = c1 == 0 || c1 == 1 || c1 == 2 || c1 == 4, r2 = c2 == 0 || c2 == 1 || c2 == 2 || c2 == 4;
        if (r1 && r2) return 4;
        if ((c1 == 0 || c1 == 5) && (c2 == 0 || c2 == 5)) return 5;
        return 3;
    };
    // instances of a batched pass: the vector bits above inst_shift, less the pair bit
    const int64_t ninst =
        batched && a.inst_shift > 0 ? (int64_t(1) << (a.n - a.inst_shift - (a.pairmask ? 1 : 0))) : int64_t(1);
    std::vector<uint8_t> scls(size_t(NM), 3);
    for (int o = 0; o < a.nops; ++o) {
        if (!strided[o]) continue;
        const KCopy& c = a.cp[o];
        const int D = 1 << c.m;
        const int cnt = c.diag ? D : D * D;
        for (int e = 0; e < cnt; ++e) {
            const int kr = c.diag ? e : e / D, kc = c.diag ? 0 : e % D;
            int sr = 0, sc = 0;
            for (int i = 0; i < c.m; ++i) {
                sr |= ((kr >> i) & 1) << c.perm[i];
                sc |= ((kc >> i) & 1) << c.perm[i];
            }
            const int64_t src = c.goff + (c.diag ? sr : sr * D + sc);
            int cl = value_class(hm[src]);
            for (int64_t i = 1; i < ninst && cl != 3; ++i) cl = join_class(cl, value_class(hm[src + i * c.stride]));
            scls[size_t(c.soff + e)] = uint8_t(cl);
        }
    }
    auto vclass = [&](int o, int idx) -> int { return strided[o] ? int(scls[size_t(idx)]) : value_class(pm[idx]); };
    auto mref = [&](int o, int idx) -> std::string {
        return (strided[o] ? "msm[" : "p.m[") + std::to_string(idx) + "]";
    };
    out.classes.resize(size_t(NM));
    for (int o = 0; o < a.nops; ++o) {
        const KCopy& c = a.cp[o];
        const int cnt = c.diag ? (1 << c.m) : (1 << (2 * c.m));
        for (int e = 0; e < cnt; ++e) out.classes[c.soff + e] = uint8_t(vclass(o, c.soff + e));
    }
    // Diagonal tables indexed by thread bits (a different entry per lane) are
    // copied to shared memory once per CTA: parameter-space loads with lane-
    // dependent addresses are serialised, shared-memory loads are not.
    std::vector<int> doff(size_t(NOPS), -1);
    int ndsm = 0;
    for (int o = 0; o < a.nops; ++o) {
        const KOp& op = a.ops[o];
        const bool dg = op.code == QS_OP_DIAG || (op.code == QS_OP_EXPECT && (op.flags & QS_OPF_DIAG));
        if (!dg || op.nh == 0 || strided[o]) continue;
        bool thr = false;
        for (int q = 0; q < op.nh; ++q) thr = thr || op.hsrc[q] < 64;
        if (!thr) continue;
        doff[size_t(o)] = ndsm;
        ndsm += 1 << a.cp[o].m;
    }
    // the table of a diagonal with other-bit index h, as an expression prefix
    auto dtab = [&](int o) -> std::string {
        if (strided[o]) return "msm[" + std::to_string(int(a.ops[o].moff)) + " + ";
        if (doff[size_t(o)] >= 0) return "dsm[" + std::to_string(doff[size_t(o)]) + " + ";
        return "p.m[" + std::to_string(int(a.ops[o].moff)) + " + ";
    };
    const unsigned hoff_n = (1u << H) < 2u ? 2u : (1u << H);  // a 16-byte multiple
    // One tile buffer instead of two (kernels only): the next tile is fetched
    // after this one's stores, and the smaller footprint lets more CTAs share
    // an SM, whose loads and arithmetic overlap.  Measured on the 30-qubit
    // spread circuit (B200): complex128 k = 10 316.7 -> 297.5 ms (8 instead of
    // 6 CTAs per SM), complex64 k = 11 213.6 -> 226.8 ms; so the default is
    // single for complex128 and double for complex64.  QS_JIT_SINGLE_BUFFER=0/1
    // overrides it.
    const bool single = devfn == nullptr && jit_single_buffer(C128);
    const int nbuf = single ? 1 : 2;
    out.threads = threads;
    out.smem = sizeof(V) * size_t(nbuf) * (size_t(1) << K) + 8 * size_t(hoff_n) +
               (a.nexp > 0 ? sizeof(double2) * size_t(nwarps) * size_t(a.nexp) : 0) +
               (batched ? sizeof(V) * size_t(NM) : 0) + sizeof(V) * size_t(ndsm);
    out.smem = (out.smem + 15) & ~size_t(15);
    // a device function keeps its parameter block in shared memory behind the
    // rest (see its prologue); the kernels read theirs from the parameter bank
    const size_t smem_main = out.smem;
    if (devfn) out.smem += 8 * out.params.size();
    if (!with_source) return true;
    const char* VT = C128 ? "double2" : "float2";
    const char* ST = C128 ? "double" : "float";
    const char* MK = C128 ? "make_double2" : "make_float2";
    const char* FMA = C128 ? "__fma_rn" : "__fmaf_rn";
    // resident threads per SM the register budget is sized for (launch bounds);
    // QS_JIT_THREADS_PER_SM overrides it
    static const int env_target = [] {
        const char* e = getenv("QS_JIT_THREADS_PER_SM");
        return e && *e ? atoi(e) : 0;
    }();
    // 512 threads per SM; plain complex64 state-vector passes (no per-instance
    // tables, no EXPECT ops) 256, i.e. the whole register file for 64-thread
    // CTAs: on the 30-qubit spread circuit (B200, k = 11) 211.6 -> 189.7 ms
    // (384: 208.2 ms).  complex128 passes are fastest at 512 (298 ms at 640,
    // 344 ms at 768).
    const int target = env_target > 0 ? env_target : (!C128 && !batched && a.nexp == 0 ? 256 : 512);
    const int minb = threads >= target ? 1 : target / threads;
    SrcBuf g;
    g.add("// generated fused pass: n=%d K=%d L=%d R=%d stages=%d ops=%d expect=%d batched=%d\n", a.n, K, L, R,
          a.nstages, a.nops, a.nexp, int(batched));
    g.add("typedef unsigned long long u64;\ntypedef unsigned int u32;\ntypedef %s V;\ntypedef %s S;\n", VT, ST);
    g.add("static __device__ __forceinline__ V cmul(V a, V b) { V r; r.x = a.x * b.x - a.y * b.y; "
          "r.y = a.x * b.y + a.y * b.x; return r; }\n");
    g.add("static __device__ __forceinline__ V cfma(V a, V b, V c) { V r; r.x = %s(a.x, b.x, %s(-a.y, b.y, c.x)); "
          "r.y = %s(a.x, b.y, %s(a.y, b.x, c.y)); return r; }\n", FMA, FMA, FMA, FMA);
    g.add("static __device__ __forceinline__ V cadd(V a, V b) { V r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }\n");
    g.add("static __device__ __forceinline__ V cneg(V a) { V r; r.x = -a.x; r.y = -a.y; return r; }\n");
    g.add("static __device__ __forceinline__ V csel(bool c, V a, V b) { V r; r.x = c ? a.x : b.x; "
          "r.y = c ? a.y : b.y; return r; }\n");
    // products with a real entry a (rmul / rfma) or an imaginary one i*b (imul / ifma)
    g.add("static __device__ __forceinline__ V rmul(S a, V v) { V r; r.x = a * v.x; r.y = a * v.y; return r; }\n");
    g.add("static __device__ __forceinline__ V rfma(S a, V v, V c) { V r; r.x = %s(a, v.x, c.x); "
          "r.y = %s(a, v.y, c.y); return r; }\n", FMA, FMA);
    g.add("static __device__ __forceinline__ V imul(S b, V v) { V r; r.x = -b * v.y; r.y = b * v.x; return r; }\n");
    g.add("static __device__ __forceinline__ V ifma(S b, V v, V c) { V r; r.x = %s(-b, v.y, c.x); "
          "r.y = %s(b, v.x, c.y); return r; }\n", FMA, FMA);
    g.add("struct __align__(16) P { V m[%d]; u64 ntiles; u64 gthr[8]; u64 gslot[%d]; u64 hibit[16]; u64 gctrl[%d]; "
          "u64 hsh[%d]; u64 mgoff[%d]; u64 mstride[%d]; u64 eslot[%d]; u64 misc[2];%s };\n", NM, E, NOPS, 4 * NOPS,
          NOPS, NOPS, NEXP, batched ? (" u32 pe[" + std::to_string(NM) + "];").c_str() : "");
    // cooperative loops (no per-thread layout): all threads of the CTA
    const std::string CT = devfn ? "threadIdx.x" : "tid";
    const std::string CS = devfn ? "blockDim.x" : std::to_string(threads) + "u";
    if (devfn) {
        g.add("extern \"C\" __device__ void %s(V* __restrict__ vec, const void* __restrict__ pv, "
              "const V* __restrict__ mats, double* __restrict__ partials, u64 tile, const u64 tend, "
              "const u32 zero_in) {\n", devfn);
    } else {
        g.add("extern \"C\" __global__ void __launch_bounds__(%d, %d) qs_pass(V* __restrict__ vec, "
              "const __grid_constant__ P p, const V* __restrict__ mats, double* __restrict__ partials) {\n", threads,
              minb);
    }
    g.add("  extern __shared__ __align__(16) unsigned char smem_raw[];\n");
    if (devfn) {
        // the parameter block moves from the plan (global memory) to shared
        // memory behind the tile buffers: matrix entries are read at shared-
        // memory latency, as the kernels read them from the constant bank
        g.add("  { const uint4* __restrict__ src = reinterpret_cast<const uint4*>(pv);\n"
              "    uint4* dst = reinterpret_cast<uint4*>(smem_raw + %zuu);\n"
              "    for (u32 i = threadIdx.x; i < %zuu; i += blockDim.x) dst[i] = src[i]; }\n"
              "  __syncthreads();\n  const P& p = *reinterpret_cast<const P*>(smem_raw + %zuu);\n",
              smem_main, out.params.size() / 2, smem_main);
    }
    g.add("  V* const b0 = reinterpret_cast<V*>(smem_raw);\n  V* const b1 = b0 + %du;\n", single ? 0u : 1u << K);
    g.add("  u64* const hoff = reinterpret_cast<u64*>(b1 + %du);\n", 1u << K);
    g.add("  double2* const ered = reinterpret_cast<double2*>(hoff + %du);\n", hoff_n);
    g.add("  V* const msm = reinterpret_cast<V*>(ered + %d);\n", a.nexp > 0 ? nwarps * a.nexp : 0);
    g.add("  V* const dsm = msm + %d;\n", batched ? NM : 0);
    if (devfn) g.add("  const u32 tid = threadIdx.x & %du;\n  const bool act = threadIdx.x < %du;\n",
                     unsigned(threads - 1), unsigned(threads));
    else g.add("  const u32 tid = threadIdx.x;\n");
    g.add("  for (u32 j = %s; j < %du; j += %s) { u64 o = 0;\n", CT.c_str(), 1u << H, CS.c_str());
    g.add("#pragma unroll\n    for (int t = 0; t < %d; ++t) if ((j >> t) & 1u) o |= p.hibit[t];\n    hoff[j] = o; }\n", H);
    for (int o = 0; o < a.nops; ++o)
        if (doff[size_t(o)] >= 0)
            g.add("  for (u32 q = %s; q < %du; q += %s) dsm[%d + q] = p.m[%d + q];\n", CT.c_str(), 1u << a.cp[o].m,
                  CS.c_str(), doff[size_t(o)], int(a.ops[o].moff));
    g.add("  u64 gthr = 0;\n");
    for (int i = 0; i < nT; ++i) g.add("  if ((tid >> %d) & 1u) gthr |= p.gthr[%d];\n", i, i);
    for (int si = 0; si < a.nstages; ++si) {
        const KStage& S = a.st[si];
        uint32_t rt[8], wt[8], tb[8];
        for (int i = 0; i < 8; ++i) {
            rt[i] = S.rthr[i];
            wt[i] = S.wthr[i];
            tb[i] = S.tbit[i];
        }
        g.add("  const u32 RD%d = %s;\n", si, thread_xor_expr(rt, nT).c_str());
        if (si > 0) g.add("  const u32 WR%d = %s;\n", si, thread_xor_expr(wt, nT).c_str());
        g.add("  const u32 TH%d = %s;\n", si, thread_xor_expr(tb, nT).c_str());
    }
    g.add("  const u64 ntiles = p.ntiles;\n");
    g.add("  auto tile_base = [&](u64 t) -> u64 { u64 b = t << %d;\n", L);
    g.add("#pragma unroll\n    for (int i = 0; i < %d; ++i) { const u64 lo = p.hibit[i] - 1ull; "
          "b = ((b & ~lo) << 1) | (b & lo); }\n    return b; };\n", H);
    if (devfn) {  // the caller's tile range
        g.add("  const u64 tstep = 1;\n");
        if (batched) g.add("  u64 staged = ~0ull;\n");
    } else if (batched) {
        // per-instance tables: contiguous runs of tiles per CTA, so that a CTA
        // restages its instance's matrices once per instance
        g.add("  const u64 chunk = (ntiles + gridDim.x - 1) / gridDim.x;\n");
        g.add("  u64 tile = u64(blockIdx.x) * chunk;\n  const u64 tend = tile + chunk < ntiles ? tile + chunk : ntiles;\n");
        g.add("  const u64 tstep = 1;\n  u64 staged = ~0ull;\n");
    } else {
        g.add("  u64 tile = blockIdx.x;\n  const u64 tend = ntiles;\n  const u64 tstep = gridDim.x;\n");
    }
    g.add("  __syncthreads();\n");
    const int EPC = 16 / int(sizeof(V));
    g.add("  auto prefetch = [&](V* dst, u64 base) {\n");
    if (devfn)
        g.add("    if (zero_in) { for (u32 e = threadIdx.x; e < %du; e += blockDim.x) { V z; z.x = (base == 0 && e == 0) "
              "? 1 : 0; z.y = 0; dst[e] = z; } } else\n", 1u << K);
    g.add("    for (u32 c = %s; c < %du; c += %s) { const u32 e = c * %du;\n", CT.c_str(), (1u << K) / EPC, CS.c_str(),
          EPC);
    g.add("      const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(dst + e));\n");
    g.add("      asm volatile(\"cp.async.cg.shared.global [%%0], [%%1], 16;\\n\" :: \"r\"(sa), "
          "\"l\"(vec + (base | hoff[e >> %d] | (e & %du))) : \"memory\"); }\n", L, (1u << L) - 1u);
    g.add("    asm volatile(\"cp.async.commit_group;\\n\" ::: \"memory\"); };\n");
    g.add("  if (tile < tend) prefetch(b0, tile_base(tile));\n");
    g.add("  for (u32 it = 0; tile < tend; ++it, tile += tstep) {\n");
    g.add("    V* const cur = (it & 1u) ? b1 : b0;\n    const u64 base = tile_base(tile);\n");
    g.add("    asm volatile(\"cp.async.wait_group 0;\\n\" ::: \"memory\");\n    __syncthreads();\n");
    if (!single) g.add("    if (tile + tstep < tend) prefetch((it & 1u) ? b0 : b1, tile_base(tile + tstep));\n");
    if (batched) {
        g.add("    { const u64 inst = (base & p.misc[0]) >> p.misc[1];\n");
        g.add("      if (inst != staged) {\n");
        g.add("        for (u32 q = %s; q < %du; q += %s) { const u32 v = p.pe[q];\n", CT.c_str(), unsigned(a.nmats),
              CS.c_str());
        g.add("          if (v >> 31) { const u32 o = (v >> 16) & 0x7fffu; "
              "msm[q] = mats[p.mgoff[o] + inst * p.mstride[o] + (v & 0xffffu)]; } }\n");
        g.add("        staged = inst;\n        __syncthreads();\n      } }\n");
    }
    // ---- body
    int fresh = 0;
    std::vector<int> var(E);  // slot -> SSA value id
    auto vname = [&](int id) { return "v" + std::to_string(id); };
    auto slot_addr = [&](const uint16_t* img, int s) {
        uint32_t c = 0;
        for (int j = 0; j < R; ++j)
            if ((s >> j) & 1) c ^= img[j];
        return c;
    };
    // the sum over the nonzero entries of one row of a (slot-order) matrix
    auto row_expr = [&](int o, int base_idx, int D, const int* in) -> std::string {
        std::string e;
        for (int c = 0; c < D; ++c) {
            const int idx = base_idx + c;
            const int cl = vclass(o, idx);
            if (cl == 0) continue;
            const std::string x = vname(in[c]);
            const std::string m = mref(o, idx);
            if (e.empty()) {
                if (cl == 1) e = x;
                else if (cl == 2) e = "cneg(" + x + ")";
                else if (cl == 4) e = "rmul(" + m + ".x, " + x + ")";
                else if (cl == 5) e = "imul(" + m + ".y, " + x + ")";
                else e = "cmul(" + m + ", " + x + ")";
            } else {
                if (cl == 1) e = "cadd(" + e + ", " + x + ")";
                else if (cl == 2) e = "cadd(" + e + ", cneg(" + x + "))";
                else if (cl == 4) e = "rfma(" + m + ".x, " + x + ", " + e + ")";
                else if (cl == 5) e = "ifma(" + m + ".y, " + x + ", " + e + ")";
                else e = "cfma(" + m + ", " + x + ", " + e + ")";
            }
        }
        if (e.empty()) e = std::string(MK) + "(0, 0)";
        return e;
    };
    // thread-dependent / outside-tile index bits of a diagonal (h), as an expression
    auto h_expr = [&](const KOp& op, int o, int si) -> std::string {
        std::string h;
        for (int q = 0; q < op.nh; ++q) {
            const int src = op.hsrc[q];
            const std::string t = src < 64 ? "((TH" + std::to_string(si) + " >> " + std::to_string(src) + ") & 1u)"
                                            : "u32((base >> p.hsh[" + std::to_string(4 * o + q) + "]) & 1ull)";
            h = h.empty() ? t : "((" + h + ") << 1) | " + t;
        }
        return h;
    };
    for (int s = 0; s < E; ++s) {
        var[s] = fresh++;
        g.add("    const V v%d = cur[RD0 ^ %uu];\n", var[s], slot_addr(a.st[0].rslot, s));
    }
    for (int si = 0; si < a.nstages; ++si) {
        const KStage& S = a.st[si];
        if (si > 0) {
            g.add("    __syncthreads();\n");
            for (int s = 0; s < E; ++s) g.add("    cur[WR%d ^ %uu] = v%d;\n", si, slot_addr(S.wslot, s), var[s]);
            g.add("    __syncthreads();\n");
            for (int s = 0; s < E; ++s) {
                var[s] = fresh++;
                g.add("    const V v%d = cur[RD%d ^ %uu];\n", var[s], si, slot_addr(S.rslot, s));
            }
        }
        for (int o = S.op_begin; o < S.op_begin + S.op_count; ++o) {
            const KOp& op = a.ops[o];
            std::string cond;
            if (op.gctrl) cond = "((base & p.gctrl[" + std::to_string(o) + "]) == p.gctrl[" + std::to_string(o) + "])";
            if (op.tctrl) {
                const std::string tc = std::to_string(unsigned(op.tctrl)) + "u";
                cond += (cond.empty() ? "" : " && ") + std::string("((TH") + std::to_string(si) + " & " + tc +
                        ") == " + tc + ")";
            }
            const int scm = op.scm;
            auto ctrl_ok = [&](int s) { return (s & scm) == scm; };
            if (!cond.empty() && op.code != QS_OP_EXPECT) g.add("    const bool c%d = %s;\n", o, cond.c_str());
            if (op.code == QS_OP_MAT) {
                const int mask = op.mask, M = popc_c(mask), D = 1 << M;
                g.add("    // op %d: dense on slot mask %d\n", o, mask);
                for (int s = 0; s < E; ++s) {
                    if ((s & mask) || !ctrl_ok(s)) continue;
                    int in[16], outid[16];
                    for (int c = 0; c < D; ++c) in[c] = var[s | pdep_c(c, mask)];
                    for (int r = 0; r < D; ++r) {
                        const std::string e = row_expr(o, op.moff + r * D, D, in);
                        outid[r] = fresh++;
                        if (cond.empty()) g.s += "    const V " + vname(outid[r]) + " = " + e + ";\n";
                        else g.s += "    const V " + vname(outid[r]) + " = c" + std::to_string(o) + " ? " + e + " : " +
                                    vname(in[r]) + ";\n";
                    }
                    for (int r = 0; r < D; ++r) var[s | pdep_c(r, mask)] = outid[r];
                }
            } else if (op.code == QS_OP_ANTI || op.code == QS_OP_SWAP) {  // plain exchanges
                int b0, b1;
                if (op.code == QS_OP_ANTI) {
                    b0 = 0;
                    b1 = op.mask;
                } else {
                    b0 = 1 << nth_bit(op.mask, 0);
                    b1 = 1 << nth_bit(op.mask, 1);
                }
                for (int s = 0; s < E; ++s) {
                    if ((s & op.mask) || !ctrl_ok(s)) continue;
                    const int x0 = var[s | b0], x1 = var[s | b1];
                    if (cond.empty()) {
                        var[s | b0] = x1;
                        var[s | b1] = x0;
                    } else {
                        const int n0 = fresh++, n1 = fresh++;
                        g.add("    const V v%d = csel(c%d, v%d, v%d);\n", n0, o, x1, x0);
                        g.add("    const V v%d = csel(c%d, v%d, v%d);\n", n1, o, x0, x1);
                        var[s | b0] = n0;
                        var[s | b1] = n1;
                    }
                }
            } else if (op.code == QS_OP_DIAG) {
                g.add("    // op %d: diagonal, %d register bits, %d other bits\n", o, op.ns, op.nh);
                if (op.nh > 0) g.s += "    const u32 h" + std::to_string(o) + " = " + h_expr(op, o, si) + ";\n";
                for (int s = 0; s < E; ++s) {
                    if (!ctrl_ok(s)) continue;
                    const int k = op.kidx[s];
                    std::string e;
                    if (op.nh == 0) {
                        const int idx = op.moff + k;
                        const int cl = vclass(o, idx);
                        if (cl == 1) continue;
                        if (cl == 2) e = "cneg(" + vname(var[s]) + ")";
                        else if (cl == 0) e = std::string(MK) + "(0, 0)";
                        else if (cl == 4) e = "rmul(" + mref(o, idx) + ".x, " + vname(var[s]) + ")";
                        else if (cl == 5) e = "imul(" + mref(o, idx) + ".y, " + vname(var[s]) + ")";
                        else e = "cmul(" + vname(var[s]) + ", " + mref(o, idx) + ")";
                    } else {
                        e = "cmul(" + vname(var[s]) + ", " + dtab(o) + "((h" + std::to_string(o) + " << " +
                            std::to_string(int(op.ns)) + ") | " + std::to_string(k) + "u)])";
                    }
                    const int nid = fresh++;
                    if (cond.empty()) g.s += "    const V " + vname(nid) + " = " + e + ";\n";
                    else g.s += "    const V " + vname(nid) + " = c" + std::to_string(o) + " ? " + e + " : " +
                                vname(var[s]) + ";\n";
                    var[s] = nid;
                }
            } else if (op.code == QS_OP_EXPECT) {
                // sum over the thread's psi/lam pairs (slot bit 0 = pair bit) of
                // conj(lam) (G psi) in the state's precision, then a warp sum in FP64
                if (!cond.empty() || scm != 0 || pair_tile < 0 || S.R[0] != pair_tile) return false;
                g.add("    { // op %d: <lam| G |psi>\n      S pr = 0, pi = 0;\n", o);
                const bool dg = op.flags & QS_OPF_DIAG;
                if (dg && op.nh > 0) g.s += "      const u32 h" + std::to_string(o) + " = " + h_expr(op, o, si) + ";\n";
                if (dg) {
                    for (int s = 0; s < E; s += 2) {
                        const int k = op.kidx[s];
                        std::string d = op.nh == 0 ? mref(o, op.moff + k)
                                                   : dtab(o) + "((h" + std::to_string(o) + " << " +
                                                         std::to_string(int(op.ns)) + ") | " + std::to_string(k) +
                                                         "u)]";
                        g.s += "      { const V acc = cmul(" + d + ", " + vname(var[s]) + "); const V l = " +
                               vname(var[s | 1]) + ";\n";
                        g.s += "        pr += l.x * acc.x + l.y * acc.y; pi += l.x * acc.y - l.y * acc.x; }\n";
                    }
                } else {
                    const int mask = op.mask, M = popc_c(mask), D = 1 << M;
                    if ((mask & 1) || M > 2) return false;
                    for (int s = 0; s < E; ++s) {
                        if ((s & mask) || (s & 1)) continue;
                        int in[4];
                        for (int c = 0; c < D; ++c) in[c] = var[s | pdep_c(c, mask)];
                        for (int r = 0; r < D; ++r) {
                            g.s += "      { const V acc = " + row_expr(o, op.moff + r * D, D, in) + "; const V l = " +
                                   vname(var[s | 1 | pdep_c(r, mask)]) + ";\n";
                            g.s += "        pr += l.x * acc.x + l.y * acc.y; pi += l.x * acc.y - l.y * acc.x; }\n";
                        }
                    }
                }
                g.add("      double re = pr, im = pi;\n");
                g.add("#pragma unroll\n      for (int off = 16; off > 0; off >>= 1) { re += __shfl_xor_sync(0xffffffffu, "
                      "re, off); im += __shfl_xor_sync(0xffffffffu, im, off); }\n");
                g.add("      if ((tid & 31u) == 0) ered[(tid >> 5) * %d + %d] = make_double2(re, im);\n    }\n", NEXP,
                      int(op.elocal));
            } else {
                return false;
            }
        }
    }
    if (devfn) g.add("    if (act) {\n");
    for (int s = 0; s < E; ++s) g.add("    vec[base | gthr | p.gslot[%d]] = v%d;\n", s, var[s]);
    if (devfn) g.add("    }\n");
    if (a.nexp > 0) {
        // per-tile partials: the warps' sums in a fixed order
        g.add("    __syncthreads();\n");
        g.add("    for (u32 e = %s; e < %du; e += %s) { double2 t = make_double2(0.0, 0.0);\n", CT.c_str(),
              unsigned(a.nexp), CS.c_str());
        g.add("      for (int w = 0; w < %d; ++w) { t.x += ered[w * %d + e].x; t.y += ered[w * %d + e].y; }\n", nwarps,
              NEXP, NEXP);
        g.add("      const u64 at = 2 * (p.eslot[e] * ntiles + tile);\n      partials[at] = t.x;\n"
              "      partials[at + 1] = t.y; }\n");
    }
    if (single)  // every thread is past its last read of the buffer
        g.add("    __syncthreads();\n    if (tile + tstep < tend) prefetch(b0, tile_base(tile + tstep));\n");
    g.add("  }\n}\n");
    if (g.truncated) return false;
    out.src.swap(g.s);
    return true;
}

// Launch memo: a planned register pass (the used parts of its RegArgs) and its
// parameter block determine the generated source completely, so repeated
// launches of the same plan (a replayed circuit, a gradient loop) reuse the
// loaded kernel without generating and hashing the source again.
struct JitMemo {
    std::string src;       // kept until the kernel is ready on some device
    void* fn[64] = {nullptr};
    int occ[64] = {0};
};

uint64_t fnv(uint64_t h, const void* p, size_t n) {
    const unsigned char* c = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < n; ++i) h = (h ^ c[i]) * 1099511628211ull;
    return h;
}

// The source depends on the plan's structure and on the entries' value
// classes, not on the matrix values: the key hashes exactly those, so a new
// parameter set of the same circuit reuses the compiled kernel.
uint64_t plan_key(const RegArgs& a, int R, size_t vsize, const std::vector<uint8_t>& classes) {
    uint64_t h = 1469598103934665603ull;
    const int hdr[] = {a.n, a.K, a.L, a.H, a.nT, a.nstages, a.nops, a.nmats, a.inst_shift, a.batched, a.nexp,
                       R, int(vsize)};
    h = fnv(h, hdr, sizeof(hdr));
    h = fnv(h, &a.pairmask, sizeof(a.pairmask));
    h = fnv(h, a.hi, sizeof(int) * size_t(a.H));
    h = fnv(h, a.eslot, sizeof(int) * size_t(a.nexp));
    h = fnv(h, a.st, sizeof(KStage) * size_t(a.nstages));
    h = fnv(h, a.ops, sizeof(KOp) * size_t(a.nops));
    for (int o = 0; o < a.nops; ++o) {  // the table layout, not where the tables sit (goff)
        const KCopy& c = a.cp[o];
        const int f[] = {int(c.soff), int(c.m), int(c.diag), int(c.stride != 0), c.perm[0], c.perm[1], c.perm[2],
                         c.perm[3]};
        h = fnv(h, f, sizeof(f));
    }
    static const int target = [] {
        const char* e = getenv("QS_JIT_THREADS_PER_SM");
        return e && *e ? atoi(e) : 0;
    }();
    h = fnv(h, &target, sizeof(target));
    const int single = jit_single_buffer(vsize == 16) ? 1 : 0;
    h = fnv(h, &single, sizeof(single));
    return fnv(h, classes.data(), classes.size());
}

// Launch the run-time compiled kernel of a planned register pass, if the
// compiler has it ready (mode SYNC: after compiling it); returns 1 when it
// was launched, 0 when the generic kernel has to run, < 0 on error.
template <typename V>
int launch_jit(V* vec, const RegArgs& args, int R, const V* hm, const V* mats, double* partials, cudaStream_t st) {
    const int jm = jit::mode();
    if (jm == QS_JIT_OFF || hm == nullptr) return 0;
    static thread_local JitPass jp;
    if (!gen_reg_pass<V>(args, R, hm, jp, false)) return 0;
    // during stream capture nothing is compiled or loaded: a kernel that is
    // not loaded yet on this device leaves the pass to the generic kernel
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) cs = cudaStreamCaptureStatusActive;
    const bool capturing = cs != cudaStreamCaptureStatusNone;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
    static std::mutex memo_mu;
    static std::unordered_map<uint64_t, std::shared_ptr<JitMemo>> memo;
    const uint64_t key = plan_key(args, R, sizeof(V), jp.classes);
    std::shared_ptr<JitMemo> m;
    {
        std::lock_guard<std::mutex> lock(memo_mu);
        auto it = memo.find(key);
        if (it != memo.end()) m = it->second;
    }
    void* fn = m ? m->fn[dev] : nullptr;
    int occ = m ? m->occ[dev] : 0;
    if (fn == nullptr) {
        if (!m) {
            m = std::make_shared<JitMemo>();
            JitPass full;
            if (!gen_reg_pass<V>(args, R, hm, full, true)) return 0;
            m->src.swap(full.src);
            std::lock_guard<std::mutex> lock(memo_mu);
            if (memo.size() > 4096) memo.clear();  // bounded: plans are cheap to regenerate
            memo[key] = m;
        }
        if (m->src.empty()) {  // loaded on another device only: regenerate the text
            JitPass full;
            if (!gen_reg_pass<V>(args, R, hm, full, true)) return 0;
            m->src.swap(full.src);
        }
        fn = jit::lookup(m->src, "qs_pass", jm == QS_JIT_SYNC && !capturing, !capturing, jp.threads, jp.smem, &occ);
        if (fn != nullptr) {
            std::lock_guard<std::mutex> lock(memo_mu);
            m->fn[dev] = fn;
            m->occ[dev] = occ;
            std::string().swap(m->src);
        }
    }
    if (fn == nullptr) {
        jit::count_launch(false);
        return 0;
    }
    if (occ < 1) occ = 1;
    int rc;
    const uint64_t ntiles = uint64_t(1) << (args.n - args.K);
    const uint64_t cap = uint64_t(sm_count()) * uint64_t(occ);
    void* vp = vec;
    const void* mp = mats;
    void* pp = partials;
    void* params[] = {&vp, jp.params.data(), &mp, &pp};
    rc = jit::launch(fn, unsigned(ntiles < cap ? ntiles : cap), unsigned(jp.threads), jp.smem, st, params);
    if (rc) return rc;
    jit::count_launch(true);
    return 1;
}

// Register bits per thread of generated passes: the generic kernel's (4 for
// complex128, 5 for complex64) unless QS_JIT_REG_BITS says otherwise (4 or 5).
inline int jit_reg_bits(int generic_r) {
    static const int env_r = [] {
        const char* e = getenv("QS_JIT_REG_BITS");
        const int v = e && *e ? atoi(e) : 0;
        return (v == 4 || v == 5) ? v : 0;
    }();
    return env_r ? env_r : generic_r;
}

template <typename V, int R, bool EXP, bool BIG>
int launch_reg_k(V* vec, int n, const qs_pass& ps, const qs_op* ops, const V* mats, double* partials, cudaStream_t st,
                 const V* hm = nullptr) {
    static thread_local RegArgs args;
    config_smem((const void*)k_fused_reg<V, R, EXP, BIG>);
    std::vector<int> rem(ps.op_count);
    for (int i = 0; i < ps.op_count; ++i) rem[i] = i;
    const int nb = sizeof(V) == 16 ? 3 : 4;  // bank-group bits of a shared-memory phase
    const int RJ = jit_reg_bits(R);
    while (!rem.empty()) {
        const int next = ps.op_begin + rem.front();
        if (!EXP && RJ != R && ps.k - RJ >= 5 && ps.k - RJ <= 8) {
            // a generated pass with its own register width plans its own launch;
            // the generic kernel re-plans the same ops when it is not ready
            std::vector<int> saved = rem;
            if (build_reg(ps, ops, rem, n, RJ, nb, args) > 0) {
                int jr = launch_jit<V>(vec, args, RJ, hm, mats, partials, st);
                if (jr < 0) return jr;
                if (jr == 1) continue;
            }
            rem.swap(saved);
        }
        int used = build_reg(ps, ops, rem, n, R, nb, args);
        if (used <= 0) {
            set_error("qs_apply_fused: op %d does not fit a register tile", next);
            return QS_EINVAL;
        }
        if (EXP || RJ == R) {
            int jr = launch_jit<V>(vec, args, R, hm, mats, partials, st);
            if (jr < 0) return jr;
            if (jr == 1) continue;
        }
        const int threads = 1 << (ps.k - R);
        const size_t smem = reg_smem_bytes<V>(args, R, EXP);
        if (smem > size_t(smem_optin())) {
            set_error("qs_apply_fused: a register pass needs %zu bytes of shared memory", smem);
            return QS_EINVAL;
        }
        uint64_t ntiles = uint64_t(1) << (n - ps.k);
        // persistent grid: as many CTAs as fit on the SMs at once (smaller
        // tiles run several CTAs per SM, whose relayouts and arithmetic overlap)
        int occ = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_fused_reg<V, R, EXP, BIG>, threads, smem);
        if (occ < 1) occ = 1;
        uint64_t cap = uint64_t(sm_count()) * uint64_t(occ);
        k_fused_reg<V, R, EXP, BIG><<<unsigned(ntiles < cap ? ntiles : cap), threads, smem, st>>>(vec, args, mats, partials);
        QS_CHECK_LAUNCH(EXP ? "qs_adjoint_pair" : "qs_apply_fused(reg)");
    }
    return QS_OK;
}

// Dense ops on 3 or 4 targets, and controlled dense ops, need the BIG kernel
// variant (adjoint pair passes take dense ops on at most 2 bits; their BIG
// variant only adds the controlled paths).
template <typename V, int R, bool EXP>
int launch_reg(V* vec, int n, const qs_pass& ps, const qs_op* ops, const V* mats, double* partials, cudaStream_t st,
               const V* hm = nullptr) {
    bool big = false;
    for (int i = 0; i < ps.op_count; ++i) {
        const qs_op& op = ops[ps.op_begin + i];
        const bool diag = op.kind == QS_OP_DIAG || (op.kind == QS_OP_EXPECT && (op.flags & QS_OPF_DIAG));
        if (op.m >= 3 && !diag) big = true;
        // dense here: MAT, and the anti-diagonal / swap ops that are not plain
        // exchanges (they run as dense matrices)
        const bool dense = op.kind == QS_OP_MAT ||
                           ((op.kind == QS_OP_ANTI || op.kind == QS_OP_SWAP) && !(op.flags & QS_OPF_UNIT));
        if (dense && op.lctrl != 0) big = true;
    }
    if constexpr (EXP) {
        for (int i = 0; i < ps.op_count; ++i) {
            const qs_op& op = ops[ps.op_begin + i];
            const bool diag = op.kind == QS_OP_DIAG || (op.kind == QS_OP_EXPECT && (op.flags & QS_OPF_DIAG));
            if (op.m >= 3 && !diag) {
                set_error("qs_adjoint_pair: pass ops act densely on at most 2 bits");
                return QS_EINVAL;
            }
        }
        return big ? launch_reg_k<V, R, true, true>(vec, n, ps, ops, mats, partials, st, hm)
                   : launch_reg_k<V, R, true, false>(vec, n, ps, ops, mats, partials, st, hm);
    } else {
        return big ? launch_reg_k<V, R, false, true>(vec, n, ps, ops, mats, partials, st, hm)
                   : launch_reg_k<V, R, false, false>(vec, n, ps, ops, mats, partials, st, hm);
    }
}

template <typename V>
constexpr int reg_bits() { return sizeof(V) == 16 ? 4 : 5; }

template <typename V>
int launch_pass(V* vec, int n, const qs_pass& ps, const qs_op* ops, const V* mats, cudaStream_t st,
                const V* hm = nullptr) {
    constexpr int R = reg_bits<V>();
    const int nT = ps.k - R;
    const size_t smem = sizeof(V) * (2 * (size_t(1) << ps.k) + QS_MAX_PASS_MATS) + 8 * ((size_t(1) << (ps.k - ps.nlow)) + (1 << R)) +
                        sizeof(KOp) * QS_MAX_PASS_OPS + 16 + sizeof(KStage) * kMaxStages + QS_MAX_PASS_MATS;
    if (nT >= 5 && nT <= 8 && ps.nlow >= 5 && smem <= size_t(smem_optin()))
        return launch_reg<V, R, false>(vec, n, ps, ops, mats, nullptr, st, hm);
    return launch_smem<V, false>(vec, nullptr, n, ps, ops, mats, nullptr, st);
}

}  // namespace

bool gen_batch_pass(const void* regargs, int R, bool c128, const void* mats_host, const char* name, std::string* src,
                    std::vector<uint64_t>* params, size_t* smem, int* threads) {
    const RegArgs& a = *static_cast<const RegArgs*>(regargs);
    JitPass jp;
    const bool ok = c128 ? gen_reg_pass<double2>(a, R, static_cast<const double2*>(mats_host), jp, true, name)
                         : gen_reg_pass<float2>(a, R, static_cast<const float2*>(mats_host), jp, true, name);
    if (!ok) return false;
    src->swap(jp.src);
    params->swap(jp.params);
    *smem = jp.smem;
    *threads = jp.threads;
    return true;
}

}  // namespace qs

using namespace qs;

extern "C" int qs_apply_fused(void* vec, int n, int dtype, const qs_pass* passes, int npasses, const qs_op* ops,
                              int64_t nops_total, const void* mats_dev, int64_t mats_count, void* stream) {
    return qs_apply_fused_ex(vec, n, dtype, passes, npasses, ops, nops_total, mats_dev, nullptr, mats_count, stream);
}

extern "C" int qs_apply_fused_ex(void* vec, int n, int dtype, const qs_pass* passes, int npasses, const qs_op* ops,
                                 int64_t nops_total, const void* mats_dev, const void* mats_host, int64_t mats_count,
                                 void* stream) {
    QS_REQUIRE(vec != nullptr, "null state vector");
    QS_REQUIRE(n >= 1 && n <= 40, "qubit count %d outside [1, 40]", n);
    QS_REQUIRE(valid_dtype(dtype), "bad dtype %d", dtype);
    QS_REQUIRE(npasses >= 0 && (npasses == 0 || passes != nullptr), "bad pass array");
    QS_REQUIRE(nops_total >= 0 && (nops_total == 0 || ops != nullptr), "bad op array");
    QS_REQUIRE(mats_count >= 0 && (mats_count == 0 || mats_dev != nullptr), "bad matrix table");
    size_t vsize = dtype == QS_C128 ? 16 : 8;
    for (int i = 0; i < npasses; ++i) {
        int rc = validate_pass(passes[i], n, ops, nops_total, mats_count);
        if (rc) return rc;
        size_t smem = vsize * (size_t(1) << passes[i].k) + 8 * (size_t(1) << (passes[i].k - passes[i].nlow));
        QS_REQUIRE(smem <= 160 * 1024, "pass %d: tile of 2^%d needs %zu bytes of shared memory", i, passes[i].k, smem);
    }
    for (int i = 0; i < npasses; ++i) {
        if (passes[i].op_count == 0) continue;
        int rc = dtype == QS_C128
                     ? launch_pass<double2>((double2*)vec, n, passes[i], ops, (const double2*)mats_dev,
                                            as_stream(stream), (const double2*)mats_host)
                     : launch_pass<float2>((float2*)vec, n, passes[i], ops, (const float2*)mats_dev,
                                           as_stream(stream), (const float2*)mats_host);
        if (rc) return rc;
    }
    return QS_OK;
}

extern "C" int qs_adjoint_fused(void* psi, void* lam, int n, int dtype, const qs_pass* passes, int npasses,
                                const qs_op* ops, int64_t nops_total, const void* mats_dev, int64_t mats_count,
                                double* partials_dev, int64_t partials_count, void* stream) {
    QS_REQUIRE(psi != nullptr && lam != nullptr && psi != lam, "psi and lam must be distinct non-null vectors");
    QS_REQUIRE(n >= 1 && n <= 40, "qubit count %d outside [1, 40]", n);
    QS_REQUIRE(valid_dtype(dtype), "bad dtype %d", dtype);
    QS_REQUIRE(npasses >= 0 && (npasses == 0 || passes != nullptr), "bad pass array");
    QS_REQUIRE(nops_total >= 0 && (nops_total == 0 || ops != nullptr), "bad op array");
    QS_REQUIRE(mats_count >= 0 && (mats_count == 0 || mats_dev != nullptr), "bad matrix table");
    QS_REQUIRE(partials_count >= 0 && (partials_count == 0 || partials_dev != nullptr), "bad partials buffer");
    size_t vsize = dtype == QS_C128 ? 16 : 8;
    for (int i = 0; i < npasses; ++i) {
        int rc = validate_pass(passes[i], n, ops, nops_total, mats_count, true, partials_count);
        if (rc) return rc;
        size_t smem = 2 * vsize * (size_t(1) << passes[i].k) + 8 * (size_t(1) << (passes[i].k - passes[i].nlow));
        QS_REQUIRE(smem <= 160 * 1024, "pass %d: two tiles of 2^%d need %zu bytes of shared memory", i,
                   passes[i].k, smem);
    }
    for (int i = 0; i < npasses; ++i) {
        if (passes[i].op_count == 0) continue;
        int rc = dtype == QS_C128
                     ? launch_smem<double2, true>((double2*)psi, (double2*)lam, n, passes[i], ops,
                                                  (const double2*)mats_dev, partials_dev, as_stream(stream))
                     : launch_smem<float2, true>((float2*)psi, (float2*)lam, n, passes[i], ops,
                                                 (const float2*)mats_dev, partials_dev, as_stream(stream));
        if (rc) return rc;
    }
    return QS_OK;
}

extern "C" int qs_adjoint_pair(void* psilam, int n, int dtype, const qs_pass* passes, int npasses, const qs_op* ops,
                               int64_t nops_total, const void* mats_dev, int64_t mats_count, double* partials_dev,
                               int64_t partials_count, void* stream) {
    return qs_adjoint_pair_ex(psilam, n, dtype, passes, npasses, ops, nops_total, mats_dev, nullptr, mats_count,
                              partials_dev, partials_count, stream);
}

extern "C" int qs_adjoint_pair_ex(void* psilam, int n, int dtype, const qs_pass* passes, int npasses,
                                  const qs_op* ops, int64_t nops_total, const void* mats_dev, const void* mats_host,
                                  int64_t mats_count, double* partials_dev, int64_t partials_count, void* stream) {
    QS_REQUIRE(psilam != nullptr, "null vector");
    QS_REQUIRE(n >= 2 && n <= 41, "bit count %d outside [2, 41]", n);
    QS_REQUIRE(valid_dtype(dtype), "bad dtype %d", dtype);
    QS_REQUIRE(npasses >= 0 && (npasses == 0 || passes != nullptr), "bad pass array");
    QS_REQUIRE(nops_total >= 0 && (nops_total == 0 || ops != nullptr), "bad op array");
    QS_REQUIRE(mats_count >= 0 && (mats_count == 0 || mats_dev != nullptr), "bad matrix table");
    QS_REQUIRE(partials_count >= 0 && (partials_count == 0 || partials_dev != nullptr), "bad partials buffer");
    const int R = dtype == QS_C128 ? reg_bits<double2>() : reg_bits<float2>();
    for (int i = 0; i < npasses; ++i) {
        int rc = validate_pass(passes[i], n, ops, nops_total, mats_count, true, partials_count);
        if (rc) return rc;
        QS_REQUIRE(passes[i].pair > 0, "pass %d: no pair bit", i);
        const int nT = passes[i].k - R;
        QS_REQUIRE(nT >= 5 && nT <= 8 && passes[i].nlow >= 5, "pass %d: tile 2^%d / nlow %d is not a register tile", i,
                   passes[i].k, passes[i].nlow);
    }
    for (int i = 0; i < npasses; ++i) {
        if (passes[i].op_count == 0) continue;
        int rc = dtype == QS_C128
                     ? launch_reg<double2, reg_bits<double2>(), true>((double2*)psilam, n, passes[i], ops,
                                                                      (const double2*)mats_dev, partials_dev,
                                                                      as_stream(stream), (const double2*)mats_host)
                     : launch_reg<float2, reg_bits<float2>(), true>((float2*)psilam, n, passes[i], ops,
                                                                    (const float2*)mats_dev, partials_dev,
                                                                    as_stream(stream), (const float2*)mats_host);
        if (rc) return rc;
    }
    return QS_OK;
}

extern "C" int qs_jit_pass_source(int n, int dtype, const qs_pass* pass, const qs_op* ops, int64_t nops_total,
                                  const void* mats_host, int64_t mats_count, int launch_index, char* out,
                                  size_t out_size, int64_t* src_len) {
    QS_REQUIRE(n >= 1 && n <= 40, "qubit count %d outside [1, 40]", n);
    QS_REQUIRE(valid_dtype(dtype), "bad dtype %d", dtype);
    QS_REQUIRE(pass != nullptr && mats_host != nullptr && src_len != nullptr, "null argument");
    QS_REQUIRE(launch_index >= 0, "negative launch index");
    // pair passes (adjoint) carry EXPECT ops; their partials buffer is not touched here
    int rc = validate_pass(*pass, n, ops, nops_total, mats_count, pass->pair > 0, INT64_MAX / 4);
    if (rc) return rc;
    const int R = jit_reg_bits(dtype == QS_C128 ? reg_bits<double2>() : reg_bits<float2>());
    const int nT = pass->k - R;
    if (!(nT >= 5 && nT <= 8 && pass->nlow >= 5)) {
        set_error("qs_jit_pass_source: tile 2^%d / nlow %d is not a register tile", pass->k, pass->nlow);
        return QS_ENOTSUP;
    }
    static thread_local RegArgs args;
    std::vector<int> rem(pass->op_count);
    for (int i = 0; i < pass->op_count; ++i) rem[i] = i;
    JitPass jp;
    bool ok = false;
    for (int li = 0; li <= launch_index; ++li) {
        if (rem.empty()) {
            set_error("qs_jit_pass_source: the pass has %d launches", li);
            return QS_EINVAL;
        }
        if (build_reg(*pass, ops, rem, n, R, dtype == QS_C128 ? 3 : 4, args) <= 0) {
            set_error("qs_jit_pass_source: an op does not fit a register tile");
            return QS_EINVAL;
        }
        if (li == launch_index)
            ok = dtype == QS_C128 ? gen_reg_pass<double2>(args, R, (const double2*)mats_host, jp)
                                  : gen_reg_pass<float2>(args, R, (const float2*)mats_host, jp);
    }
    if (!ok) {
        set_error("qs_jit_pass_source: this launch is not generated (batched, EXPECT ops or parameters too large)");
        return QS_ENOTSUP;
    }
    *src_len = int64_t(jp.src.size());
    if (out != nullptr && out_size > 0) {
        const size_t k = jp.src.size() < out_size - 1 ? jp.src.size() : out_size - 1;
        memcpy(out, jp.src.data(), k);
        out[k] = 0;
    }
    return QS_OK;
}
