// Register-resident fused passes: device code and host planning shared by
// the per-pass launches (fused.cu) and the persistent batch kernel (batch.cu).
//
// A tile holds 2^k amplitudes: vector bits 0..nlow-1 plus k-nlow chosen higher
// bits.  Each thread owns 2^R of them in registers; a "layout" assigns R tile
// bits to register-slot bits and the rest to the thread index (lanes first).
// Ops whose dense targets are slot bits run as unrolled register code; between
// stages the tile is re-laid-out through shared memory (see fused.cu for the
// whole design).
#pragma once

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

namespace qs {
namespace {


__host__ __device__ constexpr int popc_c(int x) { return x == 0 ? 0 : (x & 1) + popc_c(x >> 1); }
// position of the i-th set bit of mask
__host__ __device__ constexpr int nth_bit(int mask, int i) {
    int b = 0;
    while (true) {
        if ((mask >> b) & 1) {
            if (i == 0) return b;
            --i;
        }
        ++b;
    }
}
// deposit the low bits of k into the set positions of mask
__host__ __device__ constexpr int pdep_c(int k, int mask) {
    int r = 0, i = 0;
    for (int b = 0; b < 32; ++b)
        if ((mask >> b) & 1) {
            if ((k >> i) & 1) r |= 1 << b;
            ++i;
        }
    return r;
}
// gather the bits of s at the set positions of mask
__host__ __device__ constexpr int pext_c(int s, int mask) {
    int r = 0, i = 0;
    for (int b = 0; b < 32; ++b)
        if ((mask >> b) & 1) {
            if ((s >> b) & 1) r |= 1 << i;
            ++i;
        }
    return r;
}

__device__ __forceinline__ uint32_t ins0(uint32_t x, int b) {
    return ((x >> b) << (b + 1)) | (x & ((1u << b) - 1u));
}

// ============================================================ register-resident kernel
constexpr int kMaxStages = 40;

struct KOp {
    uint8_t code;     // QS_OP_MAT / DIAG / ANTI / SWAP
    uint8_t mask;     // slot-bit mask of the targets held in registers
    uint8_t scm;      // control mask on slot bits
    uint8_t nh;       // DIAG: targets outside the registers
    uint8_t hsrc[4];  // DIAG: their sources: < 64 tile bit, >= 64 vector bit + 64
    uint16_t tctrl;   // control mask on the thread's tile bits
    uint16_t moff;    // shared-memory offset of the slot-ordered matrix
    uint8_t flags;
    uint8_t ns;       // DIAG: number of slot targets
    uint16_t elocal;  // EXPECT: index of the op's partial among the pass's EXPECT ops
    uint64_t gctrl;   // control mask on vector bits outside the tile
    uint8_t kidx[32]; // DIAG: slot s -> index of its slot bits in the diagonal
};
struct KCopy {
    int64_t goff;     // table offset of the stored matrix
    int64_t stride;   // per-instance stride (batched passes)
    uint16_t soff;    // shared-memory offset
    uint8_t m;
    uint8_t diag;
    uint8_t perm[4];  // slot-order index bit i -> stored index bit perm[i]
};
struct __align__(16) KStage {
    // Buffer addresses for the relayout into this stage, under a linear (XOR)
    // map chosen on the host so that the writing and the reading layout both
    // spread each shared-memory phase over all banks: images of the previous
    // stage's thread bits / slot bits (writes) and of this stage's (reads).
    uint16_t wthr[8], rthr[8], wslot[8], rslot[8];
    uint16_t tbit[8]; // 1 << T[i]: this stage's thread bits as tile positions
    uint8_t R[6];     // slot bit j <-> tile bit R[j]
    uint8_t T[8];     // thread bit i <-> tile bit T[i]
    uint16_t op_begin, op_count;
    uint16_t img[QS_MAX_TILE_BITS];  // the map itself: buffer address of each tile bit
};
// Scalar part of a planned register pass.
struct RegHead {
    int n, K, L, H, nT, nstages, nops, nmats, inst_shift, batched;
    int nexp;           // EXPECT ops (adjoint pair passes)
    uint64_t pairmask;  // vector bit separating psi / lam (adjoint pair passes), else 0
    int hi[QS_MAX_TILE_BITS];
};
// A planned register pass with room for the largest one (a kernel parameter of
// the per-pass launches); the batch kernel keeps only the used entries.
struct RegArgs : RegHead {
    int eslot[QS_MAX_PASS_OPS];  // output slot of each EXPECT op
    KStage st[kMaxStages];
    KOp ops[QS_MAX_PASS_OPS];
    KCopy cp[QS_MAX_PASS_OPS];
};

__device__ __forceinline__ bool ctrl_ok(int s, uint32_t scm) { return (uint32_t(s) & scm) == scm; }

// compile-time loop: f(std::integral_constant<int, i>) for i in [0, N)
template <typename F, int... I>
__device__ __forceinline__ void sfor_impl(F&& f, std::integer_sequence<int, I...>) {
    (f(std::integral_constant<int, I>{}), ...);
}
template <int N, typename F>
__device__ __forceinline__ void sfor(F&& f) {
    sfor_impl(f, std::make_integer_sequence<int, N>{});
}

// Buffer address of slot s for the current stage: tpos ^ XOR_{j in s} rpos[j].
// (The relayout address maps are linear over GF(2), so a mapped address splits
// the same way.)
template <int R>
struct Addr {
    uint32_t tpos;
    uint32_t rpos[R];
    template <int S>
    __device__ __forceinline__ uint32_t at() const {
        uint32_t t = tpos;
#pragma unroll
        for (int j = 0; j < R; ++j)
            if ((S >> j) & 1) t ^= rpos[j];
        return t;
    }
};

// ---- dense op on the slot bits of MASK (slot-order matrix in shared memory).
// Small matrices keep inputs and outputs in registers; for 8x8 / 16x16 each
// output row goes to this thread's own positions of the tile buffer and is read
// back after the group.  No other thread reads or writes those positions: the
// thread holds exactly the amplitudes stored there (plain order in the first
// stage, the relayout's address map after it; `ad` addresses whichever applies).
// PRED: some of the op's controls are slot bits (checked per group).
template <typename V, int E, int R, int MASK, bool PRED>
__device__ __forceinline__ void r_mat(V (&x)[E], const V* __restrict__ Mm, uint32_t scm, V* __restrict__ buf,
                                      const Addr<R>& ad) {
    constexpr int M = popc_c(MASK);
    constexpr int D = 1 << M;
    constexpr bool PRELOAD = sizeof(V) == 16 ? (M == 1) : (M <= 2);
    constexpr bool BIG = M >= 3;
    V mr[PRELOAD ? D * D : 1];
    if constexpr (PRELOAD) {
#pragma unroll
        for (int i = 0; i < D * D; ++i) mr[i] = Mm[i];
    }
    sfor<E>([&](auto sc) __attribute__((always_inline)) {
        constexpr int s = decltype(sc)::value;
        if constexpr ((s & MASK) == 0) {
            if (!PRED || ctrl_ok(s, scm)) {
                if constexpr (BIG) {
                    sfor<D>([&](auto rc) __attribute__((always_inline)) {
                        constexpr int r = decltype(rc)::value;
                        V acc = cmul(Mm[r * D], x[s]);
                        sfor<D - 1>([&](auto cc) __attribute__((always_inline)) {
                            constexpr int c = decltype(cc)::value + 1;
                            acc = cfma(Mm[r * D + c], x[s | pdep_c(c, MASK)], acc);
                        });
                        buf[ad.template at<(s | pdep_c(r, MASK))>()] = acc;
                    });
                    sfor<D>([&](auto rc) __attribute__((always_inline)) {
                        constexpr int o = s | pdep_c(decltype(rc)::value, MASK);
                        x[o] = buf[ad.template at<o>()];
                    });
                } else {
                    V xi[D];
                    sfor<D>([&](auto kc) __attribute__((always_inline)) {
                        constexpr int k = decltype(kc)::value;
                        xi[k] = x[s | pdep_c(k, MASK)];
                    });
                    sfor<D>([&](auto rc) __attribute__((always_inline)) {
                        constexpr int r = decltype(rc)::value;
                        auto mat = [&](int e) -> V {
                            if constexpr (PRELOAD) return mr[e];
                            else return Mm[e];
                        };
                        V acc = cmul(mat(r * D), xi[0]);
#pragma unroll
                        for (int c = 1; c < D; ++c)
                            acc = cfma(mat(r * D + c), xi[c], acc);
                        x[s | pdep_c(r, MASK)] = acc;
                    });
                }
            }
        }
    });
}

// ---- anti-diagonal 2x2 on one slot bit (UNIT: plain exchange)
template <typename V, int E, int MASK, bool PRED, bool UNIT>
__device__ __forceinline__ void r_anti(V (&x)[E], const V* __restrict__ Mm, uint32_t scm) {
    V m01, m10;
    if constexpr (!UNIT) {
        m01 = Mm[1];
        m10 = Mm[2];
    }
    sfor<E>([&](auto sc) __attribute__((always_inline)) {
        constexpr int s = decltype(sc)::value;
        if constexpr ((s & MASK) == 0) {
            if (!PRED || ctrl_ok(s, scm)) {
                V a = x[s];
                if constexpr (UNIT) {
                    x[s] = x[s | MASK];
                    x[s | MASK] = a;
                } else {
                    x[s] = cmul(m01, x[s | MASK]);
                    x[s | MASK] = cmul(m10, a);
                }
            }
        }
    });
}

// ---- swap-like 4x4 on two slot bits (slot order: index 1 = lower bit)
template <typename V, int E, int MASK, bool PRED, bool UNIT>
__device__ __forceinline__ void r_swap(V (&x)[E], const V* __restrict__ Mm, uint32_t scm) {
    constexpr int B0 = 1 << nth_bit(MASK, 0), B1 = 1 << nth_bit(MASK, 1);
    sfor<E>([&](auto sc) __attribute__((always_inline)) {
        constexpr int s = decltype(sc)::value;
        if constexpr ((s & MASK) == 0) {
            if (!PRED || ctrl_ok(s, scm)) {
                V a = x[s | B0];
                if constexpr (UNIT) {
                    x[s | B0] = x[s | B1];
                    x[s | B1] = a;
                } else {
                    x[s | B0] = cmul(Mm[6], x[s | B1]);
                    x[s | B1] = cmul(Mm[9], a);
                    x[s] = cmul(Mm[0], x[s]);
                    x[s | B0 | B1] = cmul(Mm[15], x[s | B0 | B1]);
                }
            }
        }
    });
}

// ---- diagonal: index = (outside-register bits) << popc(SM) | slot bits of SM
template <typename V, int E, int SM, bool PRED>
__device__ __forceinline__ void r_diag(V (&x)[E], const V* __restrict__ Dm, uint32_t scm, uint32_t h) {
    constexpr int NS = popc_c(SM);
    const V* d = Dm + (h << NS);
    constexpr bool PRELOAD = NS <= 2;
    V dv[PRELOAD ? (1 << NS) : 1];
    if constexpr (PRELOAD) {
#pragma unroll
        for (int i = 0; i < (1 << NS); ++i) dv[i] = d[i];
    }
    sfor<E>([&](auto sc) __attribute__((always_inline)) {
        constexpr int s = decltype(sc)::value;
        constexpr int k = pext_c(s, SM);
        if (!PRED || ctrl_ok(s, scm)) {
            if constexpr (PRELOAD) x[s] = cmul(x[s], dv[k]);
            else x[s] = cmul(x[s], d[k]);
        }
    });
}

// ---- diagonal, one code path for every slot mask: x[s] *= d[(h << ns) | kidx[s]]
template <typename V, int E, bool PRED>
__device__ __forceinline__ void r_diag_any(V (&x)[E], const V* __restrict__ Dm, uint32_t scm, uint32_t h,
                                           const KOp& op) {
    const V* d = Dm + (h << op.ns);
    uint32_t kw[E / 4];
#pragma unroll
    for (int i = 0; i < E / 4; ++i) kw[i] = reinterpret_cast<const uint32_t*>(op.kidx)[i];
#pragma unroll
    for (int s = 0; s < E; ++s) {
        const uint32_t k = (kw[s >> 2] >> (8 * (s & 3))) & 0xffu;
        const V f = d[k];
        const V y = cmul(x[s], f);
        if constexpr (PRED) {
            const bool ok = (uint32_t(s) & scm) == scm;
            x[s].x = ok ? y.x : x[s].x;
            x[s].y = ok ? y.y : x[s].y;
        } else {
            x[s] = y;
        }
    }
}

// ---- EXPECT ops (adjoint pair passes): slot bit 0 holds the psi/lam pair bit,
// so x[s] (bit 0 clear) is a psi amplitude and x[s | 1] its lam partner.
// Adds sum conj(lam) (G psi) over the thread's amplitudes to (re, im): the
// thread's few products are summed in the state's precision (one conversion
// per op instead of one per product) and everything above that in FP64.
template <typename V, int E, int MASK>
__device__ __forceinline__ void r_expect_dense(const V (&x)[E], const V* __restrict__ Gm, double& re, double& im) {
    using S = decltype(V::x);
    constexpr int D = 1 << popc_c(MASK);
    S pr = 0, pi = 0;
    sfor<E>([&](auto sc) __attribute__((always_inline)) {
        constexpr int s = decltype(sc)::value;
        if constexpr ((s & MASK) == 0 && (s & 1) == 0) {
            sfor<D>([&](auto rc) __attribute__((always_inline)) {
                constexpr int r = decltype(rc)::value;
                V acc = cmul(Gm[r * D], x[s]);
                sfor<D - 1>([&](auto cc) __attribute__((always_inline)) {
                    constexpr int c = decltype(cc)::value + 1;
                    acc = cfma(Gm[r * D + c], x[s | pdep_c(c, MASK)], acc);
                });
                const V l = x[s | 1 | pdep_c(r, MASK)];
                pr += l.x * acc.x + l.y * acc.y;
                pi += l.x * acc.y - l.y * acc.x;
            });
        }
    });
    re += double(pr);
    im += double(pi);
}

template <typename V, int E>
__device__ __forceinline__ void r_expect_diag(const V (&x)[E], const V* __restrict__ Dm, uint32_t h, const KOp& op,
                                              double& re, double& im) {
    using S = decltype(V::x);
    const V* d = Dm + (h << op.ns);
    S pr = 0, pi = 0;
#pragma unroll
    for (int s = 0; s < E; s += 2) {
        const V acc = cmul(d[op.kidx[s]], x[s]);
        const V l = x[s | 1];
        pr += l.x * acc.x + l.y * acc.y;
        pi += l.x * acc.y - l.y * acc.x;
    }
    re += double(pr);
    im += double(pi);
}

#define QS_MASKS_1_31(F)                                                                             \
    F(1) F(2) F(3) F(4) F(5) F(6) F(7) F(8) F(9) F(10) F(11) F(12) F(13) F(14) F(15) F(16) F(17) \
        F(18) F(19) F(20) F(21) F(22) F(23) F(24) F(25) F(26) F(27) F(28) F(29) F(30) F(31)

template <typename V, int R, bool EXP, bool BIG>
__device__ __forceinline__ void r_apply(V (&x)[1 << R], const KOp& op, const V* __restrict__ msm, uint32_t thr,
                                        uint64_t base, V* __restrict__ buf, const Addr<R>& ad,
                                        double2* __restrict__ ered) {
    constexpr int E = 1 << R;
    const V* Mm = msm + op.moff;
    const uint32_t scm = op.scm;
    const bool pred = scm != 0;
    const bool unit = op.flags & QS_OPF_UNIT;
    switch (op.code) {
        case QS_OP_MAT:
            switch (op.mask) {
#define QS_CASE(MK)                                                                  \
    case MK:                                                                         \
        if constexpr ((MK) < (1 << R) && popc_c(MK) <= 2) {                          \
            if constexpr (BIG) {                                                     \
                if (pred) r_mat<V, E, R, MK, true>(x, Mm, scm, buf, ad);             \
                else r_mat<V, E, R, MK, false>(x, Mm, scm, buf, ad);                 \
            } else {                                                                 \
                r_mat<V, E, R, MK, false>(x, Mm, scm, buf, ad);                      \
            }                                                                        \
        } else if constexpr (BIG && (MK) < (1 << R) && popc_c(MK) <= 4) {            \
            r_mat<V, E, R, MK, true>(x, Mm, scm, buf, ad);                           \
        }                                                                            \
        break;
                QS_MASKS_1_31(QS_CASE)
#undef QS_CASE
            }
            break;
        case QS_OP_ANTI:  // the host routes only unit exchanges here
            switch (op.mask) {
#define QS_CASE(MK)                                                                  \
    case MK:                                                                         \
        if constexpr ((MK) < (1 << R) && popc_c(MK) == 1) r_anti<V, E, MK, true, true>(x, Mm, scm); \
        break;
                QS_MASKS_1_31(QS_CASE)
#undef QS_CASE
            }
            break;
        case QS_OP_SWAP:  // the host routes only unit exchanges here
            switch (op.mask) {
#define QS_CASE(MK)                                                                  \
    case MK:                                                                         \
        if constexpr ((MK) < (1 << R) && popc_c(MK) == 2) r_swap<V, E, MK, true, true>(x, Mm, scm); \
        break;
                QS_MASKS_1_31(QS_CASE)
#undef QS_CASE
            }
            break;
        case QS_OP_EXPECT:
            if constexpr (EXP) {
                double re = 0.0, im = 0.0;
                if (op.flags & QS_OPF_DIAG) {
                    uint32_t h = 0;
                    for (int q = 0; q < op.nh; ++q) {
                        const int src = op.hsrc[q];
                        const uint32_t bit = src < 64 ? (thr >> src) & 1u : uint32_t((base >> (src - 64)) & 1u);
                        h = (h << 1) | bit;
                    }
                    r_expect_diag<V, E>(x, Mm, h, op, re, im);
                } else {
                    switch (op.mask) {
#define QS_CASE(MK)                                                                           \
    case MK:                                                                                  \
        if constexpr ((MK) < (1 << R) && ((MK) & 1) == 0 && popc_c(MK) <= 2) r_expect_dense<V, E, MK>(x, Mm, re, im); \
        break;
                        QS_MASKS_1_31(QS_CASE)
#undef QS_CASE
                    }
                }
                // warp sum in a fixed order; lane 0 records the warp's partial
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) {
                    re += __shfl_xor_sync(0xffffffffu, re, off);
                    im += __shfl_xor_sync(0xffffffffu, im, off);
                }
                if ((threadIdx.x & 31) == 0) ered[op.elocal] = make_double2(re, im);  // this warp's row
            }
            break;
        default: {  // QS_OP_DIAG
            uint32_t h = 0;
            for (int q = 0; q < op.nh; ++q) {
                const int src = op.hsrc[q];
                const uint32_t bit = src < 64 ? (thr >> src) & 1u : uint32_t((base >> (src - 64)) & 1u);
                h = (h << 1) | bit;
            }
            if (op.ns == 0) {  // no target in registers: one factor per thread
                if (pred) r_diag<V, E, 0, true>(x, Mm, scm, h);
                else r_diag<V, E, 0, false>(x, Mm, scm, h);
            } else {
                if (pred) r_diag_any<V, E, true>(x, Mm, scm, h, op);
                else r_diag_any<V, E, false>(x, Mm, scm, h, op);
            }
        }
    }
    (void)unit;
}

// tile position of this thread's slot 0: XOR of the given images of the set
// thread-index bits (unrolled; images of unused bits are 0)
__device__ __forceinline__ uint32_t thread_pos(const uint16_t* __restrict__ img) {
    const uint4 w = *reinterpret_cast<const uint4*>(img);
    const uint32_t v[4] = {w.x, w.y, w.z, w.w};
    uint32_t t = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const uint32_t im = (v[i >> 1] >> (16 * (i & 1))) & 0xffffu;
        t ^= ((threadIdx.x >> i) & 1u) ? im : 0u;
    }
    return t;
}

template <int R>
__device__ __forceinline__ Addr<R> make_addr(const uint16_t* __restrict__ thr_img, const uint16_t* __restrict__ slot_img) {
    Addr<R> a;
    a.tpos = thread_pos(thr_img);
    const uint4 w = *reinterpret_cast<const uint4*>(slot_img);
    const uint32_t v[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int j = 0; j < R; ++j) a.rpos[j] = (v[j >> 1] >> (16 * (j & 1))) & 0xffffu;
    return a;
}

// Re-layout the registers from the previous stage's layout into stage B's
// through the buffer under B's map; returns B's addressing.
template <typename V, int R>
__device__ __forceinline__ Addr<R> r_relayout(V (&x)[1 << R], V* __restrict__ buf, const KStage& B) {
    constexpr int E = 1 << R;
    const Addr<R> aw = make_addr<R>(B.wthr, B.wslot);
    const Addr<R> ar = make_addr<R>(B.rthr, B.rslot);
    __syncthreads();  // previous readers of buf are done
    sfor<E>([&](auto sc) __attribute__((always_inline)) {
        constexpr int s = decltype(sc)::value;
        buf[aw.template at<s>()] = x[s];
    });
    __syncthreads();
    sfor<E>([&](auto sc) __attribute__((always_inline)) {
        constexpr int s = decltype(sc)::value;
        x[s] = buf[ar.template at<s>()];
    });
    return ar;
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Copy one tile (2^K amplitudes) into `dst` in plain tile order with 16-byte
// cp.async chunks (one chunk = 16 / sizeof(V) consecutive amplitudes).
// `fresh`: write the tile of |0...0> instead (amplitude 1 at global index 0);
// the barrier that follows the cp.async wait also orders these stores.
template <typename V>
__device__ __forceinline__ void tile_prefetch(V* __restrict__ dst, const V* __restrict__ vec, uint64_t base, int K,
                                              int L, const uint64_t* __restrict__ hoff, bool fresh = false) {
    constexpr int EPC = 16 / sizeof(V);
    const uint32_t chunks = (1u << K) / EPC;
    const uint32_t lmask = (1u << L) - 1u;
    if (fresh) {
        for (uint32_t e = threadIdx.x; e < (1u << K); e += blockDim.x)
            dst[e] = (base == 0 && e == 0) ? mk<V>(1.0, 0.0) : mk<V>(0.0, 0.0);
    } else {
        for (uint32_t c = threadIdx.x; c < chunks; c += blockDim.x) {
            const uint32_t e = c * EPC;
            cp_async16(dst + e, vec + (base | hoff[e >> L] | (e & lmask)));
        }
    }
    cp_async_commit();
}

// The tiles [tile, tend) in steps of tstep of one register pass (RegArgs p),
// run by the calling CTA.  EXP: adjoint pair pass (psi and lam halves in one
// vector, EXPECT ops write per-tile partials to `partials`).  BIG: code paths
// for dense ops on 3 or 4 register bits and for dense ops with controls;
// passes without such ops use the variant without them (less code to fetch
// between the ops that do run).  `fresh`: the pass reads |0...0> instead of
// the vector (the first pass of a run from the all-zero state).  The CTA may
// have more threads than the pass's 2^nT: the others repeat the work of
// thread (tid mod 2^nT), writing the same values to the same shared-memory
// words, and store nothing to global memory.  Uses the caller's dynamic shared
// memory (reg_smem_bytes) and ends with a barrier-free tail: a caller that
// reuses the shared memory afterwards synchronises first.
// The pass's stage, op, matrix-copy and EXPECT-slot arrays are read through
// pst / pops / pcp / pes (the RegArgs arrays, or compact copies of their used
// entries).
template <typename V, int R, bool EXP, bool BIG>
__device__ __forceinline__ void reg_tiles(V* __restrict__ vec, const RegHead& p, const KStage* __restrict__ pst,
                                          const KOp* __restrict__ pops, const KCopy* __restrict__ pcp,
                                          const int* __restrict__ pes, const V* __restrict__ mats,
                                          double* __restrict__ partials, uint64_t tile, const uint64_t tend,
                                          const uint64_t tstep, const bool fresh) {
    constexpr int E = 1 << R;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int K = p.K, L = p.L, H = p.H, nT = p.nT;
    const unsigned nact = 1u << nT;             // threads the pass is laid out for
    const bool act = threadIdx.x < nact;        // the others alias thread (tid mod nact)
    V* bufs[2] = {reinterpret_cast<V*>(smem_raw), reinterpret_cast<V*>(smem_raw) + (size_t(1) << K)};
    V* msm = bufs[1] + (size_t(1) << K);
    uint64_t* hoff = reinterpret_cast<uint64_t*>(msm + p.nmats);
    uint64_t* gslot_store = hoff + (size_t(1) << H);  // E entries: global offset of each slot
    // op and stage descriptors live in shared memory: the per-op loop reads
    // them with a data-dependent index, which the constant cache serves poorly
    KOp* sops = reinterpret_cast<KOp*>(gslot_store + E);
    KStage* sst = reinterpret_cast<KStage*>((reinterpret_cast<uintptr_t>(sops + p.nops) + 15) & ~uintptr_t(15));
    for (int o = threadIdx.x; o < p.nops; o += blockDim.x) sops[o] = pops[o];
    for (int o = threadIdx.x; o < p.nstages; o += blockDim.x) sst[o] = pst[o];
    // stage the pass's matrices in slot order (per instance when batched):
    // one entry per thread and step over all ops' entries, so the loads of a
    // restage are independent; `eop` maps an entry to its op
    uint8_t* eop = reinterpret_cast<uint8_t*>(sst + p.nstages);
    // EXPECT partials of the current tile: [warp][EXPECT op]; ered_w is this warp's row
    double2* ered = reinterpret_cast<double2*>((reinterpret_cast<uintptr_t>(eop + p.nmats) + 15) & ~uintptr_t(15));
    double2* ered_w = ered + ((threadIdx.x & (nact - 1u)) >> 5) * p.nexp;
    for (int o = 0; o < p.nops; ++o) {
        const KCopy& c = pcp[o];
        const int cnt = c.diag ? (1 << c.m) : (1 << (2 * c.m));
        for (int e = threadIdx.x; e < cnt; e += blockDim.x) eop[c.soff + e] = uint8_t(o);
    }
    __syncthreads();
    auto stage_mats = [&](uint64_t inst) {
        for (int g = threadIdx.x; g < p.nmats; g += blockDim.x) {
            const KCopy& c = pcp[eop[g]];
            const int e = g - c.soff;
            const int D = 1 << c.m;
            const int kr = c.diag ? e : e / D, kc = c.diag ? 0 : e % D;
            int sr = 0, sc = 0;
            for (int i = 0; i < c.m; ++i) {
                sr |= ((kr >> i) & 1) << c.perm[i];
                sc |= ((kc >> i) & 1) << c.perm[i];
            }
            msm[g] = mats[c.goff + int64_t(inst) * c.stride + (c.diag ? sr : sr * D + sc)];
        }
    };
    uint64_t staged = 0;
    stage_mats(0);
    for (uint32_t j = threadIdx.x; j < (1u << H); j += blockDim.x) {
        uint64_t o = 0;
        for (int t = 0; t < H; ++t)
            if ((j >> t) & 1) o |= uint64_t(1) << p.hi[t];
        hoff[j] = o;
    }
    auto gbit = [&](int b) -> uint64_t { return uint64_t(1) << (b < L ? b : p.hi[b - L]); };
    const KStage& SL = pst[p.nstages - 1];
    for (int s2 = threadIdx.x; s2 < E; s2 += blockDim.x) {
        uint64_t o = 0;
        for (int j = 0; j < R; ++j)
            if ((s2 >> j) & 1) o |= gbit(SL.R[j]);
        gslot_store[s2] = o;
    }
    uint64_t gthr_store = 0;
    for (int i = 0; i < nT; ++i)
        if ((threadIdx.x >> i) & 1) gthr_store |= gbit(SL.T[i]);
    __syncthreads();
    const uint64_t ntiles = uint64_t(1) << (p.n - K);
    auto tile_base = [&](uint64_t tile) {
        uint64_t b = tile << L;
        for (int t = 0; t < H; ++t) b = insert0(b, p.hi[t]);
        return b;
    };
    if (tile < tend) tile_prefetch<V>(bufs[0], vec, tile_base(tile), K, L, hoff, fresh);
    for (int it = 0; tile < tend; ++it, tile += tstep) {
        V* cur = bufs[it & 1];
        const uint64_t base = tile_base(tile);
        cp_async_wait_all();
        __syncthreads();  // tile landed; the other buffer is free; previous tile's ops are done
        if (tile + tstep < tend) tile_prefetch<V>(bufs[(it + 1) & 1], vec, tile_base(tile + tstep), K, L, hoff, fresh);
        if (p.batched) {
            const uint64_t inst = (base & ~p.pairmask) >> p.inst_shift;
            if (inst != staged) {
                stage_mats(inst);
                staged = inst;
                __syncthreads();
            }
        }
        V x[E];
        // shared memory -> registers in the first stage's (plain) layout
        Addr<R> ad = make_addr<R>(sst[0].rthr, sst[0].rslot);  // stage 0: identity map
        sfor<E>([&](auto sc) __attribute__((always_inline)) {
            constexpr int s = decltype(sc)::value;
            x[s] = cur[ad.template at<s>()];
        });
        for (int si = 0; si < p.nstages; ++si) {
            const KStage& S = sst[si];
            if (si > 0) ad = r_relayout<V, R>(x, cur, S);
            const uint32_t thr = thread_pos(S.tbit);
            const int oe = S.op_begin + S.op_count;
            for (int o = S.op_begin; o < oe; ++o) {
                const KOp& op = sops[o];
                if ((base & op.gctrl) != op.gctrl) continue;
                if ((thr & op.tctrl) != op.tctrl) continue;
                r_apply<V, R, EXP, BIG>(x, op, msm, thr, base, cur, ad, ered_w);
            }
        }
        {  // registers -> global in the last stage's layout (lanes on tile bits 0..4)
            const uint64_t b0 = base | gthr_store;
            if (act)
                sfor<E>([&](auto sc) __attribute__((always_inline)) {
                    constexpr int s = decltype(sc)::value;
                    vec[b0 | gslot_store[s]] = x[s];
                });
        }
        if constexpr (EXP) {  // per-tile partials: warp partials summed in a fixed order
            __syncthreads();
            const int nw = int(nact >> 5);
            for (int e = threadIdx.x; e < p.nexp; e += blockDim.x) {
                double2 t = make_double2(0.0, 0.0);
                for (int w = 0; w < nw; ++w) {
                    t.x += ered[w * p.nexp + e].x;
                    t.y += ered[w * p.nexp + e].y;
                }
                const uint64_t at = 2 * (uint64_t(pes[e]) * ntiles + tile);
                partials[at] = t.x;
                partials[at + 1] = t.y;
            }
        }
    }
}

// ------------------------------------------------------------------ host side
// Dynamic shared memory reg_tiles needs for a planned pass.
template <typename V>
size_t reg_smem_bytes(const RegHead& a, int R, bool exp) {
    const size_t nact = size_t(1) << a.nT;
    return sizeof(V) * (2 * (size_t(1) << a.K) + size_t(a.nmats)) + 8 * ((size_t(1) << a.H) + (size_t(1) << R)) +
           sizeof(KOp) * size_t(a.nops) + 16 + sizeof(KStage) * size_t(a.nstages) + size_t(a.nmats) +
           (exp ? 16 + sizeof(double2) * size_t(a.nexp) * (nact / 32) : 0);
}

int validate_pass(const qs_pass& ps, int n, const qs_op* ops, int64_t nops_total, int64_t mats_count,
                  bool adjoint = false, int64_t partials_count = 0) {
    QS_REQUIRE(ps.k >= 1 && ps.k <= QS_MAX_TILE_BITS && ps.k <= n, "tile bits %d outside [1, min(%d, n)]", ps.k,
               QS_MAX_TILE_BITS);
    QS_REQUIRE(ps.nlow >= 0 && ps.nlow <= ps.k, "nlow %d outside [0, k]", ps.nlow);
    QS_REQUIRE(ps.op_count >= 0 && ps.op_count <= QS_MAX_PASS_OPS, "pass has %d ops (max %d)", ps.op_count,
               QS_MAX_PASS_OPS);
    QS_REQUIRE(ps.op_begin >= 0 && int64_t(ps.op_begin) + ps.op_count <= nops_total, "op range outside op array");
    uint64_t tilemask = (uint64_t(1) << ps.nlow) - 1;
    int prev = ps.nlow - 1;
    for (int t = 0; t < ps.k - ps.nlow; ++t) {
        QS_REQUIRE(ps.hi[t] > prev && ps.hi[t] < n, "tile bits must ascend, be >= nlow and < n");
        prev = ps.hi[t];
        tilemask |= uint64_t(1) << ps.hi[t];
    }
    QS_REQUIRE(ps.inst_shift >= 0 && ps.inst_shift <= n, "inst_shift %d outside [0, n]", ps.inst_shift);
    QS_REQUIRE(ps.pair >= 0 && ps.pair <= n, "pair %d outside [0, n]", ps.pair);
    QS_REQUIRE(ps.pair == 0 || adjoint, "pair bits belong to adjoint pair passes");
    const uint64_t pairmask = ps.pair > 0 ? uint64_t(1) << (ps.pair - 1) : 0;
    QS_REQUIRE(ps.pair == 0 || ps.inst_shift == 0 || ps.pair == n, "with instances, the pair bit must be the top bit");
    if (ps.inst_shift > 0)
        QS_REQUIRE(((tilemask & ~pairmask) >> ps.inst_shift) == 0,
                   "tile bits must lie below inst_shift (one instance per tile)");
    const int64_t ninst = ps.inst_shift > 0 ? (int64_t(1) << (n - ps.inst_shift - (ps.pair > 0 ? 1 : 0))) : 1;
    const int64_t ntiles = int64_t(1) << (n - ps.k);
    int local[64];
    for (int b = 0; b < 64; ++b) local[b] = -1;
    for (int b = 0; b < ps.nlow; ++b) local[b] = b;
    for (int t = 0; t < ps.k - ps.nlow; ++t) local[ps.hi[t]] = ps.nlow + t;
    for (int i = 0; i < ps.op_count; ++i) {
        const qs_op& op = ops[ps.op_begin + i];
        QS_REQUIRE((op.kind >= QS_OP_MAT && op.kind <= QS_OP_SWAP) || (adjoint && op.kind == QS_OP_EXPECT),
                   "op %d: bad kind %d", i, op.kind);
        QS_REQUIRE(op.mat_stride >= 0 && (ps.inst_shift > 0 || op.mat_stride == 0),
                   "op %d: a per-instance matrix stride needs inst_shift > 0", i);
        if (op.kind == QS_OP_EXPECT) {
            QS_REQUIRE(op.m <= 2 || (op.flags & QS_OPF_DIAG), "op %d: dense EXPECT generators act on <= 2 bits", i);
            QS_REQUIRE(op.slot >= 0 && (int64_t(op.slot) + 1) * ntiles * 2 <= partials_count,
                       "op %d: EXPECT slot %d outside the partials buffer", i, op.slot);
            QS_REQUIRE(ps.pair == 0 || (tilemask & pairmask), "op %d: EXPECT needs the pair bit in the tile", i);
        }
        QS_REQUIRE(op.m >= 1 && op.m <= 4, "op %d: m=%d outside [1, 4]", i, op.m);
        QS_REQUIRE(op.kind != QS_OP_ANTI || op.m == 1, "op %d: ANTI needs m = 1", i);
        QS_REQUIRE(op.kind != QS_OP_SWAP || op.m == 2, "op %d: SWAP needs m = 2", i);
        QS_REQUIRE((op.gctrl >> n) == 0 && (op.gctrl & tilemask) == 0, "op %d: global controls must lie outside the tile", i);
        QS_REQUIRE((op.lctrl >> ps.k) == 0, "op %d: local controls outside the tile", i);
        uint32_t tl = 0;
        for (int j = 0; j < op.m; ++j) {
            QS_REQUIRE(op.gbit[j] >= 0 && op.gbit[j] < n, "op %d: target bit outside [0, n)", i);
            QS_REQUIRE(op.tgt[j] == local[op.gbit[j]], "op %d: tile position of target %d inconsistent", i, j);
            const bool diag = op.kind == QS_OP_DIAG || (op.kind == QS_OP_EXPECT && (op.flags & QS_OPF_DIAG));
            if (!diag) QS_REQUIRE(op.tgt[j] >= 0, "op %d: dense target outside the tile", i);
            if (op.tgt[j] >= 0) {
                QS_REQUIRE(!((tl >> op.tgt[j]) & 1), "op %d: duplicate target", i);
                tl |= 1u << op.tgt[j];
            }
        }
        QS_REQUIRE((tl & op.lctrl) == 0, "op %d: control overlaps a target", i);
        const bool dg = op.kind == QS_OP_DIAG || (op.kind == QS_OP_EXPECT && (op.flags & QS_OPF_DIAG));
        int64_t len = dg ? (int64_t(1) << op.m) : (int64_t(1) << (2 * op.m));
        QS_REQUIRE(op.mat >= 0 && op.mat + (ninst - 1) * op.mat_stride + len <= mats_count,
                   "op %d: matrix outside the table", i);
    }
    return QS_OK;
}

// Largest dynamic shared memory a block may opt into on the current device.
int smem_optin() {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return v > 0 ? v : 200 * 1024;
}

// Opt a kernel into large dynamic shared memory once per (kernel, device).
void config_smem(const void* fn) {
    static thread_local std::vector<std::pair<const void*, int>> done;
    int dev = 0;
    cudaGetDevice(&dev);
    for (const auto& d : done)
        if (d.first == fn && d.second == dev) return;
    // the opt-in limit covers static and dynamic shared memory together
    cudaFuncAttributes fa{};
    cudaFuncGetAttributes(&fa, fn);
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin() - int(fa.sharedSizeBytes));
    done.emplace_back(fn, dev);
}

// Buffer map of a relayout from layout A to layout B.  Shared memory serves
// a warp's access in phases of 2^nb lanes (thread bits 0..nb-1; 8 lanes for
// 16-byte elements, 16 for 8-byte ones); a phase is conflict-free when its
// lanes' elements fall in distinct 2^nb-element bank groups, i.e. when the map
// sends the phase's tile bits to independent vectors of the low nb address
// bits.  The map keeps every address bit and XORs a host-chosen column H[b]
// into the bank bits for each tile bit b >= nb (invertible: unitriangular);
// H is searched so that both A's and B's phase bits are independent.
void relayout_map(const KStage& A, KStage& B, int K, int nb) {
    int H[QS_MAX_TILE_BITS] = {0};
    int vars[16], nv = 0;
    auto add_var = [&](int b) {
        if (b < nb) return;
        for (int i = 0; i < nv; ++i)
            if (vars[i] == b) return;
        vars[nv++] = b;
    };
    for (int i = 0; i < nb; ++i) add_var(A.T[i]);
    for (int i = 0; i < nb; ++i) add_var(B.T[i]);
    auto col = [&](int b) { return b < nb ? (1 << b) : H[b]; };
    // are the already-known phase columns of layout S linearly independent?
    auto indep = [&](const KStage& S, int assigned) {
        int basis[8] = {0};  // basis[k]: stored vector whose leading bit is k
        for (int i = 0; i < nb; ++i) {
            const int b = S.T[i];
            bool known = b < nb;
            for (int v = 0; v < assigned && !known; ++v) known = vars[v] == b;
            if (!known) continue;
            int c = col(b);
            for (int k = nb - 1; k >= 0 && c; --k) {
                if (!((c >> k) & 1)) continue;
                if (!basis[k]) {
                    basis[k] = c;
                    break;
                }
                c ^= basis[k];
            }
            if (c == 0) return false;
        }
        return true;
    };
    long budget = 200000;
    bool ok = false;
    // depth-first search over the columns of the phase bits
    auto dfs = [&](auto&& self, int v) -> bool {
        if (--budget < 0) return false;
        if (v == nv) return true;
        for (int c = 1; c < (1 << nb); ++c) {
            H[vars[v]] = c;
            if (indep(A, v + 1) && indep(B, v + 1) && self(self, v + 1)) return true;
        }
        H[vars[v]] = 0;
        return false;
    };
    ok = dfs(dfs, 0);
    if (!ok)
        for (int b = 0; b < QS_MAX_TILE_BITS; ++b) H[b] = 0;
    for (int b = 0; b < QS_MAX_TILE_BITS; ++b) B.img[b] = uint16_t(b < K ? ((1 << b) ^ (b >= nb ? H[b] : 0)) : 0);
}

// Build the register-kernel arguments for the ops of a pass listed in `rem`
// (positions within the pass); returns how many were scheduled and removes
// them from `rem` (a pass whose stages or matrices overflow the argument block
// is split into several launches over the same tiles).
//
// Stage schedule: the ops form a dependency graph (two ops stay ordered when
// one acts non-diagonally on a tile bit the other touches; all other pairs
// commute).  A stage holds R tile bits in registers and runs every op whose
// dense targets it holds once the op's predecessors have run.  Stages are
// chosen greedily: every R-bit set is scored by the number of ops it would
// run; ties prefer sets off the lane bits (no extra store relayout).
int build_reg(const qs_pass& ps, const qs_op* ops, std::vector<int>& rem, int n, int R, int nb, RegArgs& a) {
    const int K = ps.k, L = ps.nlow, nT = K - R;
    a.n = n; a.K = K; a.L = L; a.H = K - L; a.nT = nT;
    a.inst_shift = ps.inst_shift;
    a.batched = 0;
    a.nexp = 0;
    a.pairmask = ps.pair > 0 ? uint64_t(1) << (ps.pair - 1) : 0;
    for (int t = 0; t < QS_MAX_TILE_BITS; ++t) a.hi[t] = t < K - L ? ps.hi[t] : 0;
    // tile position of the psi/lam pair bit (adjoint pair passes): EXPECT ops
    // need it in registers, where it always takes slot bit 0
    int pair_tile = -1;
    if (ps.pair > 0) {
        if (ps.pair - 1 < L) pair_tile = ps.pair - 1;
        for (int t = 0; t < K - L; ++t)
            if (ps.hi[t] == ps.pair - 1) pair_tile = L + t;
    }
    const int lowlanes = 5;  // tile bits 0..4 are the lanes of the load/store layout
    const uint32_t lanemask = (1u << lowlanes) - 1u;
    // slot j <-> tile bit order[j] (the pair bit, when present, is slot 0)
    auto make_stage = [&](uint32_t bits, KStage& S, const uint8_t* order) {
        int j = 0, i = 0;
        for (; j < R; ++j) S.R[j] = order[j];
        for (int b = 0; b < K; ++b)
            if (!((bits >> b) & 1)) S.T[i++] = uint8_t(b);
        for (; j < 6; ++j) S.R[j] = 0;
        for (; i < 8; ++i) S.T[i] = 0;
    };
    auto plain_order = [&](uint32_t bits, uint8_t* order) {
        int j = 0;
        if (pair_tile >= 0 && ((bits >> pair_tile) & 1)) order[j++] = uint8_t(pair_tile);
        for (int b = 0; b < K; ++b)
            if (((bits >> b) & 1) && b != pair_tile) order[j++] = uint8_t(b);
    };
    // ---- dependency graph
    const int m = int(rem.size());
    using Set = std::array<uint64_t, (QS_MAX_PASS_OPS + 63) / 64>;
    std::vector<uint32_t> xm(m), am(m), need(m);  // dense bits, all bits, bits needed in registers
    std::vector<int> msz(m);
    std::vector<Set> pred(m);
    for (int i = 0; i < m; ++i) {
        const qs_op& op = ops[ps.op_begin + rem[i]];
        const bool dg = op.kind == QS_OP_DIAG || (op.kind == QS_OP_EXPECT && (op.flags & QS_OPF_DIAG));
        uint32_t x = 0, all = op.lctrl;
        for (int j = 0; j < op.m; ++j)
            if (op.tgt[j] >= 0) {
                all |= 1u << op.tgt[j];
                if (!dg) x |= 1u << op.tgt[j];
            }
        xm[i] = x;
        am[i] = all;
        // EXPECT ops read psi/lam pairs: the pair bit must be in registers (no
        // other op touches it, so it adds no ordering)
        need[i] = x | (op.kind == QS_OP_EXPECT && pair_tile >= 0 ? 1u << pair_tile : 0u);
        msz[i] = dg ? (1 << op.m) : (1 << (2 * op.m));
        pred[i].fill(0);
        for (int h = 0; h < i; ++h)
            if ((xm[h] & am[i]) | (am[h] & xm[i])) pred[i][h >> 6] |= uint64_t(1) << (h & 63);
    }
    auto has = [](const Set& d, int i) { return (d[i >> 6] >> (i & 63)) & 1; };
    auto ready = [&](const Set& d, int i) {
        for (size_t w = 0; w < d.size(); ++w)
            if (pred[i][w] & ~d[w]) return false;
        return true;
    };
    // ops a stage holding `bits` runs from state d (one forward sweep: every
    // predecessor has a smaller position)
    auto score = [&](uint32_t bits, Set d) {
        int c = 0;
        for (int i = 0; i < m; ++i)
            if (!has(d, i) && !(need[i] & ~bits) && ready(d, i)) {
                d[i >> 6] |= uint64_t(1) << (i & 63);
                ++c;
            }
        return c;
    };
    Set done;
    done.fill(0);
    int ndone = 0, mats = 0;
    bool full = false;
    std::vector<uint32_t> stage_bits;
    std::vector<std::vector<int>> stage_ops;
    while (ndone < m && !full && int(stage_bits.size()) < kMaxStages - 1) {
        const bool first_stage = stage_bits.empty();
        uint32_t best = 0;
        int best_score = -1;
        for (uint32_t bits = (1u << R) - 1u; bits < (1u << K);) {
            if (!(first_stage && (bits & lanemask))) {
                const int sc = 2 * score(bits, done) + ((bits & lanemask) == 0);
                if (sc > best_score && (sc >= 2 || first_stage)) {
                    best_score = sc;
                    best = bits;
                }
            }
            const uint32_t c = bits & (0u - bits), r = bits + c;  // next set of R bits
            bits = (((r ^ bits) >> 2) / c) | r;
        }
        if (best_score < 0) break;
        std::vector<int> order;
        for (int i = 0; i < m; ++i)
            if (!has(done, i) && !(need[i] & ~best) && ready(done, i)) {
                if (mats + msz[i] > QS_MAX_PASS_MATS) {
                    full = true;
                    continue;
                }
                mats += msz[i];
                done[i >> 6] |= uint64_t(1) << (i & 63);
                order.push_back(i);
                ++ndone;
            }
        if (order.empty() && !first_stage) break;
        stage_bits.push_back(best);
        stage_ops.push_back(order);
    }
    // ---- slot order per stage.  Register ops dispatch on (kind, slot mask),
    // one code path each; ordering each stage's slots so that its ops reuse
    // the paths earlier stages of this launch already run keeps the set of
    // code paths in use (the instruction working set) small.
    std::vector<std::array<uint8_t, 6>> orders(stage_bits.size());
    std::vector<int> used_keys;
    for (size_t st = 0; st < stage_bits.size(); ++st) {
        uint8_t base_order[6] = {0};
        plain_order(stage_bits[st], base_order);
        // the ops' register targets (tile bits) and dispatch codes
        std::vector<std::pair<int, uint32_t>> dense;
        for (int pos : stage_ops[st]) {
            const qs_op& op = ops[ps.op_begin + rem[pos]];
            const bool dg = op.kind == QS_OP_DIAG || (op.kind == QS_OP_EXPECT && (op.flags & QS_OPF_DIAG));
            if (dg) continue;
            int code = op.kind;
            if ((op.kind == QS_OP_ANTI || op.kind == QS_OP_SWAP) && !(op.flags & QS_OPF_UNIT)) code = QS_OP_MAT;
            uint32_t tb = 0;
            for (int j = 0; j < op.m; ++j) tb |= 1u << op.tgt[j];
            dense.emplace_back(code, tb);
        }
        const int fixed0 = (pair_tile >= 0 && ((stage_bits[st] >> pair_tile) & 1)) ? 1 : 0;
        uint8_t perm[6], best[6];
        for (int j = 0; j < R; ++j) perm[j] = best[j] = base_order[j];
        int best_new = 1 << 30, best_sum = 1 << 30;
        std::sort(perm + fixed0, perm + R);
        do {
            int nnew = 0, sum = 0;
            std::vector<int> keys;
            for (const auto& d : dense) {
                uint32_t mask = 0;
                for (int j = 0; j < R; ++j)
                    if ((d.second >> perm[j]) & 1) mask |= 1u << j;
                const int key = d.first * 64 + int(mask);
                sum += int(mask);
                if (std::find(used_keys.begin(), used_keys.end(), key) == used_keys.end() &&
                    std::find(keys.begin(), keys.end(), key) == keys.end()) {
                    ++nnew;
                    keys.push_back(key);
                }
            }
            if (nnew < best_new || (nnew == best_new && sum < best_sum)) {
                best_new = nnew;
                best_sum = sum;
                for (int j = 0; j < R; ++j) best[j] = perm[j];
            }
        } while (!dense.empty() && std::next_permutation(perm + fixed0, perm + R));
        for (const auto& d : dense) {
            uint32_t mask = 0;
            for (int j = 0; j < R; ++j)
                if ((d.second >> best[j]) & 1) mask |= 1u << j;
            const int key = d.first * 64 + int(mask);
            if (std::find(used_keys.begin(), used_keys.end(), key) == used_keys.end()) used_keys.push_back(key);
        }
        for (int j = 0; j < 6; ++j) orders[st][j] = j < R ? best[j] : 0;
    }
    // ---- emit stages and translate each op into its stage's layout
    int ns = 0, nops = 0, moff = 0;
    for (size_t st = 0; st < stage_bits.size(); ++st) {
        make_stage(stage_bits[st], a.st[ns], orders[st].data());
        a.st[ns].op_begin = uint16_t(nops);
        a.st[ns].op_count = 0;
        ++ns;
        for (int pos : stage_ops[st]) {
            const qs_op& op = ops[ps.op_begin + rem[pos]];
            const int msize = msz[pos];
            // translate the op into the current layout
            KStage& S = a.st[ns - 1];
            auto slot_of = [&](int b) {
                for (int j = 0; j < R; ++j)
                    if (S.R[j] == b) return j;
                return -1;
            };
            KOp& k = a.ops[nops];
            KCopy& c = a.cp[nops];
            k = KOp{};
            c = KCopy{};
            k.code = uint8_t(op.kind);
            k.flags = uint8_t(op.flags);
            // only plain exchanges keep their own code paths; scaled anti-diagonal /
            // swap matrices run as dense matrices (their stored 2x2 / 4x4 is complete)
            if ((op.kind == QS_OP_ANTI || op.kind == QS_OP_SWAP) && !(op.flags & QS_OPF_UNIT)) k.code = QS_OP_MAT;
            k.gctrl = op.gctrl;
            uint32_t scm = 0, tct = 0;
            for (int b = 0; b < K; ++b)
                if ((op.lctrl >> b) & 1) {
                    int sl = slot_of(b);
                    if (sl >= 0) scm |= 1u << sl;
                    else tct |= 1u << b;
                }
            k.scm = uint8_t(scm);
            k.tctrl = uint16_t(tct);
            c.goff = op.mat;
            c.stride = op.mat_stride;
            if (op.mat_stride != 0) a.batched = 1;
            c.soff = uint16_t(moff);
            c.m = uint8_t(op.m);
            c.diag = op.kind == QS_OP_DIAG || (op.kind == QS_OP_EXPECT && (op.flags & QS_OPF_DIAG));
            if (op.kind == QS_OP_EXPECT) {
                k.elocal = uint16_t(a.nexp);
                a.eslot[a.nexp++] = op.slot;
            }
            k.moff = uint16_t(moff);
            // slot-ordered bit permutation
            int slots[4], js[4], ns_ = 0;
            int hj[4], nh = 0;
            for (int j = 0; j < op.m; ++j) {
                int sl = op.tgt[j] >= 0 ? slot_of(op.tgt[j]) : -1;
                if (sl >= 0) {
                    slots[ns_] = sl;
                    js[ns_++] = j;
                } else {
                    hj[nh++] = j;
                }
            }
            for (int x = 0; x < ns_; ++x)  // sort by slot position
                for (int y = 0; y + 1 < ns_ - x; ++y)
                    if (slots[y] > slots[y + 1]) {
                        std::swap(slots[y], slots[y + 1]);
                        std::swap(js[y], js[y + 1]);
                    }
            uint32_t mask = 0;
            for (int x = 0; x < ns_; ++x) {
                mask |= 1u << slots[x];
                c.perm[x] = uint8_t(op.m - 1 - js[x]);
            }
            for (int q = 0; q < nh; ++q) {
                c.perm[ns_ + (nh - 1 - q)] = uint8_t(op.m - 1 - hj[q]);
                const int j = hj[q];
                k.hsrc[q] = op.tgt[j] >= 0 ? uint8_t(op.tgt[j]) : uint8_t(64 + op.gbit[j]);
            }
            k.mask = uint8_t(mask);
            k.nh = uint8_t(nh);
            k.ns = uint8_t(ns_);
            for (int sidx = 0; sidx < (1 << R) && sidx < 32; ++sidx) {
                int kv = 0;
                for (int x2 = 0; x2 < ns_; ++x2)
                    if ((sidx >> slots[x2]) & 1) kv |= 1 << x2;
                k.kidx[sidx] = uint8_t(kv);
            }
            moff += msize;
            ++nops;
            ++S.op_count;
        }
    }
    // final store layout must keep the lanes on tile bits 0..4
    const uint32_t last = stage_bits.empty() ? 0u : stage_bits.back();
    if (last & lanemask) {
        uint32_t bits = 0;
        for (int b = K - 1, c = 0; b >= lowlanes && c < R; --b, ++c) bits |= 1u << b;
        uint8_t order[6] = {0};
        plain_order(bits, order);
        make_stage(bits, a.st[ns], order);
        a.st[ns].op_begin = uint16_t(nops);
        a.st[ns].op_count = 0;
        ++ns;
    }
    for (int b = 0; b < QS_MAX_TILE_BITS; ++b) a.st[0].img[b] = uint16_t(b < K ? 1 << b : 0);
    for (int si = 1; si < ns; ++si) relayout_map(a.st[si - 1], a.st[si], K, nb);
    for (int si = 0; si < ns; ++si) {
        KStage& S = a.st[si];
        const KStage& P = a.st[si > 0 ? si - 1 : 0];
        for (int i = 0; i < 8; ++i) {
            S.wthr[i] = i < nT ? S.img[P.T[i]] : 0;
            S.rthr[i] = i < nT ? S.img[S.T[i]] : 0;
            S.tbit[i] = i < nT ? uint16_t(1u << S.T[i]) : 0;
            S.wslot[i] = i < R ? S.img[P.R[i]] : 0;
            S.rslot[i] = i < R ? S.img[S.R[i]] : 0;
        }
    }
    a.nstages = ns;
    a.nops = nops;
    a.nmats = moff;
    std::vector<int> left;
    for (int i = 0; i < m; ++i)
        if (!has(done, i)) left.push_back(rem[i]);
    rem.swap(left);
    return ndone;
}

}  // namespace

// Generated source of a planned register pass (`regargs`: a RegArgs filled by
// build_reg; the struct has the same layout in every file that includes this
// header) as the `extern "C" __device__` function `name` called by the
// linked persistent batch kernel; its parameter block, dynamic shared memory
// and thread count.  mats_host: the host matrix table in the state's
// precision.  False when the pass is not generated (fused.cu).
bool gen_batch_pass(const void* regargs, int R, bool c128, const void* mats_host, const char* name, std::string* src,
                    std::vector<uint64_t>* params, size_t* smem, int* threads);

}  // namespace qs
