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

namespace qs {
namespace {

constexpr int kFT = 256;

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
struct RegArgs {
    int n, K, L, H, nT, nstages, nops, nmats, inst_shift, batched;
    int nexp;           // EXPECT ops (adjoint pair passes)
    uint64_t pairmask;  // vector bit separating psi / lam (adjoint pair passes), else 0
    int hi[QS_MAX_TILE_BITS];
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
template <typename V>
__device__ __forceinline__ void tile_prefetch(V* __restrict__ dst, const V* __restrict__ vec, uint64_t base, int K,
                                              int L, const uint64_t* __restrict__ hoff) {
    constexpr int EPC = 16 / sizeof(V);
    const uint32_t chunks = (1u << K) / EPC;
    const uint32_t lmask = (1u << L) - 1u;
    for (uint32_t c = threadIdx.x; c < chunks; c += blockDim.x) {
        const uint32_t e = c * EPC;
        cp_async16(dst + e, vec + (base | hoff[e >> L] | (e & lmask)));
    }
    cp_async_commit();
}

// EXP: adjoint pair pass (psi and lam halves in one vector, EXPECT ops write
// per-tile partials to `partials`).  BIG: code paths for dense ops on 3 or 4
// register bits and for dense ops with controls; passes without such ops use
// the variant without them (less code to fetch between the ops that do run).
template <typename V, int R, bool EXP, bool BIG>
__global__ void __launch_bounds__(256, 1) k_fused_reg(V* __restrict__ vec, const __grid_constant__ RegArgs p,
                                                      const V* __restrict__ mats, double* __restrict__ partials) {
    constexpr int E = 1 << R;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int K = p.K, L = p.L, H = p.H, nT = p.nT;
    V* bufs[2] = {reinterpret_cast<V*>(smem_raw), reinterpret_cast<V*>(smem_raw) + (size_t(1) << K)};
    V* msm = bufs[1] + (size_t(1) << K);
    uint64_t* hoff = reinterpret_cast<uint64_t*>(msm + p.nmats);
    uint64_t* gslot_store = hoff + (size_t(1) << H);  // E entries: global offset of each slot
    // op and stage descriptors live in shared memory: the per-op loop reads
    // them with a data-dependent index, which the constant cache serves poorly
    KOp* sops = reinterpret_cast<KOp*>(gslot_store + E);
    KStage* sst = reinterpret_cast<KStage*>((reinterpret_cast<uintptr_t>(sops + p.nops) + 15) & ~uintptr_t(15));
    for (int o = threadIdx.x; o < p.nops; o += blockDim.x) sops[o] = p.ops[o];
    for (int o = threadIdx.x; o < p.nstages; o += blockDim.x) sst[o] = p.st[o];
    // stage the pass's matrices in slot order (per instance when batched):
    // one entry per thread and step over all ops' entries, so the loads of a
    // restage are independent; `eop` maps an entry to its op
    uint8_t* eop = reinterpret_cast<uint8_t*>(sst + p.nstages);
    // EXPECT partials of the current tile: [warp][EXPECT op]; ered_w is this warp's row
    double2* ered = reinterpret_cast<double2*>((reinterpret_cast<uintptr_t>(eop + p.nmats) + 15) & ~uintptr_t(15));
    double2* ered_w = ered + (threadIdx.x >> 5) * p.nexp;
    for (int o = 0; o < p.nops; ++o) {
        const KCopy& c = p.cp[o];
        const int cnt = c.diag ? (1 << c.m) : (1 << (2 * c.m));
        for (int e = threadIdx.x; e < cnt; e += blockDim.x) eop[c.soff + e] = uint8_t(o);
    }
    __syncthreads();
    auto stage_mats = [&](uint64_t inst) {
        for (int g = threadIdx.x; g < p.nmats; g += blockDim.x) {
            const KCopy& c = p.cp[eop[g]];
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
    const KStage& SL = p.st[p.nstages - 1];
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
    // tile order: strided over the grid; batched passes take contiguous runs
    // of tiles instead, so that a CTA restages per-instance matrices once per
    // instance rather than once per tile
    uint64_t tile, tend, tstep;
    if (p.batched) {
        const uint64_t chunk = (ntiles + gridDim.x - 1) / gridDim.x;
        tile = uint64_t(blockIdx.x) * chunk;
        tend = tile + chunk < ntiles ? tile + chunk : ntiles;
        tstep = 1;
    } else {
        tile = blockIdx.x;
        tend = ntiles;
        tstep = gridDim.x;
    }
    if (tile < tend) tile_prefetch<V>(bufs[0], vec, tile_base(tile), K, L, hoff);
    for (int it = 0; tile < tend; ++it, tile += tstep) {
        V* cur = bufs[it & 1];
        const uint64_t base = tile_base(tile);
        cp_async_wait_all();
        __syncthreads();  // tile landed; the other buffer is free; previous tile's ops are done
        if (tile + tstep < tend) tile_prefetch<V>(bufs[(it + 1) & 1], vec, tile_base(tile + tstep), K, L, hoff);
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
            sfor<E>([&](auto sc) __attribute__((always_inline)) {
                constexpr int s = decltype(sc)::value;
                vec[b0 | gslot_store[s]] = x[s];
            });
        }
        if constexpr (EXP) {  // per-tile partials: warp partials summed in a fixed order
            __syncthreads();
            const int nw = blockDim.x >> 5;
            for (int e = threadIdx.x; e < p.nexp; e += blockDim.x) {
                double2 t = make_double2(0.0, 0.0);
                for (int w = 0; w < nw; ++w) {
                    t.x += ered[w * p.nexp + e].x;
                    t.y += ered[w * p.nexp + e].y;
                }
                const uint64_t at = 2 * (uint64_t(p.eslot[e]) * ntiles + tile);
                partials[at] = t.x;
                partials[at + 1] = t.y;
            }
        }
    }
}

// ------------------------------------------------------------------ host side
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

template <typename V>
bool gen_reg_pass(const RegArgs& a, int R, const V* hm, JitPass& out, bool with_source = true) {
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
    out.threads = threads;
    out.smem = sizeof(V) * 2 * (size_t(1) << K) + 8 * size_t(hoff_n) +
               (a.nexp > 0 ? sizeof(double2) * size_t(nwarps) * size_t(a.nexp) : 0) +
               (batched ? sizeof(V) * size_t(NM) : 0) + sizeof(V) * size_t(ndsm);
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
    const int target = env_target > 0 ? env_target : 512;
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
    g.add("extern \"C\" __global__ void __launch_bounds__(%d, %d) qs_pass(V* __restrict__ vec, "
          "const __grid_constant__ P p, const V* __restrict__ mats, double* __restrict__ partials) {\n", threads, minb);
    g.add("  extern __shared__ __align__(16) unsigned char smem_raw[];\n");
    g.add("  V* const b0 = reinterpret_cast<V*>(smem_raw);\n  V* const b1 = b0 + %du;\n", 1u << K);
    g.add("  u64* const hoff = reinterpret_cast<u64*>(b1 + %du);\n", 1u << K);
    g.add("  double2* const ered = reinterpret_cast<double2*>(hoff + %du);\n", hoff_n);
    g.add("  V* const msm = reinterpret_cast<V*>(ered + %d);\n", a.nexp > 0 ? nwarps * a.nexp : 0);
    g.add("  V* const dsm = msm + %d;\n", batched ? NM : 0);
    g.add("  const u32 tid = threadIdx.x;\n");
    g.add("  for (u32 j = tid; j < %du; j += %du) { u64 o = 0;\n", 1u << H, threads);
    g.add("#pragma unroll\n    for (int t = 0; t < %d; ++t) if ((j >> t) & 1u) o |= p.hibit[t];\n    hoff[j] = o; }\n", H);
    for (int o = 0; o < a.nops; ++o)
        if (doff[size_t(o)] >= 0)
            g.add("  for (u32 q = tid; q < %du; q += %du) dsm[%d + q] = p.m[%d + q];\n", 1u << a.cp[o].m,
                  unsigned(threads), doff[size_t(o)], int(a.ops[o].moff));
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
    if (batched) {
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
    g.add("    for (u32 c = tid; c < %du; c += %du) { const u32 e = c * %du;\n", (1u << K) / EPC, threads, EPC);
    g.add("      const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(dst + e));\n");
    g.add("      asm volatile(\"cp.async.cg.shared.global [%%0], [%%1], 16;\\n\" :: \"r\"(sa), "
          "\"l\"(vec + (base | hoff[e >> %d] | (e & %du))) : \"memory\"); }\n", L, (1u << L) - 1u);
    g.add("    asm volatile(\"cp.async.commit_group;\\n\" ::: \"memory\"); };\n");
    g.add("  if (tile < tend) prefetch(b0, tile_base(tile));\n");
    g.add("  for (u32 it = 0; tile < tend; ++it, tile += tstep) {\n");
    g.add("    V* const cur = (it & 1u) ? b1 : b0;\n    const u64 base = tile_base(tile);\n");
    g.add("    asm volatile(\"cp.async.wait_group 0;\\n\" ::: \"memory\");\n    __syncthreads();\n");
    g.add("    if (tile + tstep < tend) prefetch((it & 1u) ? b0 : b1, tile_base(tile + tstep));\n");
    if (batched) {
        g.add("    { const u64 inst = (base & p.misc[0]) >> p.misc[1];\n");
        g.add("      if (inst != staged) {\n");
        g.add("        for (u32 q = tid; q < %du; q += %du) { const u32 v = p.pe[q];\n", unsigned(a.nmats), threads);
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
    for (int s = 0; s < E; ++s) g.add("    vec[base | gthr | p.gslot[%d]] = v%d;\n", s, var[s]);
    if (a.nexp > 0) {
        // per-tile partials: the warps' sums in a fixed order
        g.add("    __syncthreads();\n");
        g.add("    for (u32 e = tid; e < %du; e += %du) { double2 t = make_double2(0.0, 0.0);\n", unsigned(a.nexp),
              threads);
        g.add("      for (int w = 0; w < %d; ++w) { t.x += ered[w * %d + e].x; t.y += ered[w * %d + e].y; }\n", nwarps,
              NEXP, NEXP);
        g.add("      const u64 at = 2 * (p.eslot[e] * ntiles + tile);\n      partials[at] = t.x;\n"
              "      partials[at + 1] = t.y; }\n");
    }
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
        size_t smem = sizeof(V) * (2 * (size_t(1) << ps.k) + args.nmats) + 8 * ((size_t(1) << (ps.k - ps.nlow)) + (1 << R)) +
                      sizeof(KOp) * args.nops + 16 + sizeof(KStage) * args.nstages + args.nmats +
                      (EXP ? 16 + sizeof(double2) * size_t(args.nexp) * (threads / 32) : 0);
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
