// Single-gate streaming kernels: one HBM pass per gate, 64-bit indexing.
//
// Each kernel streams only the amplitudes the gate changes:
//   dense 1q on a bit >= 5 : amplitude pairs, both halves warp-contiguous
//   dense 1q on a bit <  5 : every lane loads one contiguous amplitude and
//                            gets its partner with __shfl_xor_sync
//   diagonal               : flat walk; entries equal to 1 are not touched
//                            (phase gates f = 1/2, controlled phase f = 1/4)
//   anti-diagonal (X, CX)  : pairs (or shuffles for low bits)
//   2q dense / swap        : quads (swap touches only |01>, |10>)
// Reference kernels replaced: QuICT/ops/gate_kernel/gate_function.py:31-1031.
#include "common.cuh"

namespace qs {

namespace {

constexpr int kThreads = 256;
constexpr int kUnroll = 4;
constexpr int kMaxIns = 48;

using Plan = InsertPlan<kMaxIns>;

Plan make_plan(uint64_t mask) {
    Plan p; p.nb = 0;
    for (int b = 0; b < 64; ++b)
        if ((mask >> b) & 1) p.b[p.nb++] = b;
    return p;
}

template <typename V>
__device__ __forceinline__ V shfl_xor(V a, int lanemask) {
    V r;
    r.x = __shfl_xor_sync(0xffffffffu, a.x, lanemask);
    r.y = __shfl_xor_sync(0xffffffffu, a.y, lanemask);
    return r;
}

// ---------------------------------------------------------------- init/scale
template <typename V>
__global__ void __launch_bounds__(kThreads) k_init_zero(V* __restrict__ v, uint64_t N) {
    uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < N; i += stride)
        v[i] = mk<V>(i == 0 ? 1.0 : 0.0, 0.0);
}

template <typename V>
__global__ void __launch_bounds__(kThreads) k_scale(V* __restrict__ v, uint64_t N, V s) {
    uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < N; i += stride)
        v[i] = cmul(v[i], s);
}

// ---------------------------------------------------------------- 1q, pairs
// KIND: QS_K_DENSE or QS_K_ANTIDIAG.  Work item j -> i0 = expand(j) | cmask.
template <typename V, int KIND>
__global__ void __launch_bounds__(kThreads)
k_1q_pair(V* __restrict__ v, uint64_t items, Plan plan, uint64_t cmask, uint64_t off, Mat<V, 4> M) {
    const uint64_t step = uint64_t(gridDim.x) * kThreads * kUnroll;
    for (uint64_t j0 = uint64_t(blockIdx.x) * kThreads * kUnroll + threadIdx.x; j0 < items; j0 += step) {
        V a[kUnroll], b[kUnroll];
        uint64_t i0[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            uint64_t j = j0 + uint64_t(u) * kThreads;
            if (j < items) {
                i0[u] = expand(j, plan) | cmask;
                a[u] = v[i0[u]];
                b[u] = v[i0[u] + off];
            }
        }
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            uint64_t j = j0 + uint64_t(u) * kThreads;
            if (j < items) {
                V x, y;
                if (KIND == QS_K_DENSE) {
                    x = cfma(M.m[0], a[u], cmul(M.m[1], b[u]));
                    y = cfma(M.m[2], a[u], cmul(M.m[3], b[u]));
                } else {
                    x = cmul(M.m[1], b[u]);
                    y = cmul(M.m[2], a[u]);
                }
                v[i0[u]] = x;
                v[i0[u] + off] = y;
            }
        }
    }
}

// complex64, target and control bits >= 1: two adjacent work items are two
// adjacent amplitudes, so each thread moves float4s (128-bit accesses).
template <int KIND>
__global__ void __launch_bounds__(kThreads)
k_1q_pair_v2(float2* __restrict__ v, uint64_t items2, Plan plan, uint64_t cmask, uint64_t off, Mat<float2, 4> M) {
    const uint64_t step = uint64_t(gridDim.x) * kThreads * kUnroll;
    float4* __restrict__ v4 = reinterpret_cast<float4*>(v);
    const uint64_t off4 = off >> 1;
    for (uint64_t j0 = uint64_t(blockIdx.x) * kThreads * kUnroll + threadIdx.x; j0 < items2; j0 += step) {
        float4 a[kUnroll], b[kUnroll];
        uint64_t q[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            const uint64_t j = j0 + uint64_t(u) * kThreads;
            if (j < items2) {
                q[u] = (expand(2 * j, plan) | cmask) >> 1;  // even amplitude index -> float4 index
                a[u] = v4[q[u]];
                b[u] = v4[q[u] + off4];
            }
        }
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            const uint64_t j = j0 + uint64_t(u) * kThreads;
            if (j >= items2) continue;
            const float2 a0 = make_float2(a[u].x, a[u].y), a1 = make_float2(a[u].z, a[u].w);
            const float2 b0 = make_float2(b[u].x, b[u].y), b1 = make_float2(b[u].z, b[u].w);
            float2 x0, y0, x1, y1;
            if (KIND == QS_K_DENSE) {
                x0 = cfma(M.m[0], a0, cmul(M.m[1], b0));
                y0 = cfma(M.m[2], a0, cmul(M.m[3], b0));
                x1 = cfma(M.m[0], a1, cmul(M.m[1], b1));
                y1 = cfma(M.m[2], a1, cmul(M.m[3], b1));
            } else {
                x0 = cmul(M.m[1], b0);
                y0 = cmul(M.m[2], a0);
                x1 = cmul(M.m[1], b1);
                y1 = cmul(M.m[2], a1);
            }
            v4[q[u]] = make_float4(x0.x, x0.y, x1.x, x1.y);
            v4[q[u] + off4] = make_float4(y0.x, y0.y, y1.x, y1.y);
        }
    }
}

// complex64 diagonal with 128-bit accesses: bit 0 is neither fixed nor the
// selector's `hi` bit, so each float4 holds a pair (even, odd) of amplitudes.
__global__ void __launch_bounds__(kThreads)
k_diag_v2(float2* __restrict__ v, uint64_t items2, Plan plan, uint64_t fixed, int bhi, int blo, Mat<float2, 4> D) {
    const uint64_t step = uint64_t(gridDim.x) * kThreads * kUnroll;
    float4* __restrict__ v4 = reinterpret_cast<float4*>(v);
    for (uint64_t j0 = uint64_t(blockIdx.x) * kThreads * kUnroll + threadIdx.x; j0 < items2; j0 += step) {
        float4 a[kUnroll];
        uint64_t idx[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            const uint64_t j = j0 + uint64_t(u) * kThreads;
            if (j < items2) {
                idx[u] = expand(2 * j, plan) | fixed;
                a[u] = v4[idx[u] >> 1];
            }
        }
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            const uint64_t j = j0 + uint64_t(u) * kThreads;
            if (j >= items2) continue;
            int s0 = 0, s1 = 0;
            if (bhi >= 0) s0 = s1 = int((idx[u] >> bhi) & 1) << 1;
            if (blo == 0) {
                s1 |= 1;
            } else if (blo > 0) {
                const int b = int((idx[u] >> blo) & 1);
                s0 |= b;
                s1 |= b;
            }
            const float2 y0 = cmul(make_float2(a[u].x, a[u].y), D.m[s0]);
            const float2 y1 = cmul(make_float2(a[u].z, a[u].w), D.m[s1]);
            v4[idx[u] >> 1] = make_float4(y0.x, y0.y, y1.x, y1.y);
        }
    }
}

// complex64, target bit < 5: each lane moves a float4 (amplitudes 2l, 2l+1
// of a 64-amplitude chunk); the partner of bit 0 is the lane's other half,
// the partner of bit b >= 1 sits in lane l ^ 2^(b-1).  Control bits 0..5 are
// checked per amplitude (cmask_lo), higher ones are fixed by the chunk plan.
template <int KIND>
__global__ void __launch_bounds__(kThreads)
k_1q_shfl_v2(float2* __restrict__ v, uint64_t chunks, Plan plan_hi, uint64_t cmask_hi, uint32_t cmask_lo, int bit,
             Mat<float2, 4> M) {
    const int lane = threadIdx.x & 31;
    const uint64_t warps = uint64_t(gridDim.x) * (kThreads / 32);
    const uint64_t w0 = uint64_t(blockIdx.x) * (kThreads / 32) + (threadIdx.x >> 5);
    float4* __restrict__ v4 = reinterpret_cast<float4*>(v);
    const bool one = bit > 0 && ((lane >> (bit - 1)) & 1);
    const bool act0 = (uint32_t(2 * lane) & cmask_lo) == cmask_lo;
    const bool act1 = (uint32_t(2 * lane + 1) & cmask_lo) == cmask_lo;
    for (uint64_t c0 = w0; c0 < chunks; c0 += warps * kUnroll) {
        float4 a[kUnroll];
        uint64_t q[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            const uint64_t c = c0 + uint64_t(u) * warps;
            if (c < chunks) {  // warp-uniform
                q[u] = ((expand(c << 6, plan_hi) | cmask_hi) >> 1) + lane;
                a[u] = v4[q[u]];
            }
        }
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            const uint64_t c = c0 + uint64_t(u) * warps;
            if (c >= chunks) continue;
            const float2 x0 = make_float2(a[u].x, a[u].y), x1 = make_float2(a[u].z, a[u].w);
            float2 y0, y1;
            if (bit == 0) {
                if (KIND == QS_K_DENSE) {
                    y0 = cfma(M.m[0], x0, cmul(M.m[1], x1));
                    y1 = cfma(M.m[2], x0, cmul(M.m[3], x1));
                } else {
                    y0 = cmul(M.m[1], x1);
                    y1 = cmul(M.m[2], x0);
                }
            } else {
                const int pm = 1 << (bit - 1);
                float4 pa;
                pa.x = __shfl_xor_sync(0xffffffffu, a[u].x, pm);
                pa.y = __shfl_xor_sync(0xffffffffu, a[u].y, pm);
                pa.z = __shfl_xor_sync(0xffffffffu, a[u].z, pm);
                pa.w = __shfl_xor_sync(0xffffffffu, a[u].w, pm);
                const float2 p0 = make_float2(pa.x, pa.y), p1 = make_float2(pa.z, pa.w);
                if (KIND == QS_K_DENSE) {
                    y0 = one ? cfma(M.m[2], p0, cmul(M.m[3], x0)) : cfma(M.m[0], x0, cmul(M.m[1], p0));
                    y1 = one ? cfma(M.m[2], p1, cmul(M.m[3], x1)) : cfma(M.m[0], x1, cmul(M.m[1], p1));
                } else {
                    y0 = one ? cmul(M.m[2], p0) : cmul(M.m[1], p0);
                    y1 = one ? cmul(M.m[2], p1) : cmul(M.m[1], p1);
                }
            }
            if (!act0) y0 = x0;
            if (!act1) y1 = x1;
            if (act0 || act1) v4[q[u]] = make_float4(y0.x, y0.y, y1.x, y1.y);
        }
    }
}

// ------------------------------------------------------------ 1q, shuffles
// Target bit < 5 and n >= 5.  Each warp owns 32 consecutive amplitudes of the
// compact space (control bits >= 5 removed); lane partner = lane ^ (1<<bit).
template <typename V, int KIND>
__global__ void __launch_bounds__(kThreads)
k_1q_shfl(V* __restrict__ v, uint64_t chunks, Plan plan_hi, uint64_t cmask_hi, uint32_t cmask_lo,
          int bit, Mat<V, 4> M) {
    const int lane = threadIdx.x & 31;
    const uint64_t warps = uint64_t(gridDim.x) * (kThreads / 32);
    const uint64_t w0 = uint64_t(blockIdx.x) * (kThreads / 32) + (threadIdx.x >> 5);
    const bool one = (lane >> bit) & 1;
    const bool active = (uint32_t(lane) & cmask_lo) == cmask_lo;
    for (uint64_t c0 = w0; c0 < chunks; c0 += warps * kUnroll) {
        V a[kUnroll];
        uint64_t idx[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            uint64_t c = c0 + uint64_t(u) * warps;
            if (c < chunks) {  // warp-uniform
                idx[u] = (expand(c << 5, plan_hi) | cmask_hi) + lane;
                a[u] = v[idx[u]];
            }
        }
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            uint64_t c = c0 + uint64_t(u) * warps;
            if (c < chunks) {
                V p = shfl_xor(a[u], 1 << bit);
                V out;
                if (KIND == QS_K_DENSE) {
                    out = one ? cfma(M.m[2], p, cmul(M.m[3], a[u])) : cfma(M.m[0], a[u], cmul(M.m[1], p));
                } else {
                    out = one ? cmul(M.m[2], p) : cmul(M.m[1], p);
                }
                if (active) v[idx[u]] = out;
            }
        }
    }
}

// ------------------------------------------- 1q, controls among the low bits
// Target bit < 5 with controls below bit 5: the lanes walk the 5 lowest bits
// that are not controls (lanemask) and every control bit is fixed to 1, so a
// warp loads and stores only amplitudes the gate changes (the chunk kernels
// above load the whole 32- or 64-amplitude chunk and store the lanes whose
// controls are set: 1.5x the bytes for one control).  r: the target's
// position among the lane bits; its partner is lane ^ 2^r.
__device__ __forceinline__ uint64_t lane_offset(int lane, uint64_t lanemask) {
    uint64_t o = 0;
    for (int i = 0, b = 0; i < 5; ++b)
        if ((lanemask >> b) & 1) {
            if ((lane >> i) & 1) o |= uint64_t(1) << b;
            ++i;
        }
    return o;
}

template <typename V, int KIND>
__global__ void __launch_bounds__(kThreads)
k_1q_lanes(V* __restrict__ v, uint64_t chunks, Plan plan, uint64_t cmask, uint64_t lanemask, int r, Mat<V, 4> M) {
    const int lane = threadIdx.x & 31;
    const uint64_t warps = uint64_t(gridDim.x) * (kThreads / 32);
    const uint64_t w0 = uint64_t(blockIdx.x) * (kThreads / 32) + (threadIdx.x >> 5);
    const uint64_t loff = lane_offset(lane, lanemask) | cmask;
    const bool one = (lane >> r) & 1;
    for (uint64_t c0 = w0; c0 < chunks; c0 += warps * kUnroll) {
        V a[kUnroll];
        uint64_t idx[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            const uint64_t c = c0 + uint64_t(u) * warps;
            if (c < chunks) {  // warp-uniform
                idx[u] = expand(c, plan) | loff;
                a[u] = v[idx[u]];
            }
        }
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            const uint64_t c = c0 + uint64_t(u) * warps;
            if (c >= chunks) continue;
            const V p = shfl_xor(a[u], 1 << r);
            V out;
            if (KIND == QS_K_DENSE) out = one ? cfma(M.m[2], p, cmul(M.m[3], a[u])) : cfma(M.m[0], a[u], cmul(M.m[1], p));
            else out = one ? cmul(M.m[2], p) : cmul(M.m[1], p);
            v[idx[u]] = out;
        }
    }
}

// complex64 form with 128-bit accesses (bit 0 is not a control): each lane
// moves the amplitude pair (bit 0 = 0, 1) as a float4; the lanes walk the 5
// lowest non-control bits above bit 0.  A target on bit 0 is the lane's own
// pair; any other target's partner is lane ^ 2^r.
template <int KIND>
__global__ void __launch_bounds__(kThreads)
k_1q_lanes_v2(float2* __restrict__ v, uint64_t chunks, Plan plan, uint64_t cmask, uint64_t lanemask, int bit, int r,
              Mat<float2, 4> M) {
    const int lane = threadIdx.x & 31;
    const uint64_t warps = uint64_t(gridDim.x) * (kThreads / 32);
    const uint64_t w0 = uint64_t(blockIdx.x) * (kThreads / 32) + (threadIdx.x >> 5);
    float4* __restrict__ v4 = reinterpret_cast<float4*>(v);
    const uint64_t loff = lane_offset(lane, lanemask) | cmask;
    const bool one = bit > 0 && ((lane >> r) & 1);
    for (uint64_t c0 = w0; c0 < chunks; c0 += warps * kUnroll) {
        float4 a[kUnroll];
        uint64_t q[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            const uint64_t c = c0 + uint64_t(u) * warps;
            if (c < chunks) {  // warp-uniform
                q[u] = (expand(c, plan) | loff) >> 1;
                a[u] = v4[q[u]];
            }
        }
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            const uint64_t c = c0 + uint64_t(u) * warps;
            if (c >= chunks) continue;
            const float2 x0 = make_float2(a[u].x, a[u].y), x1 = make_float2(a[u].z, a[u].w);
            float2 y0, y1;
            if (bit == 0) {
                if (KIND == QS_K_DENSE) {
                    y0 = cfma(M.m[0], x0, cmul(M.m[1], x1));
                    y1 = cfma(M.m[2], x0, cmul(M.m[3], x1));
                } else {
                    y0 = cmul(M.m[1], x1);
                    y1 = cmul(M.m[2], x0);
                }
            } else {
                const int pm = 1 << r;
                const float2 p0 = make_float2(__shfl_xor_sync(0xffffffffu, a[u].x, pm),
                                              __shfl_xor_sync(0xffffffffu, a[u].y, pm));
                const float2 p1 = make_float2(__shfl_xor_sync(0xffffffffu, a[u].z, pm),
                                              __shfl_xor_sync(0xffffffffu, a[u].w, pm));
                if (KIND == QS_K_DENSE) {
                    y0 = one ? cfma(M.m[2], p0, cmul(M.m[3], x0)) : cfma(M.m[0], x0, cmul(M.m[1], p0));
                    y1 = one ? cfma(M.m[2], p1, cmul(M.m[3], x1)) : cfma(M.m[0], x1, cmul(M.m[1], p1));
                } else {
                    y0 = one ? cmul(M.m[2], p0) : cmul(M.m[1], p0);
                    y1 = one ? cmul(M.m[2], p1) : cmul(M.m[1], p1);
                }
            }
            v4[q[u]] = make_float4(y0.x, y0.y, y1.x, y1.y);
        }
    }
}

// ------------------------------------------------------------- diagonal, flat
// Walks the compact space of the non-fixed bits; amplitude i gets factor
// D[sel(i)], sel built from up to two diagonal bits (hi, lo).  `fixed` bits are
// forced to 1 (controls, and targets whose 0-entries are skipped).
template <typename V>
__global__ void __launch_bounds__(kThreads)
k_diag(V* __restrict__ v, uint64_t items, Plan plan, uint64_t fixed, int bhi, int blo, Mat<V, 4> D) {
    const uint64_t step = uint64_t(gridDim.x) * kThreads * kUnroll;
    for (uint64_t j0 = uint64_t(blockIdx.x) * kThreads * kUnroll + threadIdx.x; j0 < items; j0 += step) {
        V a[kUnroll];
        uint64_t idx[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            uint64_t j = j0 + uint64_t(u) * kThreads;
            if (j < items) {
                idx[u] = expand(j, plan) | fixed;
                a[u] = v[idx[u]];
            }
        }
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            uint64_t j = j0 + uint64_t(u) * kThreads;
            if (j < items) {
                int s = 0;
                if (bhi >= 0) s |= int((idx[u] >> bhi) & 1) << 1;
                if (blo >= 0) s |= int((idx[u] >> blo) & 1);
                v[idx[u]] = cmul(a[u], D.m[s]);
            }
        }
    }
}

// ------------------------------------------------------------------ 2q quads
template <typename V, int KIND>
__global__ void __launch_bounds__(kThreads)
k_2q_quad(V* __restrict__ v, uint64_t items, Plan plan, uint64_t cmask, uint64_t ohi, uint64_t olo,
          Mat<V, 16> M, bool touch_diag) {
    // four quads per thread, all loads issued before any store: 16 (dense)
    // or 8 (swap) independent loads in flight per thread
    constexpr int U = 4;
    const uint64_t step = uint64_t(gridDim.x) * kThreads * U;
    for (uint64_t j0 = uint64_t(blockIdx.x) * kThreads * U + threadIdx.x; j0 < items; j0 += step) {
        uint64_t i00[U];
        V x[U][4];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint64_t j = j0 + uint64_t(u) * kThreads;
            if (j < items) {
                i00[u] = expand(j, plan) | cmask;
                if (KIND == QS_K_DENSE || touch_diag) x[u][0] = v[i00[u]];
                x[u][1] = v[i00[u] | olo];
                x[u][2] = v[i00[u] | ohi];
                if (KIND == QS_K_DENSE || touch_diag) x[u][3] = v[i00[u] | ohi | olo];
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint64_t j = j0 + uint64_t(u) * kThreads;
            if (j >= items) continue;
            const uint64_t i01 = i00[u] | olo, i10 = i00[u] | ohi, i11 = i00[u] | ohi | olo;
            if (KIND == QS_K_DENSE) {
                V y[4];
#pragma unroll
                for (int r = 0; r < 4; ++r) {
                    V acc = cmul(M.m[4 * r + 0], x[u][0]);
                    acc = cfma(M.m[4 * r + 1], x[u][1], acc);
                    acc = cfma(M.m[4 * r + 2], x[u][2], acc);
                    acc = cfma(M.m[4 * r + 3], x[u][3], acc);
                    y[r] = acc;
                }
                v[i00[u]] = y[0]; v[i01] = y[1]; v[i10] = y[2]; v[i11] = y[3];
            } else {  // QS_K_SWAP
                v[i01] = cmul(M.m[6], x[u][2]);
                v[i10] = cmul(M.m[9], x[u][1]);
                if (touch_diag) {
                    v[i00[u]] = cmul(M.m[0], x[u][0]);
                    v[i11] = cmul(M.m[15], x[u][3]);
                }
            }
        }
    }
}

// --------------------------------------------------------- k-qubit dense, K<=4
template <typename V, int K>
__global__ void __launch_bounds__(128)
k_kq_reg(V* __restrict__ v, uint64_t items, Plan plan, uint64_t cmask, InsertPlan<10> spread,
         const double2* __restrict__ M) {
    constexpr int D = 1 << K;
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t j = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < items; j += stride) {
        uint64_t base = expand(j, plan) | cmask;
        uint64_t idx[D];
        V x[D];
#pragma unroll
        for (int r = 0; r < D; ++r) {
            uint64_t o = 0;
#pragma unroll
            for (int t = 0; t < K; ++t)
                if ((r >> (K - 1 - t)) & 1) o |= uint64_t(1) << spread.b[t];
            idx[r] = base | o;
            x[r] = v[idx[r]];
        }
#pragma unroll
        for (int r = 0; r < D; ++r) {
            V acc = mk<V>(0.0, 0.0);
#pragma unroll
            for (int c = 0; c < D; ++c) {
                double2 m = __ldg(&M[r * D + c]);
                acc = cfma(mk<V>(m.x, m.y), x[c], acc);
            }
            v[idx[r]] = acc;
        }
    }
}

// -------------------------------------------------- k-qubit dense, 5<=K<=10
// One CTA per group: gather 2^k amplitudes into shared memory, each thread
// produces rows r = tid, tid + blockDim ...
template <typename V>
__global__ void __launch_bounds__(256)
k_kq_smem(V* __restrict__ v, uint64_t items, Plan plan, uint64_t cmask, InsertPlan<10> spread, int k,
          const double2* __restrict__ M) {
    extern __shared__ unsigned char smem_raw[];
    V* s = reinterpret_cast<V*>(smem_raw);
    const int D = 1 << k;
    for (uint64_t j = blockIdx.x; j < items; j += gridDim.x) {
        uint64_t base = expand(j, plan) | cmask;
        __syncthreads();
        for (int r = threadIdx.x; r < D; r += blockDim.x) {
            uint64_t o = 0;
            for (int t = 0; t < k; ++t)
                if ((r >> (k - 1 - t)) & 1) o |= uint64_t(1) << spread.b[t];
            s[r] = v[base | o];
        }
        __syncthreads();
        for (int r = threadIdx.x; r < D; r += blockDim.x) {
            V acc = mk<V>(0.0, 0.0);
            for (int c = 0; c < D; ++c) {
                double2 m = M[uint64_t(r) * D + c];
                acc = cfma(mk<V>(m.x, m.y), s[c], acc);
            }
            uint64_t o = 0;
            for (int t = 0; t < k; ++t)
                if ((r >> (k - 1 - t)) & 1) o |= uint64_t(1) << spread.b[t];
            v[base | o] = acc;
        }
    }
}

// ------------------------------------------------------------------ host side
bool is_one(const double* z) { return z[0] == 1.0 && z[1] == 0.0; }

int check_common(void* vec, int n, int dtype) {
    QS_REQUIRE(vec != nullptr, "null state vector");
    QS_REQUIRE(n >= 1 && n <= 40, "qubit count %d outside [1, 40]", n);
    QS_REQUIRE(valid_dtype(dtype), "bad dtype %d", dtype);
    return QS_OK;
}

// Diagonal launch: complex64 pairs of adjacent amplitudes move as float4
// when bit 0 is neither fixed nor the selector's high bit.
template <typename V>
void launch_diag(V* v, uint64_t items, const Plan& p, uint64_t fixed, int bhi, int blo, const Mat<V, 4>& D,
                 cudaStream_t st) {
    if constexpr (sizeof(V) == 8) {
        if (!(fixed & 1) && bhi != 0 && items >= 2) {
            const uint64_t items2 = items >> 1;
            k_diag_v2<<<grid_for(items2, kThreads * kUnroll, 8), kThreads, 0, st>>>((float2*)v, items2, p, fixed, bhi,
                                                                                   blo, D);
            return;
        }
    }
    k_diag<V><<<grid_for(items, kThreads * kUnroll, 8), kThreads, 0, st>>>(v, items, p, fixed, bhi, blo, D);
}

template <typename R>
int apply_1q_t(void* vec, int n, int bit, uint64_t cmask, int kind, const double* mat, cudaStream_t st) {
    using V = typename CT<R>::V;
    V* v = static_cast<V*>(vec);
    Mat<V, 4> M = load_host_mat<V, 4>(mat);
    const uint64_t tbit = uint64_t(1) << bit;
    if (kind == QS_K_DIAG) {
        bool skip0 = is_one(mat);
        if (skip0 && is_one(mat + 6)) return QS_OK;  // identity
        uint64_t fixed = cmask | (skip0 ? tbit : 0);
        Plan p = make_plan(fixed);
        uint64_t items = uint64_t(1) << (n - p.nb);
        Mat<V, 4> D;
        D.m[0] = M.m[0]; D.m[1] = M.m[3]; D.m[2] = M.m[0]; D.m[3] = M.m[3];
        launch_diag<V>(v, items, p, fixed, -1, bit, D, st);
        QS_CHECK_LAUNCH("qs_apply_1q(diag)");
        return QS_OK;
    }
    if (bit < 5 && (cmask & 31) != 0) {  // controls among the low bits: lanes on the free bits
        // the 5 lowest non-control bits from `from` up, as a mask (0 if too few)
        auto lane_bits = [&](int from) -> uint64_t {
            uint64_t lm = 0;
            int cnt = 0;
            for (int b = from; b < n && cnt < 5; ++b)
                if (!((cmask >> b) & 1)) {
                    lm |= uint64_t(1) << b;
                    ++cnt;
                }
            return cnt == 5 ? lm : 0;
        };
        if constexpr (sizeof(V) == 8) {
            const uint64_t lm = (cmask & 1) ? 0 : lane_bits(1);
            if (lm != 0) {
                const int r = bit == 0 ? 0 : __builtin_popcountll(lm & ((uint64_t(1) << bit) - 1));
                Plan p = make_plan(cmask | lm | 1);
                const uint64_t chunks = uint64_t(1) << (n - p.nb);
                const unsigned grid = grid_for(chunks, (kThreads / 32) * kUnroll, 8);
                if (kind == QS_K_DENSE)
                    k_1q_lanes_v2<QS_K_DENSE><<<grid, kThreads, 0, st>>>((float2*)v, chunks, p, cmask, lm, bit, r, M);
                else
                    k_1q_lanes_v2<QS_K_ANTIDIAG><<<grid, kThreads, 0, st>>>((float2*)v, chunks, p, cmask, lm, bit, r,
                                                                           M);
                QS_CHECK_LAUNCH("qs_apply_1q(low controls, float4)");
                return QS_OK;
            }
        }
        const uint64_t lm = lane_bits(0);
        if (lm != 0) {
            const int r = __builtin_popcountll(lm & ((uint64_t(1) << bit) - 1));
            Plan p = make_plan(cmask | lm);
            const uint64_t chunks = uint64_t(1) << (n - p.nb);
            const unsigned grid = grid_for(chunks, (kThreads / 32) * kUnroll, 8);
            if (kind == QS_K_DENSE)
                k_1q_lanes<V, QS_K_DENSE><<<grid, kThreads, 0, st>>>(v, chunks, p, cmask, lm, r, M);
            else
                k_1q_lanes<V, QS_K_ANTIDIAG><<<grid, kThreads, 0, st>>>(v, chunks, p, cmask, lm, r, M);
            QS_CHECK_LAUNCH("qs_apply_1q(low controls)");
            return QS_OK;
        }
    }
    if constexpr (sizeof(V) == 8) {
        if (bit < 5 && n >= 6) {  // 64-amplitude chunks, float4 per lane
            const uint64_t chi = cmask & ~uint64_t(63);
            Plan p = make_plan(chi);
            uint64_t chunks = (uint64_t(1) << (n - p.nb)) >> 6;
            unsigned grid = grid_for(chunks, (kThreads / 32) * kUnroll, 8);
            if (kind == QS_K_DENSE)
                k_1q_shfl_v2<QS_K_DENSE><<<grid, kThreads, 0, st>>>((float2*)v, chunks, p, chi, uint32_t(cmask & 63),
                                                                    bit, M);
            else
                k_1q_shfl_v2<QS_K_ANTIDIAG><<<grid, kThreads, 0, st>>>((float2*)v, chunks, p, chi,
                                                                       uint32_t(cmask & 63), bit, M);
            QS_CHECK_LAUNCH("qs_apply_1q(shfl, float4)");
            return QS_OK;
        }
    }
    const uint64_t cmask_hi = cmask & ~uint64_t(31);
    if (bit < 5 && n >= 5) {
        Plan p = make_plan(cmask_hi);
        uint64_t chunks = (uint64_t(1) << (n - p.nb)) >> 5;
        unsigned grid = grid_for(chunks, (kThreads / 32) * kUnroll, 8);
        if (kind == QS_K_DENSE)
            k_1q_shfl<V, QS_K_DENSE><<<grid, kThreads, 0, st>>>(v, chunks, p, cmask_hi, uint32_t(cmask & 31), bit, M);
        else
            k_1q_shfl<V, QS_K_ANTIDIAG><<<grid, kThreads, 0, st>>>(v, chunks, p, cmask_hi, uint32_t(cmask & 31), bit, M);
        QS_CHECK_LAUNCH("qs_apply_1q(shfl)");
        return QS_OK;
    }
    Plan p = make_plan(cmask | tbit);
    uint64_t items = uint64_t(1) << (n - p.nb);
    if constexpr (sizeof(V) == 8) {
        if (!(cmask & 1) && bit >= 1 && items >= 2) {  // adjacent amplitude pairs: float4 accesses
            const uint64_t items2 = items >> 1;
            unsigned grid2 = grid_for(items2, kThreads * kUnroll, 8);
            if (kind == QS_K_DENSE)
                k_1q_pair_v2<QS_K_DENSE><<<grid2, kThreads, 0, st>>>((float2*)v, items2, p, cmask, tbit, M);
            else
                k_1q_pair_v2<QS_K_ANTIDIAG><<<grid2, kThreads, 0, st>>>((float2*)v, items2, p, cmask, tbit, M);
            QS_CHECK_LAUNCH("qs_apply_1q(pair, float4)");
            return QS_OK;
        }
    }
    unsigned grid = grid_for(items, kThreads * kUnroll, 8);
    if (kind == QS_K_DENSE)
        k_1q_pair<V, QS_K_DENSE><<<grid, kThreads, 0, st>>>(v, items, p, cmask, tbit, M);
    else
        k_1q_pair<V, QS_K_ANTIDIAG><<<grid, kThreads, 0, st>>>(v, items, p, cmask, tbit, M);
    QS_CHECK_LAUNCH("qs_apply_1q(pair)");
    return QS_OK;
}

template <typename R>
int apply_2q_t(void* vec, int n, int bhi, int blo, uint64_t cmask, int kind, const double* mat, cudaStream_t st) {
    using V = typename CT<R>::V;
    V* v = static_cast<V*>(vec);
    Mat<V, 16> M = load_host_mat<V, 16>(mat);
    const uint64_t ohi = uint64_t(1) << bhi, olo = uint64_t(1) << blo;
    if (kind == QS_K_DIAG) {
        Plan p = make_plan(cmask);
        uint64_t items = uint64_t(1) << (n - p.nb);
        Mat<V, 4> D;
        D.m[0] = M.m[0]; D.m[1] = M.m[5]; D.m[2] = M.m[10]; D.m[3] = M.m[15];
        launch_diag<V>(v, items, p, cmask, bhi, blo, D, st);
        QS_CHECK_LAUNCH("qs_apply_2q(diag)");
        return QS_OK;
    }
    Plan p = make_plan(cmask | ohi | olo);
    uint64_t items = uint64_t(1) << (n - p.nb);
    unsigned grid = grid_for(items, kThreads * 4, 8);
    if (kind == QS_K_DENSE) {
        k_2q_quad<V, QS_K_DENSE><<<grid, kThreads, 0, st>>>(v, items, p, cmask, ohi, olo, M, true);
    } else {
        bool touch = !(is_one(mat) && is_one(mat + 30));
        k_2q_quad<V, QS_K_SWAP><<<grid, kThreads, 0, st>>>(v, items, p, cmask, ohi, olo, M, touch);
    }
    QS_CHECK_LAUNCH("qs_apply_2q");
    return QS_OK;
}

template <typename R>
int apply_kq_t(void* vec, int n, int k, const int32_t* bits, uint64_t cmask, const void* mat, cudaStream_t st) {
    using V = typename CT<R>::V;
    V* v = static_cast<V*>(vec);
    uint64_t tmask = 0;
    InsertPlan<10> spread; spread.nb = k;
    for (int t = 0; t < k; ++t) { spread.b[t] = bits[t]; tmask |= uint64_t(1) << bits[t]; }
    Plan p = make_plan(cmask | tmask);
    uint64_t items = uint64_t(1) << (n - p.nb);
    const double2* M = static_cast<const double2*>(mat);
    switch (k) {
        case 1: k_kq_reg<V, 1><<<grid_for(items, 128, 16), 128, 0, st>>>(v, items, p, cmask, spread, M); break;
        case 2: k_kq_reg<V, 2><<<grid_for(items, 128, 16), 128, 0, st>>>(v, items, p, cmask, spread, M); break;
        case 3: k_kq_reg<V, 3><<<grid_for(items, 128, 16), 128, 0, st>>>(v, items, p, cmask, spread, M); break;
        case 4: k_kq_reg<V, 4><<<grid_for(items, 128, 16), 128, 0, st>>>(v, items, p, cmask, spread, M); break;
        default: {
            size_t sm = sizeof(V) << k;
            k_kq_smem<V><<<grid_for(items, 1, 8), 256, sm, st>>>(v, items, p, cmask, spread, k, M);
        }
    }
    QS_CHECK_LAUNCH("qs_apply_kq");
    return QS_OK;
}

}  // namespace
}  // namespace qs

using namespace qs;

extern "C" int qs_init_zero(void* vec, int n, int dtype, void* stream) {
    int rc = check_common(vec, n, dtype);
    if (rc) return rc;
    uint64_t N = uint64_t(1) << n;
    unsigned grid = grid_for(N, kThreads, 8);
    if (dtype == QS_C128) k_init_zero<double2><<<grid, kThreads, 0, as_stream(stream)>>>((double2*)vec, N);
    else                  k_init_zero<float2><<<grid, kThreads, 0, as_stream(stream)>>>((float2*)vec, N);
    QS_CHECK_LAUNCH("qs_init_zero");
    return QS_OK;
}

extern "C" int qs_scale(void* vec, int n, int dtype, double re, double im, void* stream) {
    int rc = check_common(vec, n, dtype);
    if (rc) return rc;
    uint64_t N = uint64_t(1) << n;
    unsigned grid = grid_for(N, kThreads, 8);
    if (dtype == QS_C128) k_scale<double2><<<grid, kThreads, 0, as_stream(stream)>>>((double2*)vec, N, mk<double2>(re, im));
    else                  k_scale<float2><<<grid, kThreads, 0, as_stream(stream)>>>((float2*)vec, N, mk<float2>(re, im));
    QS_CHECK_LAUNCH("qs_scale");
    return QS_OK;
}

extern "C" int qs_apply_1q(void* vec, int n, int dtype, int bit, uint64_t ctrl_mask, int kind,
                           const double* mat, void* stream) {
    int rc = check_common(vec, n, dtype);
    if (rc) return rc;
    QS_REQUIRE(mat != nullptr, "null matrix");
    QS_REQUIRE(bit >= 0 && bit < n, "target bit %d outside [0, %d)", bit, n);
    QS_REQUIRE((ctrl_mask >> n) == 0, "control mask has bits >= n");
    QS_REQUIRE(!((ctrl_mask >> bit) & 1), "target bit %d is also a control", bit);
    QS_REQUIRE(kind == QS_K_DENSE || kind == QS_K_DIAG || kind == QS_K_ANTIDIAG, "bad 1q kind %d", kind);
    if (dtype == QS_C128) return apply_1q_t<double>(vec, n, bit, ctrl_mask, kind, mat, as_stream(stream));
    return apply_1q_t<float>(vec, n, bit, ctrl_mask, kind, mat, as_stream(stream));
}

extern "C" int qs_apply_2q(void* vec, int n, int dtype, int bit_hi, int bit_lo, uint64_t ctrl_mask,
                           int kind, const double* mat, void* stream) {
    int rc = check_common(vec, n, dtype);
    if (rc) return rc;
    QS_REQUIRE(mat != nullptr, "null matrix");
    QS_REQUIRE(n >= 2, "2-qubit gate on a %d-qubit vector", n);
    QS_REQUIRE(bit_hi >= 0 && bit_hi < n && bit_lo >= 0 && bit_lo < n && bit_hi != bit_lo,
               "bad target bits (%d, %d) for n=%d", bit_hi, bit_lo, n);
    QS_REQUIRE((ctrl_mask >> n) == 0, "control mask has bits >= n");
    QS_REQUIRE(!((ctrl_mask >> bit_hi) & 1) && !((ctrl_mask >> bit_lo) & 1), "target bit is also a control");
    QS_REQUIRE(kind == QS_K_DENSE || kind == QS_K_DIAG || kind == QS_K_SWAP, "bad 2q kind %d", kind);
    if (dtype == QS_C128) return apply_2q_t<double>(vec, n, bit_hi, bit_lo, ctrl_mask, kind, mat, as_stream(stream));
    return apply_2q_t<float>(vec, n, bit_hi, bit_lo, ctrl_mask, kind, mat, as_stream(stream));
}

extern "C" int qs_apply_kq(void* vec, int n, int dtype, int k, const int32_t* bits, uint64_t ctrl_mask,
                           const void* mat_dev, void* stream) {
    int rc = check_common(vec, n, dtype);
    if (rc) return rc;
    QS_REQUIRE(bits != nullptr && mat_dev != nullptr, "null bits or matrix");
    QS_REQUIRE(k >= 1 && k <= 10 && k <= n, "k=%d outside [1, min(10, n)]", k);
    QS_REQUIRE((ctrl_mask >> n) == 0, "control mask has bits >= n");
    uint64_t seen = 0;
    for (int t = 0; t < k; ++t) {
        QS_REQUIRE(bits[t] >= 0 && bits[t] < n, "target bit %d outside [0, %d)", bits[t], n);
        QS_REQUIRE(!((seen >> bits[t]) & 1), "duplicate target bit %d", bits[t]);
        QS_REQUIRE(!((ctrl_mask >> bits[t]) & 1), "target bit %d is also a control", bits[t]);
        seen |= uint64_t(1) << bits[t];
    }
    if (dtype == QS_C128) return apply_kq_t<double>(vec, n, k, bits, ctrl_mask, mat_dev, as_stream(stream));
    return apply_kq_t<float>(vec, n, k, bits, ctrl_mask, mat_dev, as_stream(stream));
}
