// Shared device/host helpers for libqsim (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/qsim.h"

namespace qs {

// ---- error plumbing --------------------------------------------------------
void set_error(const char* fmt, ...);

#define QS_REQUIRE(cond, ...)                  \
    do {                                       \
        if (!(cond)) {                         \
            ::qs::set_error(__VA_ARGS__);      \
            return QS_EINVAL;                  \
        }                                      \
    } while (0)

#define QS_CHECK_LAUNCH(what)                                              \
    do {                                                                   \
        cudaError_t _e = cudaGetLastError();                               \
        if (_e != cudaSuccess) {                                           \
            ::qs::set_error("%s: %s", what, cudaGetErrorString(_e));       \
            return QS_ECUDA;                                               \
        }                                                                  \
    } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

int sm_count();  // cached per device

// ---- complex arithmetic on float2 / double2 --------------------------------
template <typename R> struct CT;
template <> struct CT<float>  { using V = float2;  };
template <> struct CT<double> { using V = double2; };

template <typename V> __host__ __device__ __forceinline__ V mk(double re, double im) {
    V v; v.x = re; v.y = im; return v;
}
template <typename V> __device__ __forceinline__ V cadd(V a, V b) { V r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename V> __device__ __forceinline__ V cmul(V a, V b) {
    V r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.x * b.y + a.y * b.x;
    return r;
}
// a*b + c with fused multiply-adds
template <typename V> __device__ __forceinline__ V cfma(V a, V b, V c) {
    V r;
    r.x = fma(a.x, b.x, fma(-a.y, b.y, c.x));
    r.y = fma(a.x, b.y, fma(a.y, b.x, c.y));
    return r;
}
template <typename V> __device__ __forceinline__ V cscale(V a, double s) {
    V r; r.x = a.x * s; r.y = a.y * s; return r;
}
template <typename V> __device__ __forceinline__ double cnorm2(V a) {
    double x = a.x, y = a.y;
    return fma(x, x, y * y);
}

// Host-side matrix packet passed by value into kernels.
template <typename V, int N> struct Mat { V m[N]; };

template <typename V, int N>
inline Mat<V, N> load_host_mat(const double* src) {
    Mat<V, N> r;
    for (int i = 0; i < N; ++i) {
        r.m[i].x = static_cast<decltype(r.m[i].x)>(src[2 * i]);
        r.m[i].y = static_cast<decltype(r.m[i].y)>(src[2 * i + 1]);
    }
    return r;
}

// ---- bit helpers -------------------------------------------------------------
// Insert a zero bit at position b of x.
__host__ __device__ __forceinline__ uint64_t insert0(uint64_t x, int b) {
    uint64_t lo = x & ((uint64_t(1) << b) - 1);
    return ((x >> b) << (b + 1)) | lo;
}

// Positions (ascending) of the set bits of `mask`, at most 64.
struct SortedBits {
    int n;
    int pos[64];
};
inline SortedBits sorted_bits(uint64_t mask) {
    SortedBits s; s.n = 0;
    for (int b = 0; b < 64; ++b)
        if ((mask >> b) & 1) s.pos[s.n++] = b;
    return s;
}

// Expand a compact index into the vector index whose `m` sorted zero-bit
// positions are removed (ascending order required).
template <int MAXB>
struct InsertPlan {
    int nb;
    int b[MAXB];
};
template <int MAXB>
__device__ __forceinline__ uint64_t expand(uint64_t x, const InsertPlan<MAXB>& p) {
#pragma unroll 1
    for (int i = 0; i < p.nb; ++i) x = insert0(x, p.b[i]);
    return x;
}

inline bool valid_dtype(int dtype) { return dtype == QS_C64 || dtype == QS_C128; }

// grid size helper: enough CTAs to cover `items` at `per_cta` each, capped at
// `waves` full waves of `ctas_per_sm` per SM.
inline unsigned grid_for(uint64_t items, uint64_t per_cta, int ctas_per_sm, int waves = 1) {
    uint64_t need = (items + per_cta - 1) / per_cta;
    uint64_t cap = uint64_t(sm_count()) * ctas_per_sm * waves;
    if (need < 1) need = 1;
    return static_cast<unsigned>(need < cap ? need : cap);
}

}  // namespace qs
