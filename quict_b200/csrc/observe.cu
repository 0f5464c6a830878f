// Observables: Pauli-sum application (lam = H psi), per-instance inner
// products and segment sums of FP64 partials.  All reductions accumulate in
// FP64 in a fixed order (deterministic).
#include <algorithm>

#include "common.cuh"

namespace qs {
namespace {

constexpr int kThreads = 256;
constexpr int kMaxTerms = 128;
constexpr uint64_t kMaxInnerBlocks = 1024;  // partial sums per instance (workspace: 16 B each)

// Terms sorted by X mask; group g holds terms [gbeg[g], gbeg[g+1]) sharing x[g].
struct PauliTerms {
    int n, ngroups;
    uint64_t x[kMaxTerms];                   // per group
    int gbeg[kMaxTerms + 1];
    uint64_t z[kMaxTerms];                   // per term
    double cre[kMaxTerms], cim[kMaxTerms];  // coefficient times i^popc(x & z)
};

// out[j] = sum_t c_t (-1)^popc(z_t & (j ^ x_t)) psi[j ^ x_t]: per group of
// terms with the same X mask, psi[j ^ x] is read once and multiplied by the
// group's signed coefficient sum (FP64)
template <typename V>
__global__ void __launch_bounds__(kThreads)
k_pauli_sum(const V* __restrict__ psi, V* __restrict__ out, uint64_t N, const __grid_constant__ PauliTerms p) {
    const uint64_t stride = uint64_t(gridDim.x) * kThreads;
    for (uint64_t j = uint64_t(blockIdx.x) * kThreads + threadIdx.x; j < N; j += stride) {
        double re = 0.0, im = 0.0;
        for (int g = 0; g < p.ngroups; ++g) {
            const uint64_t src = j ^ p.x[g];
            const V a = psi[src];
            double sr = 0.0, si = 0.0;
            for (int t = p.gbeg[g]; t < p.gbeg[g + 1]; ++t) {
                const bool neg = __popcll(p.z[t] & src) & 1;
                sr += neg ? -p.cre[t] : p.cre[t];
                si += neg ? -p.cim[t] : p.cim[t];
            }
            const double ar = double(a.x), ai = double(a.y);
            re += sr * ar - si * ai;
            im += sr * ai + si * ar;
        }
        out[j] = mk<V>(re, im);
    }
}

// Per-instance partial sums of conj(a) b: grid = (blocks per instance, instances).
template <typename V>
__global__ void __launch_bounds__(kThreads)
k_inner_partial(const V* __restrict__ a, const V* __restrict__ b, uint64_t inst_len, double* __restrict__ part) {
    const uint64_t inst = blockIdx.y;
    const V* ai = a + inst * inst_len;
    const V* bi = b + inst * inst_len;
    double re = 0.0, im = 0.0;
    for (uint64_t j = uint64_t(blockIdx.x) * kThreads + threadIdx.x; j < inst_len; j += uint64_t(gridDim.x) * kThreads) {
        const V u = ai[j], v = bi[j];
        re += double(u.x) * double(v.x) + double(u.y) * double(v.y);
        im += double(u.x) * double(v.y) - double(u.y) * double(v.x);
    }
    __shared__ double sr[kThreads / 32], si[kThreads / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        re += __shfl_xor_sync(0xffffffffu, re, o);
        im += __shfl_xor_sync(0xffffffffu, im, o);
    }
    if ((threadIdx.x & 31) == 0) {
        sr[threadIdx.x >> 5] = re;
        si[threadIdx.x >> 5] = im;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0.0, i = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) { r += sr[w]; i += si[w]; }
        const uint64_t at = 2 * (inst * gridDim.x + blockIdx.x);
        part[at] = r;
        part[at + 1] = i;
    }
}

// Sums of `nseg` segments of `seglen` complex FP64 values, one warp per
// segment: lane l adds elements l, l + 32, ... (coalesced), then a fixed
// shuffle tree (the same order on every run).
__global__ void __launch_bounds__(kThreads) k_segsum(const double* __restrict__ in, int64_t nseg, int64_t seglen,
                                                     double* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = int64_t(gridDim.x) * (kThreads / 32);
    for (int64_t s = int64_t(blockIdx.x) * (kThreads / 32) + (threadIdx.x >> 5); s < nseg; s += warps) {
        const double2* p = reinterpret_cast<const double2*>(in) + s * seglen;
        double r = 0.0, i = 0.0;
        for (int64_t t = lane; t < seglen; t += 32) {
            const double2 v = p[t];
            r += v.x;
            i += v.y;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            r += __shfl_xor_sync(0xffffffffu, r, o);
            i += __shfl_xor_sync(0xffffffffu, i, o);
        }
        if (lane == 0) {
            out[2 * s] = r;
            out[2 * s + 1] = i;
        }
    }
}

}  // namespace
}  // namespace qs

using namespace qs;

extern "C" int qs_apply_pauli_sum(const void* psi, void* out, int n, int dtype, const uint64_t* xmask,
                                  const uint64_t* zmask, const double* coeff, int nterms, void* stream) {
    QS_REQUIRE(psi != nullptr && out != nullptr && psi != out, "psi and out must be distinct non-null vectors");
    QS_REQUIRE(n >= 1 && n <= 40, "qubit count %d outside [1, 40]", n);
    QS_REQUIRE(valid_dtype(dtype), "bad dtype %d", dtype);
    QS_REQUIRE(nterms >= 1 && nterms <= kMaxTerms, "term count %d outside [1, %d]", nterms, kMaxTerms);
    QS_REQUIRE(xmask != nullptr && zmask != nullptr && coeff != nullptr, "null term arrays");
    static thread_local PauliTerms p;
    p.n = nterms;
    // terms in the order of their X masks (stable), grouped by mask
    int order[kMaxTerms];
    for (int t = 0; t < nterms; ++t) {
        QS_REQUIRE((xmask[t] >> n) == 0 && (zmask[t] >> n) == 0, "term %d acts on bits >= n", t);
        order[t] = t;
    }
    std::stable_sort(order, order + nterms, [&](int a, int b) { return xmask[a] < xmask[b]; });
    p.ngroups = 0;
    for (int i = 0; i < nterms; ++i) {
        const int t = order[i];
        if (i == 0 || xmask[t] != xmask[order[i - 1]]) {
            p.x[p.ngroups] = xmask[t];
            p.gbeg[p.ngroups++] = i;
        }
        p.z[i] = zmask[t];
        // fold i^popc(x & z) (Y = i X Z) into the coefficient
        double re = coeff[2 * t], im = coeff[2 * t + 1];
        for (int k = 0; k < (__builtin_popcountll(xmask[t] & zmask[t]) & 3); ++k) {
            double r2 = -im, i2 = re;
            re = r2;
            im = i2;
        }
        p.cre[i] = re;
        p.cim[i] = im;
    }
    p.gbeg[p.ngroups] = nterms;
    const uint64_t N = uint64_t(1) << n;
    unsigned grid = grid_for(N, kThreads, 8);
    if (dtype == QS_C128) k_pauli_sum<double2><<<grid, kThreads, 0, as_stream(stream)>>>((const double2*)psi, (double2*)out, N, p);
    else                  k_pauli_sum<float2><<<grid, kThreads, 0, as_stream(stream)>>>((const float2*)psi, (float2*)out, N, p);
    QS_CHECK_LAUNCH("qs_apply_pauli_sum");
    return QS_OK;
}

extern "C" int qs_inner_batched(const void* a, const void* b, int n, int dtype, int inst_bits, double* out_dev,
                                void* ws, size_t ws_bytes, void* stream) {
    QS_REQUIRE(a != nullptr && b != nullptr && out_dev != nullptr, "null argument");
    QS_REQUIRE(n >= 1 && n <= 40 && inst_bits >= 1 && inst_bits <= n, "bad sizes n=%d inst_bits=%d", n, inst_bits);
    QS_REQUIRE(valid_dtype(dtype), "bad dtype %d", dtype);
    const uint64_t ninst = uint64_t(1) << (n - inst_bits);
    const uint64_t len = uint64_t(1) << inst_bits;
    // blocks per instance: up to one per 2048 amplitudes, enough in total to
    // fill the GPU (8 CTAs per SM), at most kMaxInnerBlocks
    uint64_t per = (len + kThreads * 8 - 1) / (kThreads * 8);
    uint64_t fill = (uint64_t(sm_count()) * 8 + ninst - 1) / ninst;
    if (per > fill) per = fill;
    if (per > kMaxInnerBlocks) per = kMaxInnerBlocks;
    const uint64_t fits = ws == nullptr ? 0 : uint64_t(ws_bytes / (sizeof(double) * 2 * ninst));
    if (per > fits) per = fits;  // as many partials as the workspace holds
    if (per < 1) {
        set_error("qs_inner_batched needs at least %zu bytes of workspace", sizeof(double) * 2 * size_t(ninst));
        return QS_EWORKSPACE;
    }
    QS_REQUIRE(ninst <= 65535, "at most 65535 instances per call");
    const dim3 grid = dim3(unsigned(per), unsigned(ninst), 1u);
    double* part = static_cast<double*>(ws);
    if (dtype == QS_C128) k_inner_partial<double2><<<grid, kThreads, 0, as_stream(stream)>>>((const double2*)a, (const double2*)b, len, part);
    else                  k_inner_partial<float2><<<grid, kThreads, 0, as_stream(stream)>>>((const float2*)a, (const float2*)b, len, part);
    k_segsum<<<grid_for(ninst, kThreads / 32, 8), kThreads, 0, as_stream(stream)>>>(part, int64_t(ninst), int64_t(per),
                                                                                    out_dev);
    QS_CHECK_LAUNCH("qs_inner_batched");
    return QS_OK;
}

extern "C" int qs_segment_sum(const double* in_dev, int64_t nseg, int64_t seglen, double* out_dev, void* stream) {
    QS_REQUIRE(in_dev != nullptr && out_dev != nullptr && nseg >= 1 && seglen >= 1, "bad arguments");
    k_segsum<<<grid_for(uint64_t(nseg), kThreads / 32, 8), kThreads, 0, as_stream(stream)>>>(in_dev, nseg, seglen,
                                                                                              out_dev);
    QS_CHECK_LAUNCH("qs_segment_sum");
    return QS_OK;
}
