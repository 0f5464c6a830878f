// Measurement, reset, FP64 reductions and sampling.
//
// Sampling replaces the reference's shots x qubits loop (one reduction, one
// device->host read and one collapse kernel per qubit per shot,
// statevector_simulator.py:595-626) with a sum tree built once: FP64 sums of
// 2^B-amplitude blocks at the leaves, a binary heap above them.  Each shot is
// one warp that walks the heap from the root (qubit 0 = the vector's top bit
// first) and finishes inside its leaf block from the block's own amplitudes.
#include <mutex>

#include "common.cuh"

namespace qs {
namespace {

constexpr int kThreads = 256;
constexpr int kReduceCtas = 1024;     // partial-sum slots in the reduce workspace
constexpr int kBlockBits = 10;        // leaf block = 2^10 probabilities

// p_i of a probability source
template <typename V, int SRC>
__device__ __forceinline__ double prob_at(const V* __restrict__ s, uint64_t i, uint64_t dstride) {
    if (SRC == QS_SRC_SV) return cnorm2(s[i]);
    return double(s[i * dstride].x);
}

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

// Block-level sum; result valid in thread 0.
__device__ __forceinline__ double block_sum(double x) {
    __shared__ double part[32];
    x = warp_sum(x);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) part[w] = x;
    __syncthreads();
    double r = 0.0;
    if (w == 0) {
        r = (l < int(blockDim.x >> 5)) ? part[l] : 0.0;
        r = warp_sum(r);
    }
    __syncthreads();
    return r;
}

// Sum of p over the compact space with `bit` removed (bit < 0: everything).
template <typename V, int SRC>
__global__ void __launch_bounds__(kThreads)
k_partial(const V* __restrict__ s, uint64_t items, int bit, uint64_t dstride, double* __restrict__ part) {
    double acc = 0.0;
    const uint64_t stride = uint64_t(gridDim.x) * kThreads;
    for (uint64_t j = uint64_t(blockIdx.x) * kThreads + threadIdx.x; j < items; j += stride) {
        uint64_t i = bit >= 0 ? insert0(j, bit) : j;
        acc += prob_at<V, SRC>(s, i, dstride);
    }
    acc = block_sum(acc);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

__global__ void __launch_bounds__(kThreads) k_finish(const double* __restrict__ part, int nparts, double* out) {
    double acc = 0.0;
    for (int i = threadIdx.x; i < nparts; i += kThreads) acc += part[i];
    acc = block_sum(acc);
    if (threadIdx.x == 0) *out = acc;
}

template <typename V>
__global__ void __launch_bounds__(kThreads) k_collapse(V* __restrict__ v, uint64_t N, int bit, int outcome, double scale) {
    const uint64_t stride = uint64_t(gridDim.x) * kThreads;
    for (uint64_t i = uint64_t(blockIdx.x) * kThreads + threadIdx.x; i < N; i += stride) {
        if (int((i >> bit) & 1) == outcome) {
            V a = v[i];
            a.x *= scale; a.y *= scale;
            v[i] = a;
        } else {
            v[i] = mk<V>(0.0, 0.0);
        }
    }
}

// Reference reset rule: alpha = sqrt(P0); alpha < 1e-6 -> v0 <- v1, else
// v0 <- v0 / alpha; v1 <- 0 either way.
template <typename V>
__global__ void __launch_bounds__(kThreads) k_reset(V* __restrict__ v, uint64_t items, int bit, double alpha, bool move) {
    const uint64_t stride = uint64_t(gridDim.x) * kThreads;
    const uint64_t off = uint64_t(1) << bit;
    for (uint64_t j = uint64_t(blockIdx.x) * kThreads + threadIdx.x; j < items; j += stride) {
        uint64_t i0 = insert0(j, bit);
        V a;
        if (move) {
            a = v[i0 + off];
        } else {
            a = v[i0];
            a.x /= alpha; a.y /= alpha;
        }
        v[i0] = a;
        v[i0 + off] = mk<V>(0.0, 0.0);
    }
}

// -------------------------------------------------------------- sum tree
// ws layout: double tree[2 * nleaf]; heap with root at 1, leaves at
// [nleaf, 2*nleaf), leaf b = sum of p over block b (2^bb probabilities).
template <typename V, int SRC>
__global__ void __launch_bounds__(kThreads)
k_leaves(const V* __restrict__ s, uint64_t nleaf, int bb, uint64_t dstride, double* __restrict__ tree) {
    const int lane = threadIdx.x & 31;
    const uint64_t warps = uint64_t(gridDim.x) * (kThreads / 32);
    const uint64_t bsz = uint64_t(1) << bb;
    for (uint64_t b = uint64_t(blockIdx.x) * (kThreads / 32) + (threadIdx.x >> 5); b < nleaf; b += warps) {
        double acc = 0.0;
        for (uint64_t e = lane; e < bsz; e += 32) acc += prob_at<V, SRC>(s, b * bsz + e, dstride);
        acc = warp_sum(acc);
        if (lane == 0) tree[nleaf + b] = acc;
    }
}

__global__ void __launch_bounds__(kThreads) k_level(double* __restrict__ tree, uint64_t lo, uint64_t cnt) {
    const uint64_t stride = uint64_t(gridDim.x) * kThreads;
    for (uint64_t j = uint64_t(blockIdx.x) * kThreads + threadIdx.x; j < cnt; j += stride) {
        uint64_t i = lo + j;
        tree[i] = tree[2 * i] + tree[2 * i + 1];
    }
}

// CDF descent step: go right when u lies beyond the left half's mass, but
// never into a half of zero mass.  The in-block half sums are added in a
// different order from the leaf sums above them, so u can exceed a block's
// recomputed total by a rounding error; the guard then ends the descent on
// the block's last element of nonzero probability instead of one with p = 0.
__device__ __forceinline__ bool cdf_right(double uc, double acc, double sl, double sr) {
    if (!(sr > 0.0)) return false;
    if (!(sl > 0.0)) return true;
    return !(uc <= acc + sl);
}

// One warp per shot.  Within the leaf block lane l owns elements
// [l*E, (l+1)*E), E = 2^bb / 32 (or one element per lane for tiny blocks).
template <typename V, int SRC, int MODE>
__global__ void __launch_bounds__(kThreads)
k_sample(const V* __restrict__ s, int n, uint64_t nleaf, int bb, uint64_t dstride, const double* __restrict__ tree,
         const double* __restrict__ u, int64_t shots, int64_t* __restrict__ out) {
    constexpr int EMAX = (1 << kBlockBits) / 32;
    const int lane = threadIdx.x & 31;
    const int64_t warps = int64_t(gridDim.x) * (kThreads / 32);
    const int top = n - bb;  // heap levels above the leaves
    const int bsz = 1 << bb;
    const int E = bsz >= 32 ? bsz / 32 : 1;
    for (int64_t shot = int64_t(blockIdx.x) * (kThreads / 32) + (threadIdx.x >> 5); shot < shots; shot += warps) {
        const double* us = MODE == QS_SAMPLE_SEQ ? u + shot * n : u + shot;
        // CDF mode compares against unnormalised FP64 partial sums, so the
        // uniform is scaled by the total mass (the root): a state whose norm
        // has drifted below 1 (complex64, a density matrix's trace) then
        // never runs off the end of the distribution
        double uc = MODE == QS_SAMPLE_SEQ ? us[0] : us[0] * tree[1];
        double acc = 0.0;  // CDF mode: mass strictly left of the current node
        uint64_t node = 1;
        for (int lvl = 0; lvl < top; ++lvl) {
            double sl = tree[2 * node], sr = tree[2 * node + 1];
            bool right;
            if (MODE == QS_SAMPLE_SEQ) {
                double tot = sl + sr;
                right = uc > sl / tot;
                uc = us[lvl + 1 < n ? lvl + 1 : n - 1];
            } else {
                right = cdf_right(uc, acc, sl, sr);
                if (right) acc += sl;
            }
            node = 2 * node + (right ? 1 : 0);
        }
        const uint64_t blk = node - nleaf;
        const uint64_t base = blk * uint64_t(bsz);
        double p[EMAX];
#pragma unroll
        for (int e = 0; e < EMAX; ++e) {
            int idx = lane * E + e;
            p[e] = (e < E && idx < bsz) ? prob_at<V, SRC>(s, base + idx, dstride) : 0.0;
        }
        // descend inside the block over ranges [lo, lo + size)
        int lo = 0;
        int lvl = top;
        for (int size = bsz; size > 1; size >>= 1, ++lvl) {
            const int half = size >> 1;
            double sl, sr;
            if (half >= E) {
                // whole lanes: lanes [lo/E, (lo+half)/E) left, [(lo+half)/E, (lo+size)/E) right
                double mine = 0.0;
#pragma unroll
                for (int e = 0; e < EMAX; ++e) mine += (e < E) ? p[e] : 0.0;
                const int l0 = lo / E, lm = (lo + half) / E, l1 = (lo + size) / E;
                sl = warp_sum((lane >= l0 && lane < lm) ? mine : 0.0);
                sr = warp_sum((lane >= lm && lane < l1) ? mine : 0.0);
            } else {
                // inside one lane
                const int owner = lo / E, off = lo % E;
                double a = 0.0, b = 0.0;
#pragma unroll
                for (int e = 0; e < EMAX; ++e) {
                    if (e >= off && e < off + half) a += p[e];
                    if (e >= off + half && e < off + size) b += p[e];
                }
                sl = __shfl_sync(0xffffffffu, a, owner);
                sr = __shfl_sync(0xffffffffu, b, owner);
            }
            bool right;
            if (MODE == QS_SAMPLE_SEQ) {
                right = uc > sl / (sl + sr);
                uc = us[lvl + 1 < n ? lvl + 1 : n - 1];
            } else {
                right = cdf_right(uc, acc, sl, sr);
                if (right) acc += sl;
            }
            if (right) lo += half;
        }
        if (lane == 0) out[shot] = int64_t(base + lo);
    }
}

__global__ void k_hist(const int64_t* __restrict__ idx, int64_t shots, unsigned long long* counts, int64_t ncounts) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t s = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; s < shots; s += stride) {
        int64_t i = idx[s];
        if (i >= 0 && i < ncounts) atomicAdd(&counts[i], 1ull);
    }
}

int check_src(const void* src, int n, int dtype, int src_kind) {
    QS_REQUIRE(src != nullptr, "null source");
    QS_REQUIRE(valid_dtype(dtype), "bad dtype %d", dtype);
    QS_REQUIRE(src_kind == QS_SRC_SV || src_kind == QS_SRC_DM, "bad source kind %d", src_kind);
    QS_REQUIRE(n >= 1 && n <= (src_kind == QS_SRC_SV ? 40 : 20), "qubit count %d out of range", n);
    return QS_OK;
}

template <typename V>
int reduce_t(const void* src, int n, int src_kind, int bit, void* ws, double* out, cudaStream_t st) {
    const V* s = static_cast<const V*>(src);
    uint64_t items = uint64_t(1) << (bit >= 0 ? n - 1 : n);
    uint64_t dstride = (uint64_t(1) << n) + 1;
    unsigned grid = grid_for(items, kThreads * 4, 4);
    if (grid > kReduceCtas) grid = kReduceCtas;
    double* part = static_cast<double*>(ws);
    if (src_kind == QS_SRC_SV) k_partial<V, QS_SRC_SV><<<grid, kThreads, 0, st>>>(s, items, bit, dstride, part);
    else                       k_partial<V, QS_SRC_DM><<<grid, kThreads, 0, st>>>(s, items, bit, dstride, part);
    k_finish<<<1, kThreads, 0, st>>>(part, int(grid), out);
    QS_CHECK_LAUNCH("reduce");
    return QS_OK;
}

int tree_shape(int n, uint64_t* nleaf, int* bb) {
    *bb = n < kBlockBits ? n : kBlockBits;
    *nleaf = uint64_t(1) << (n - *bb);
    return QS_OK;
}

template <typename V>
int prepare_t(const void* src, int n, int src_kind, double* tree, cudaStream_t st) {
    const V* s = static_cast<const V*>(src);
    uint64_t nleaf; int bb;
    tree_shape(n, &nleaf, &bb);
    uint64_t dstride = (uint64_t(1) << n) + 1;
    unsigned grid = grid_for(nleaf, kThreads / 32, 8, 4);
    if (src_kind == QS_SRC_SV) k_leaves<V, QS_SRC_SV><<<grid, kThreads, 0, st>>>(s, nleaf, bb, dstride, tree);
    else                       k_leaves<V, QS_SRC_DM><<<grid, kThreads, 0, st>>>(s, nleaf, bb, dstride, tree);
    for (uint64_t lo = nleaf / 2; lo >= 1; lo /= 2)
        k_level<<<grid_for(lo, kThreads, 8), kThreads, 0, st>>>(tree, lo, lo);
    QS_CHECK_LAUNCH("qs_sample_prepare");
    return QS_OK;
}

template <typename V>
int sample_t(const void* src, int n, int src_kind, const double* tree, const double* u, int64_t shots, int mode,
             int64_t* out, cudaStream_t st) {
    const V* s = static_cast<const V*>(src);
    uint64_t nleaf; int bb;
    tree_shape(n, &nleaf, &bb);
    uint64_t dstride = (uint64_t(1) << n) + 1;
    unsigned grid = grid_for(uint64_t(shots), kThreads / 32, 8, 4);
#define QS_SAMPLE_LAUNCH(SRC, MODE) \
    k_sample<V, SRC, MODE><<<grid, kThreads, 0, st>>>(s, n, nleaf, bb, dstride, tree, u, shots, out)
    if (src_kind == QS_SRC_SV) {
        if (mode == QS_SAMPLE_SEQ) QS_SAMPLE_LAUNCH(QS_SRC_SV, QS_SAMPLE_SEQ);
        else                       QS_SAMPLE_LAUNCH(QS_SRC_SV, QS_SAMPLE_CDF);
    } else {
        if (mode == QS_SAMPLE_SEQ) QS_SAMPLE_LAUNCH(QS_SRC_DM, QS_SAMPLE_SEQ);
        else                       QS_SAMPLE_LAUNCH(QS_SRC_DM, QS_SAMPLE_CDF);
    }
#undef QS_SAMPLE_LAUNCH
    QS_CHECK_LAUNCH("qs_sample");
    return QS_OK;
}

}  // namespace
}  // namespace qs

using namespace qs;

extern "C" size_t qs_reduce_ws_bytes(int) { return sizeof(double) * kReduceCtas; }

extern "C" int qs_prob0(const void* src, int n, int dtype, int src_kind, int bit, void* ws, size_t ws_bytes,
                        double* out_dev, void* stream) {
    int rc = check_src(src, n, dtype, src_kind);
    if (rc) return rc;
    QS_REQUIRE(bit >= 0 && bit < n, "bit %d outside [0, %d)", bit, n);
    QS_REQUIRE(out_dev != nullptr, "null output");
    if (ws == nullptr || ws_bytes < qs_reduce_ws_bytes(n)) {
        set_error("reduce workspace needs %zu bytes", qs_reduce_ws_bytes(n));
        return QS_EWORKSPACE;
    }
    if (dtype == QS_C128) return reduce_t<double2>(src, n, src_kind, bit, ws, out_dev, as_stream(stream));
    return reduce_t<float2>(src, n, src_kind, bit, ws, out_dev, as_stream(stream));
}

extern "C" int qs_norm2(const void* src, int n, int dtype, int src_kind, void* ws, size_t ws_bytes, double* out_dev,
                        void* stream) {
    int rc = check_src(src, n, dtype, src_kind);
    if (rc) return rc;
    QS_REQUIRE(out_dev != nullptr, "null output");
    if (ws == nullptr || ws_bytes < qs_reduce_ws_bytes(n)) {
        set_error("reduce workspace needs %zu bytes", qs_reduce_ws_bytes(n));
        return QS_EWORKSPACE;
    }
    if (dtype == QS_C128) return reduce_t<double2>(src, n, src_kind, -1, ws, out_dev, as_stream(stream));
    return reduce_t<float2>(src, n, src_kind, -1, ws, out_dev, as_stream(stream));
}

extern "C" int qs_collapse(void* vec, int n, int dtype, int bit, int outcome, double scale, void* stream) {
    int rc = check_src(vec, n, dtype, QS_SRC_SV);
    if (rc) return rc;
    QS_REQUIRE(bit >= 0 && bit < n, "bit %d outside [0, %d)", bit, n);
    QS_REQUIRE(outcome == 0 || outcome == 1, "outcome must be 0 or 1");
    uint64_t N = uint64_t(1) << n;
    unsigned grid = grid_for(N, kThreads * 4, 8);
    if (dtype == QS_C128) k_collapse<double2><<<grid, kThreads, 0, as_stream(stream)>>>((double2*)vec, N, bit, outcome, scale);
    else                  k_collapse<float2><<<grid, kThreads, 0, as_stream(stream)>>>((float2*)vec, N, bit, outcome, scale);
    QS_CHECK_LAUNCH("qs_collapse");
    return QS_OK;
}

extern "C" int qs_reset(void* vec, int n, int dtype, int bit, double p0, void* stream) {
    int rc = check_src(vec, n, dtype, QS_SRC_SV);
    if (rc) return rc;
    QS_REQUIRE(bit >= 0 && bit < n, "bit %d outside [0, %d)", bit, n);
    double alpha = sqrt(p0 > 0 ? p0 : 0.0);
    bool move = alpha < 1e-6;
    uint64_t items = uint64_t(1) << (n - 1);
    unsigned grid = grid_for(items, kThreads * 4, 8);
    if (dtype == QS_C128) k_reset<double2><<<grid, kThreads, 0, as_stream(stream)>>>((double2*)vec, items, bit, alpha, move);
    else                  k_reset<float2><<<grid, kThreads, 0, as_stream(stream)>>>((float2*)vec, items, bit, alpha, move);
    QS_CHECK_LAUNCH("qs_reset");
    return QS_OK;
}

extern "C" size_t qs_sample_ws_bytes(int n) {
    uint64_t nleaf; int bb;
    tree_shape(n, &nleaf, &bb);
    return sizeof(double) * 2 * nleaf;
}

extern "C" int qs_sample_prepare(const void* src, int n, int dtype, int src_kind, void* ws, size_t ws_bytes,
                                 void* stream) {
    int rc = check_src(src, n, dtype, src_kind);
    if (rc) return rc;
    if (ws == nullptr || ws_bytes < qs_sample_ws_bytes(n)) {
        set_error("sample workspace needs %zu bytes", qs_sample_ws_bytes(n));
        return QS_EWORKSPACE;
    }
    if (dtype == QS_C128) return prepare_t<double2>(src, n, src_kind, (double*)ws, as_stream(stream));
    return prepare_t<float2>(src, n, src_kind, (double*)ws, as_stream(stream));
}

extern "C" int qs_sample(const void* src, int n, int dtype, int src_kind, const void* ws, size_t ws_bytes,
                         const double* u_dev, int64_t shots, int mode, int64_t* out_idx_dev, void* stream) {
    int rc = check_src(src, n, dtype, src_kind);
    if (rc) return rc;
    QS_REQUIRE(mode == QS_SAMPLE_CDF || mode == QS_SAMPLE_SEQ, "bad sample mode %d", mode);
    QS_REQUIRE(shots >= 0, "negative shot count");
    QS_REQUIRE(u_dev != nullptr && out_idx_dev != nullptr, "null uniforms or output");
    if (ws == nullptr || ws_bytes < qs_sample_ws_bytes(n)) {
        set_error("sample workspace needs %zu bytes", qs_sample_ws_bytes(n));
        return QS_EWORKSPACE;
    }
    if (shots == 0) return QS_OK;
    if (dtype == QS_C128)
        return sample_t<double2>(src, n, src_kind, (const double*)ws, u_dev, shots, mode, out_idx_dev, as_stream(stream));
    return sample_t<float2>(src, n, src_kind, (const double*)ws, u_dev, shots, mode, out_idx_dev, as_stream(stream));
}

extern "C" int qs_histogram(const int64_t* idx_dev, int64_t shots, int64_t* counts_dev, int64_t ncounts, void* stream) {
    QS_REQUIRE(shots >= 0 && ncounts >= 1, "bad sizes");
    QS_REQUIRE((shots == 0 || idx_dev != nullptr) && counts_dev != nullptr, "null pointer");
    if (shots == 0) return QS_OK;
    unsigned grid = grid_for(uint64_t(shots), 256, 4);
    k_hist<<<grid, 256, 0, as_stream(stream)>>>(idx_dev, shots, (unsigned long long*)counts_dev, ncounts);
    QS_CHECK_LAUNCH("qs_histogram");
    return QS_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free sampling.  The sum tree lives in a file-scope device array
// instead of a caller workspace, for callers that can only hand over the
// state, the uniforms and the output buffer (see include/qsim.h).
// ---------------------------------------------------------------------------
namespace {
constexpr int kNoAllocMaxQubits = QS_NOALLOC_SAMPLE_MAX_QUBITS;
constexpr size_t kNoAllocTreeDoubles = size_t(2) << (kNoAllocMaxQubits - kBlockBits);  // 1 MiB
}  // namespace

static __device__ __align__(256) double g_noalloc_tree[kNoAllocTreeDoubles];

namespace {
// Device address of g_noalloc_tree on the current device (the array's
// host-side name is not a device address).  It is looked up with that device
// current on every call made outside stream capture, so a context rebuilt
// after cudaDeviceReset gets its new address; inside a capture the address
// recorded by the last call outside one is used.
int noalloc_tree_ptr(cudaStream_t st, double** out) {
    static std::mutex mu;
    static double* addr[64] = {nullptr};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        set_error("qs_sample_noalloc: cudaGetDevice: %s", cudaGetErrorString(e));
        return QS_ECUDA;
    }
    QS_REQUIRE(dev >= 0 && dev < 64, "qs_sample_noalloc: device %d outside [0, 64)", dev);
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    e = cudaStreamIsCapturing(st, &cs);
    if (e != cudaSuccess) {
        set_error("qs_sample_noalloc: cudaStreamIsCapturing: %s", cudaGetErrorString(e));
        return QS_ECUDA;
    }
    std::lock_guard<std::mutex> lock(mu);
    if (addr[dev] == nullptr || cs == cudaStreamCaptureStatusNone) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_tree);
        if (e != cudaSuccess || p == nullptr) {
            set_error("qs_sample_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
            return QS_ECUDA;
        }
        addr[dev] = static_cast<double*>(p);
    }
    *out = addr[dev];
    return QS_OK;
}
}  // namespace

extern "C" int qs_sample_noalloc(const void* src, int n, int dtype, int src_kind, const double* u_dev,
                                 int64_t shots, int mode, int64_t* out_idx_dev, void* stream) {
    int rc = check_src(src, n, dtype, src_kind);
    if (rc) return rc;
    if (n > kNoAllocMaxQubits) {
        set_error("qs_sample_noalloc: %d qubits exceed its fixed %d-qubit limit (a %zu-byte static sum tree); "
                  "use qs_sample_prepare/qs_sample with a workspace",
                  n, kNoAllocMaxQubits, sizeof(double) * kNoAllocTreeDoubles);
        return QS_EINVAL;
    }
    QS_REQUIRE(mode == QS_SAMPLE_CDF || mode == QS_SAMPLE_SEQ, "bad sample mode %d", mode);
    QS_REQUIRE(shots >= 0, "negative shot count");
    QS_REQUIRE(u_dev != nullptr && out_idx_dev != nullptr, "null uniforms or output");
    if (shots == 0) return QS_OK;
    cudaStream_t st = as_stream(stream);
    double* tree = nullptr;
    rc = noalloc_tree_ptr(st, &tree);
    if (rc) return rc;
    // every node the descent reads is written by the prepare step, so the
    // tree needs no clearing between calls
    if (dtype == QS_C128) {
        rc = prepare_t<double2>(src, n, src_kind, tree, st);
        return rc ? rc : sample_t<double2>(src, n, src_kind, tree, u_dev, shots, mode, out_idx_dev, st);
    }
    rc = prepare_t<float2>(src, n, src_kind, tree, st);
    return rc ? rc : sample_t<float2>(src, n, src_kind, tree, u_dev, shots, mode, out_idx_dev, st);
}
