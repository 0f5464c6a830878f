// Fused passes: one launch streams the state through shared-memory tiles once
// and applies every op of the pass to each tile.
//
// A tile holds 2^k amplitudes: vector bits 0..nlow-1 (contiguous, so each
// warp reads 2^nlow consecutive amplitudes) plus k-nlow chosen higher bits.
// Ops whose non-diagonal targets lie in the tile are applied in shared
// memory; diagonal factors and controls on bits outside the tile are
// resolved per tile from the tile's base index, so they fuse into any pass.
// The reference has no fusion: one kernel and one full HBM pass per gate
// (statevector_simulator.py:155-164, gate_function.py:31-1031).
#include "common.cuh"

namespace qs {
namespace {

constexpr int kFT = 256;  // threads per CTA

struct PassArgs {
    int n, k, nlow, nops;
    int hi[QS_MAX_TILE_BITS];
    qs_op ops[QS_MAX_PASS_OPS];
};

__device__ __forceinline__ uint32_t ins0(uint32_t x, int b) {
    return ((x >> b) << (b + 1)) | (x & ((1u << b) - 1u));
}

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

// Dense 2^M x 2^M on tile-local targets op.tgt[0..M-1].
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
    if (M <= 2) {
        V mr[D * D];
#pragma unroll
        for (int i = 0; i < D * D; ++i) mr[i] = mat[i];
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
                V acc = cmul(mr[r * D], x[0]);
#pragma unroll
                for (int c = 1; c < D; ++c) acc = cfma(mr[r * D + c], x[c], acc);
                tile[i0 | spread[r]] = acc;
            }
        }
    } else {
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
}

// Diagonal on op.m bits; bits outside the tile contribute a per-tile constant.
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
    if (m <= 2) {
        V d[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) d[i] = (i < (1 << m)) ? mat[i] : mk<V>(1.0, 0.0);
        for (uint32_t e = threadIdx.x; e < T; e += kFT) {
            if ((e & lctrl) != lctrl) continue;
            uint32_t sidx = ext;
#pragma unroll
            for (int j = 0; j < 2; ++j)
                if (j < m && lpos[j] >= 0) sidx |= ((e >> lpos[j]) & 1u) << (m - 1 - j);
            tile[e] = cmul(tile[e], d[sidx]);
        }
    } else {
        for (uint32_t e = threadIdx.x; e < T; e += kFT) {
            if ((e & lctrl) != lctrl) continue;
            uint32_t sidx = ext;
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (j < m && lpos[j] >= 0) sidx |= ((e >> lpos[j]) & 1u) << (m - 1 - j);
            tile[e] = cmul(tile[e], __ldg(&mat[sidx]));
        }
    }
}

template <typename V>
__global__ void __launch_bounds__(kFT) k_fused(V* __restrict__ vec, const __grid_constant__ PassArgs p,
                                                const V* __restrict__ mats) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int K = p.k, L = p.nlow, H = K - L;
    const uint32_t T = 1u << K;
    V* tile = reinterpret_cast<V*>(smem_raw);
    uint64_t* hoff = reinterpret_cast<uint64_t*>(smem_raw + sizeof(V) * T);
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
        for (uint32_t e = threadIdx.x; e < T; e += kFT)
            tile[e] = vec[base | hoff[e >> L] | (e & lmask)];
        __syncthreads();
        for (int o = 0; o < p.nops; ++o) {
            const qs_op& op = p.ops[o];
            if ((base & op.gctrl) != op.gctrl) continue;  // CTA-uniform
            const V* mat = mats + op.mat;
            if (op.kind == QS_OP_MAT) {
                switch (op.m) {
                    case 1: tile_mat<V, 1>(tile, K, op, mat); break;
                    case 2: tile_mat<V, 2>(tile, K, op, mat); break;
                    case 3: tile_mat<V, 3>(tile, K, op, mat); break;
                    default: tile_mat<V, 4>(tile, K, op, mat); break;
                }
            } else {
                tile_diag<V>(tile, K, base, op, mat);
            }
            __syncthreads();
        }
        for (uint32_t e = threadIdx.x; e < T; e += kFT)
            vec[base | hoff[e >> L] | (e & lmask)] = tile[e];
        __syncthreads();
    }
}

int validate_pass(const qs_pass& ps, int n, const qs_op* ops, int64_t nops_total, int64_t mats_count) {
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
    // global bit -> local position
    int local[64];
    for (int b = 0; b < 64; ++b) local[b] = -1;
    for (int b = 0; b < ps.nlow; ++b) local[b] = b;
    for (int t = 0; t < ps.k - ps.nlow; ++t) local[ps.hi[t]] = ps.nlow + t;
    for (int i = 0; i < ps.op_count; ++i) {
        const qs_op& op = ops[ps.op_begin + i];
        QS_REQUIRE(op.kind == QS_OP_MAT || op.kind == QS_OP_DIAG, "op %d: bad kind %d", i, op.kind);
        QS_REQUIRE(op.m >= 1 && op.m <= 4, "op %d: m=%d outside [1, 4]", i, op.m);
        QS_REQUIRE((op.gctrl >> n) == 0 && (op.gctrl & tilemask) == 0, "op %d: global controls must lie outside the tile", i);
        QS_REQUIRE((op.lctrl >> ps.k) == 0, "op %d: local controls outside the tile", i);
        uint32_t tl = 0;
        for (int j = 0; j < op.m; ++j) {
            QS_REQUIRE(op.gbit[j] >= 0 && op.gbit[j] < n, "op %d: target bit outside [0, n)", i);
            QS_REQUIRE(op.tgt[j] == local[op.gbit[j]], "op %d: tile position of target %d inconsistent", i, j);
            if (op.kind == QS_OP_MAT) QS_REQUIRE(op.tgt[j] >= 0, "op %d: dense target outside the tile", i);
            if (op.tgt[j] >= 0) {
                QS_REQUIRE(!((tl >> op.tgt[j]) & 1), "op %d: duplicate target", i);
                tl |= 1u << op.tgt[j];
            }
        }
        QS_REQUIRE((tl & op.lctrl) == 0, "op %d: control overlaps a target", i);
        int64_t len = op.kind == QS_OP_MAT ? (int64_t(1) << (2 * op.m)) : (int64_t(1) << op.m);
        QS_REQUIRE(op.mat >= 0 && op.mat + len <= mats_count, "op %d: matrix outside the table", i);
    }
    return QS_OK;
}

template <typename V>
int launch_pass(V* vec, int n, const qs_pass& ps, const qs_op* ops, const V* mats, cudaStream_t st) {
    static thread_local PassArgs args;  // ~10 KB, keep off the stack
    args.n = n; args.k = ps.k; args.nlow = ps.nlow; args.nops = ps.op_count;
    for (int t = 0; t < QS_MAX_TILE_BITS; ++t) args.hi[t] = t < ps.k - ps.nlow ? ps.hi[t] : 0;
    for (int i = 0; i < ps.op_count; ++i) args.ops[i] = ops[ps.op_begin + i];
    size_t smem = sizeof(V) * (size_t(1) << ps.k) + sizeof(uint64_t) * (size_t(1) << (ps.k - ps.nlow));
    static int configured[2] = {0, 0};
    int slot = sizeof(V) == 16 ? 1 : 0;
    if (!configured[slot]) {
        cudaFuncSetAttribute(k_fused<V>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        configured[slot] = 1;
    }
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_fused<V>, kFT, smem);
    if (occ < 1) occ = 1;
    uint64_t ntiles = uint64_t(1) << (n - ps.k);
    uint64_t cap = uint64_t(sm_count()) * occ;
    unsigned grid = unsigned(ntiles < cap ? ntiles : cap);
    k_fused<V><<<grid, kFT, smem, st>>>(vec, args, mats);
    QS_CHECK_LAUNCH("qs_apply_fused");
    return QS_OK;
}

}  // namespace
}  // namespace qs

using namespace qs;

extern "C" int qs_apply_fused(void* vec, int n, int dtype, const qs_pass* passes, int npasses, const qs_op* ops,
                              int64_t nops_total, const void* mats_dev, int64_t mats_count, void* stream) {
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
        QS_REQUIRE(smem <= 200 * 1024, "pass %d: tile of 2^%d needs %zu bytes of shared memory", i, passes[i].k, smem);
    }
    for (int i = 0; i < npasses; ++i) {
        if (passes[i].op_count == 0) continue;
        int rc = dtype == QS_C128
                     ? launch_pass<double2>((double2*)vec, n, passes[i], ops, (const double2*)mats_dev, as_stream(stream))
                     : launch_pass<float2>((float2*)vec, n, passes[i], ops, (const float2*)mats_dev, as_stream(stream));
        if (rc) return rc;
    }
    return QS_OK;
}
