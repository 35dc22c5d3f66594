// Particle reordering by cell, so that the threads of a warp gather corner
// records from the same or neighbouring cells (L1/L2 sector reuse).
//
// Counting sort on a spatial bucket key: the map-0 cell of each particle is
// coarsened to 2x2x2-cell blocks, the block coordinates are Morton-interleaved
// and shifted down to at most 2^20 buckets (octree nodes, so neighbouring
// buckets stay spatially close); particles outside the map share one last
// bucket.  Histogram (atomics) -> exclusive scan -> scatter into a scratch
// copy -> copy back.  Order inside a bucket is arbitrary; `order` records
// slot -> row so outputs are written in the caller's row order, and every
// particle's arithmetic is independent of its slot.
#include <cstring>

#include "track_params.cuh"

namespace ppt {

constexpr int kMaxBucketBits = 20;
constexpr int kScanTile = 1024;

__device__ __forceinline__ uint32_t spread3(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

struct SortGeom {
    double lo[3];
    double inv_d[3];
    int n[3];          // nodes per axis
    int shift;
    uint32_t outside;  // bucket of particles outside the map
};

__device__ __forceinline__ uint32_t bucket_of_cells(const SortGeom& G, int c0, int c1, int c2) {
    if ((unsigned)c0 > (unsigned)(G.n[0] - 2) || (unsigned)c1 > (unsigned)(G.n[1] - 2) ||
        (unsigned)c2 > (unsigned)(G.n[2] - 2))
        return G.outside;
    uint32_t m = spread3((uint32_t)c0 >> 1) | (spread3((uint32_t)c1 >> 1) << 1) | (spread3((uint32_t)c2 >> 1) << 2);
    return m >> G.shift;
}

__global__ void sort_keys_f64(int64_t n, const double* __restrict__ st, SortGeom G, uint32_t* __restrict__ key,
                              uint32_t* __restrict__ count) {
    int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= n) return;
    int c[3];
    for (int a = 0; a < 3; ++a) {
        double u = (st[a * n + s] - G.lo[a]) * G.inv_d[a];
        c[a] = (u >= 0.0 && u < 2.0e9) ? (int)u : -1;
    }
    uint32_t b = bucket_of_cells(G, c[0], c[1], c[2]);
    key[s] = b;
    atomicAdd(count + b, 1u);
}

__global__ void sort_keys_mixed(int64_t n, const int32_t* __restrict__ ci, SortGeom G, uint32_t* __restrict__ key,
                                uint32_t* __restrict__ count) {
    int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= n) return;
    uint32_t b = bucket_of_cells(G, ci[s], ci[n + s], ci[2 * n + s]);
    key[s] = b;
    atomicAdd(count + b, 1u);
}

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* sh, uint32_t& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0u;
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        sh[lane] = w;   // inclusive warp totals
    }
    __syncthreads();
    total = sh[(blockDim.x >> 5) - 1];
    uint32_t before = warp > 0 ? sh[warp - 1] : 0u;
    uint32_t r = before + x - v;
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(kScanTile) scan_tiles(int64_t nb, const uint32_t* __restrict__ count,
                                                        uint32_t* __restrict__ offset, uint32_t* __restrict__ tile_sum) {
    __shared__ uint32_t sh[32];
    int64_t i = blockIdx.x * (int64_t)kScanTile + threadIdx.x;
    uint32_t v = i < nb ? count[i] : 0u;
    uint32_t total;
    uint32_t ex = block_exclusive_scan(v, sh, total);
    if (i < nb) offset[i] = ex;
    if (threadIdx.x == 0) tile_sum[blockIdx.x] = total;
}

// exclusive scan of up to kScanTile * 2 tile sums in one block
__global__ void __launch_bounds__(kScanTile) scan_top(int ntiles, uint32_t* __restrict__ tile_sum) {
    __shared__ uint32_t sh[32];
    uint32_t carry = 0;
    for (int base = 0; base < ntiles; base += kScanTile) {
        int i = base + threadIdx.x;
        uint32_t v = i < ntiles ? tile_sum[i] : 0u;
        uint32_t total;
        uint32_t ex = block_exclusive_scan(v, sh, total);
        if (i < ntiles) tile_sum[i] = ex + carry;
        carry += total;
    }
}

__global__ void scan_add(int64_t nb, uint32_t* __restrict__ offset, const uint32_t* __restrict__ tile_sum) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < nb) offset[i] += tile_sum[i / kScanTile];
}

// Scatter every word of a slot's state: ncols64 columns of 8-byte words, and
// na + nb columns of 4-byte words taken from two sources (mixed state: the
// int32 cells, then the float32 columns) into one destination block.
__global__ void sort_scatter(int64_t n, const uint32_t* __restrict__ key, uint32_t* __restrict__ offset,
                             int ncols64, const double* __restrict__ src64, double* __restrict__ dst64, int na,
                             const uint32_t* __restrict__ src_a, int nb, const uint32_t* __restrict__ src_b,
                             uint32_t* __restrict__ dst32, const int64_t* __restrict__ order,
                             int64_t* __restrict__ order_out, const double* __restrict__ phase,
                             double* __restrict__ phase_out) {
    int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int64_t d = atomicAdd(offset + key[s], 1u);
    for (int c = 0; c < ncols64; ++c) dst64[c * n + d] = src64[c * n + s];
    for (int c = 0; c < na; ++c) dst32[c * n + d] = src_a[c * n + s];
    for (int c = 0; c < nb; ++c) dst32[(na + c) * n + d] = src_b[c * n + s];
    order_out[d] = order[s];
    if (phase) phase_out[d] = phase[s];
}

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

struct SortLayout {
    size_t key, count, tiles, tmp64, tmp32, order, phase, total;
};

static SortLayout sort_layout(int64_t n) {
    SortLayout L;
    const size_t nb = ((size_t)1 << kMaxBucketBits) + 1;
    size_t o = 0;
    L.key = o;   o += align256((size_t)n * 4);
    L.count = o; o += align256(nb * 4);
    L.tiles = o; o += align256((nb / kScanTile + 2) * 4);
    L.tmp64 = o; o += align256((size_t)n * 6 * 8);     // float64 state, or mixed f32 part (9 words) below
    L.tmp32 = o; o += align256((size_t)n * 12 * 4);    // mixed: 3 int32 + 9 float32 columns
    L.order = o; o += align256((size_t)n * 8);
    L.phase = o; o += align256((size_t)n * 8);
    L.total = o;
    return L;
}

}  // namespace ppt

using namespace ppt;

extern "C" int64_t ppt_cell_sort_scratch_bytes(int64_t n) {
    if (n < 0) return -1;
    return (int64_t)sort_layout(n).total;
}

extern "C" int ppt_cell_sort(ppt_state* st, const ppt_fields* fields, int64_t* order, double* rf_phase,
                             void* scratch, void* stream) {
    int rc = check_state(st);
    if (rc) return rc;
    if (st->n == 0) return PPT_OK;
    if (st->n > 0x7fffffffLL) return fail(PPT_ERR_UNSUPPORTED, "cell sort handles at most 2^31-1 particles");
    if (!order || !scratch) return fail(PPT_ERR_ARG, "order and scratch must not be NULL");
    FieldsDev F;
    rc = build_fields(fields, &F);
    if (rc) return rc;
    if (F.n_maps == 0) return PPT_OK;   // no map: nothing to be local to
    const MapDev& m = F.maps[0];
    SortGeom G;
    int bits = 0;
    for (int a = 0; a < 3; ++a) {
        G.lo[a] = m.ax[a].lo;
        G.inv_d[a] = m.ax[a].inv_d;
        G.n[a] = m.ax[a].n;
        int coarse = (m.ax[a].n - 1 + 1) / 2;
        int b = 0;
        while ((1 << b) < coarse) ++b;
        bits = b > bits ? b : bits;
    }
    if (bits > 10) return fail(PPT_ERR_UNSUPPORTED, "cell sort handles maps up to 2048 nodes per axis");
    const int key_bits = 3 * bits;
    G.shift = key_bits > kMaxBucketBits ? key_bits - kMaxBucketBits : 0;
    G.outside = (uint32_t)((1u << (key_bits - G.shift)));
    const int64_t nb = (int64_t)G.outside + 1;
    if (st->precision == PPT_PREC_MIXED && !m.all_uniform)
        return fail(PPT_ERR_UNSUPPORTED, "mixed state needs a uniform map");
    if (st->precision == PPT_PREC_F64 && !m.all_uniform)
        return fail(PPT_ERR_UNSUPPORTED, "cell sort needs uniform axes (non-uniform maps: skip sorting)");

    const int64_t n = st->n;
    SortLayout L = sort_layout(n);
    char* base = static_cast<char*>(scratch);
    uint32_t* key = reinterpret_cast<uint32_t*>(base + L.key);
    uint32_t* count = reinterpret_cast<uint32_t*>(base + L.count);
    uint32_t* tiles = reinterpret_cast<uint32_t*>(base + L.tiles);
    double* tmp64 = reinterpret_cast<double*>(base + L.tmp64);
    uint32_t* tmp32 = reinterpret_cast<uint32_t*>(base + L.tmp32);
    int64_t* order_tmp = reinterpret_cast<int64_t*>(base + L.order);
    double* phase_tmp = reinterpret_cast<double*>(base + L.phase);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int block = 256;

    PPT_CUDA_TRY(cudaMemsetAsync(count, 0, (size_t)nb * 4, s));
    if (st->precision == PPT_PREC_F64)
        sort_keys_f64<<<grid_for(n, block), block, 0, s>>>(n, st->f64, G, key, count);
    else
        sort_keys_mixed<<<grid_for(n, block), block, 0, s>>>(n, st->i32, G, key, count);
    const int ntiles = (int)((nb + kScanTile - 1) / kScanTile);
    scan_tiles<<<ntiles, kScanTile, 0, s>>>(nb, count, count, tiles);
    scan_top<<<1, kScanTile, 0, s>>>(ntiles, tiles);
    scan_add<<<grid_for(nb, block), block, 0, s>>>(nb, count, tiles);
    if (st->precision == PPT_PREC_F64) {
        sort_scatter<<<grid_for(n, block), block, 0, s>>>(n, key, count, 6, st->f64, tmp64, 0, nullptr, 0, nullptr,
                                                          nullptr, order, order_tmp, rf_phase, phase_tmp);
        PPT_CUDA_TRY(cudaGetLastError());
        PPT_CUDA_TRY(cudaMemcpyAsync(st->f64, tmp64, (size_t)n * 6 * 8, cudaMemcpyDeviceToDevice, s));
    } else {
        // 3 int32 cell columns then 9 float32 columns, all 4-byte words
        sort_scatter<<<grid_for(n, block), block, 0, s>>>(
            n, key, count, 0, nullptr, nullptr, 3, reinterpret_cast<const uint32_t*>(st->i32), 9,
            reinterpret_cast<const uint32_t*>(st->f32), tmp32, order, order_tmp, rf_phase, phase_tmp);
        PPT_CUDA_TRY(cudaGetLastError());
        PPT_CUDA_TRY(cudaMemcpyAsync(st->i32, tmp32, (size_t)n * 3 * 4, cudaMemcpyDeviceToDevice, s));
        PPT_CUDA_TRY(cudaMemcpyAsync(st->f32, tmp32 + 3 * n, (size_t)n * 9 * 4, cudaMemcpyDeviceToDevice, s));
    }
    PPT_CUDA_TRY(cudaGetLastError());
    PPT_CUDA_TRY(cudaMemcpyAsync(order, order_tmp, (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
    if (rf_phase) PPT_CUDA_TRY(cudaMemcpyAsync(rf_phase, phase_tmp, (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
    return PPT_OK;
}
