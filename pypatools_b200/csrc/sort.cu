// Particle reordering by cell, so that the threads of a warp gather the same
// corner records (one L1 wavefront per corner load instead of one per
// distinct cell).
//
// Counting sort on the particle's map-0 cell: bucket = linear cell index
// (k fastest) modulo 2^22 -- exact for maps up to 4M cells, a hash beyond;
// particles outside the map share one last bucket.  Histogram -> exclusive
// scan -> scatter into a scratch copy -> copy back, with warp-aggregated
// atomics (lanes with equal keys combine before touching memory).  The
// reordering runs when at least 1/16 of the particles are inside the map, or
// when the warps holding in-map particles exceed the ones those particles
// need by n/512 (a few particles still in the map after the bunch has left,
// spread over many warps: each such warp runs the gather path for one lane).
// Otherwise every kernel after the histogram returns at once: the sort is a
// no-op decided on the device, so the caller's stream never waits.
// Order inside a bucket is arbitrary; `order` records slot -> row so outputs
// land in the caller's row order, and each particle's arithmetic is
// independent of its slot.
#include <cstring>

#include "track_params.cuh"

namespace ppt {

constexpr int kBucketBits = 22;
constexpr int kScanTile = 1024;

struct SortGeom {
    double lo[3];
    double inv_d[3];
    int n[3];           // nodes per axis
    uint32_t n_in;      // buckets for in-map cells
    uint32_t outside;   // bucket of particles outside the map (= n_in)
    int flat[3];        // the map does not vary along the axis: its cell is not part of the key
};

__device__ __forceinline__ bool cell_inside(const SortGeom& G, int c0, int c1, int c2) {
    return (unsigned)c0 <= (unsigned)(G.n[0] - 2) && (unsigned)c1 <= (unsigned)(G.n[1] - 2) &&
           (unsigned)c2 <= (unsigned)(G.n[2] - 2);
}

__device__ __forceinline__ uint32_t bucket_of_cells(const SortGeom& G, int c0, int c1, int c2) {
    if (!cell_inside(G, c0, c1, c2)) return G.outside;
    const uint64_t lin = ((uint64_t)c0 * (uint64_t)(G.n[1] - 1) + (uint64_t)c1) * (uint64_t)(G.n[2] - 1) + (uint64_t)c2;
    return (uint32_t)(lin % G.n_in);
}

// Histogram of the in-map keys (one atomic per distinct key per warp), the
// in-map count and the number of warps with an in-map particle (one atomic
// each per block).  Particles outside the map touch no counter: their
// bucket's size is n minus the in-map count, filled in by the scan, so a
// bunch that has left the map costs no same-address atomics.  Called by every
// thread of the block (full warps).
__device__ __forceinline__ void count_key(uint32_t b, bool inside, uint32_t* count, uint32_t* ctrl) {
    __shared__ unsigned block_in, block_warps;
    if (threadIdx.x == 0) block_in = block_warps = 0;
    __syncthreads();
    if (__any_sync(0xffffffffu, inside) && (threadIdx.x & 31) == 0) atomicAdd(&block_warps, 1u);
    if (inside) {
        const unsigned active = __activemask();
        const unsigned same = __match_any_sync(active, b);
        const int lane = threadIdx.x & 31;
        if (lane == __ffs(same) - 1) {
            atomicAdd(count + b, (uint32_t)__popc(same));
            atomicAdd(&block_in, (unsigned)__popc(same));
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && block_in) {
        atomicAdd(ctrl, block_in);
        atomicAdd(ctrl + 1, block_warps);
    }
}

__global__ void sort_keys_f64(int64_t n, const double* __restrict__ st, SortGeom G, uint32_t* __restrict__ key,
                              uint32_t* __restrict__ count, uint32_t* __restrict__ ctrl) {
    const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    uint32_t b = G.outside;
    if (s < n) {
        int c[3];
        for (int a = 0; a < 3; ++a) {
            double u = (st[a * n + s] - G.lo[a]) * G.inv_d[a];
            c[a] = (u >= 0.0 && u < 2.0e9) ? (int)u : -1;
        }
        b = bucket_of_cells(G, c[0], c[1], c[2]);
        key[s] = b;
    }
    count_key(b, s < n && b != G.outside, count, ctrl);
}

__global__ void sort_keys_mixed(int64_t n, const int32_t* __restrict__ ci, SortGeom G, uint32_t* __restrict__ key,
                                uint32_t* __restrict__ count, uint32_t* __restrict__ ctrl) {
    const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    uint32_t b = G.outside;
    if (s < n) {
        // mixed-form cells on an axis the map does not vary along count
        // on their own grid, not the map's single layer
        b = bucket_of_cells(G, G.flat[0] ? 0 : ci[s], G.flat[1] ? 0 : ci[n + s], G.flat[2] ? 0 : ci[2 * n + s]);
        key[s] = b;
    }
    count_key(b, s < n && b != G.outside, count, ctrl);
}

__device__ __forceinline__ bool sort_wanted(const uint32_t* ctrl, int64_t n) {
    const int64_t in = ctrl[0], excess_warps = (int64_t)ctrl[1] - (in + 31) / 32;
    return in * 16 >= n || (in > 0 && excess_warps * 512 >= n);
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
                                                        uint32_t* __restrict__ offset, uint32_t* __restrict__ tile_sum,
                                                        const uint32_t* __restrict__ ctrl, int64_t n) {
    if (!sort_wanted(ctrl, n)) return;
    __shared__ uint32_t sh[32];
    int64_t i = blockIdx.x * (int64_t)kScanTile + threadIdx.x;
    uint32_t v = i < nb ? count[i] : 0u;
    if (i == nb - 1) v = (uint32_t)(n - (int64_t)ctrl[0]);   // the outside bucket: everything not in the map
    uint32_t total;
    uint32_t ex = block_exclusive_scan(v, sh, total);
    if (i < nb) offset[i] = ex;
    if (threadIdx.x == 0) tile_sum[blockIdx.x] = total;
}

// exclusive scan of the tile sums in one block
__global__ void __launch_bounds__(kScanTile) scan_top(int ntiles, uint32_t* __restrict__ tile_sum,
                                                      const uint32_t* __restrict__ ctrl, int64_t n) {
    if (!sort_wanted(ctrl, n)) return;
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

__global__ void scan_add(int64_t nb, uint32_t* __restrict__ offset, const uint32_t* __restrict__ tile_sum,
                         const uint32_t* __restrict__ ctrl, int64_t n) {
    if (!sort_wanted(ctrl, n)) return;
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < nb) offset[i] += tile_sum[i / kScanTile];
}

// Scatter every word of a slot's state: ncols64 columns of 8-byte words, and
// na + nb columns of 4-byte words taken from two sources (mixed state: the
// int32 cells, then the float32 columns) into one destination block.
__global__ void sort_scatter(int64_t n, const uint32_t* __restrict__ key, uint32_t* __restrict__ offset,
                             const uint32_t* __restrict__ ctrl, int ncols64, const double* __restrict__ src64,
                             double* __restrict__ dst64, int na, const uint32_t* __restrict__ src_a, int nb,
                             const uint32_t* __restrict__ src_b, uint32_t* __restrict__ dst32,
                             const int64_t* __restrict__ order, int64_t* __restrict__ order_out,
                             const double* __restrict__ phase, double* __restrict__ phase_out) {
    if (!sort_wanted(ctrl, n)) return;
    int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= n) return;
    const uint32_t b = key[s];
    const unsigned active = __activemask();
    const unsigned same = __match_any_sync(active, b);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(same) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(offset + b, (uint32_t)__popc(same));
    base = __shfl_sync(same, base, leader);
    const int64_t d = (int64_t)base + __popc(same & ((1u << lane) - 1u));
    for (int c = 0; c < ncols64; ++c) dst64[c * n + d] = src64[c * n + s];
    for (int c = 0; c < na; ++c) dst32[c * n + d] = src_a[c * n + s];
    for (int c = 0; c < nb; ++c) dst32[(na + c) * n + d] = src_b[c * n + s];
    order_out[d] = order[s];
    if (phase) phase_out[d] = phase[s];
}

// Copy the permuted block back (only when the sort ran).
__global__ void sort_copy_back(int64_t words, const uint32_t* __restrict__ src, uint32_t* __restrict__ dst,
                               const uint32_t* __restrict__ ctrl, int64_t n) {
    if (!sort_wanted(ctrl, n)) return;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < words; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

// Back to row order: position d takes the slot s with order[s] = d.  First
// the inverse, perm[order[s]] = s (order is a permutation of 0 .. n-1, kept
// so by the sorts; a value outside [0, n) is skipped), then a gather that
// reads the slots scattered and writes every column in order: for the cell
// order of a bunch that has crossed its map, 2.8 ms against 6.8 ms for the
// scatter (slot s written to position order[s]) at 1e7 mixed-form particles.
// (The cell sort keeps its scatter: for the random order of a fresh bunch the
// gather took 4.5 ms against 2.4 ms.)
__global__ void restore_inverse(int64_t n, const int64_t* __restrict__ order, uint32_t* __restrict__ perm) {
    const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int64_t d = order[s];
    if (d >= 0 && d < n) perm[d] = (uint32_t)s;
}

// Position d of the permuted copy takes slot perm[d]: ncols64 columns of
// 8-byte words and na + nb columns of 4-byte words from two sources (mixed
// state: the int32 cells, then the float32 columns) into one destination
// block, and the RF phase.  perm values outside [0, n) (positions no slot
// claimed; none for a permutation) leave position d unwritten.
__global__ void restore_gather(int64_t n, const uint32_t* __restrict__ perm, int ncols64,
                               const double* __restrict__ src64, double* __restrict__ dst64, int na,
                               const uint32_t* __restrict__ src_a, int nb, const uint32_t* __restrict__ src_b,
                               uint32_t* __restrict__ dst32, const double* __restrict__ phase,
                               double* __restrict__ phase_out) {
    const int64_t d = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (d >= n) return;
    const uint32_t s = perm[d];
    if ((int64_t)s >= n) return;
    for (int c = 0; c < ncols64; ++c) dst64[c * n + d] = src64[c * n + s];
    for (int c = 0; c < na; ++c) dst32[c * n + d] = src_a[c * n + s];
    for (int c = 0; c < nb; ++c) dst32[(na + c) * n + d] = src_b[c * n + s];
    if (phase) phase_out[d] = phase[s];
}

__global__ void iota_rows(int64_t n, int64_t* __restrict__ order) {
    const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s < n) order[s] = s;
}

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

struct SortLayout {
    size_t key, count, tiles, ctrl, tmp64, tmp32, order, phase, perm, total;
};

static SortLayout sort_layout(int64_t n) {
    SortLayout L;
    const size_t nb = ((size_t)1 << kBucketBits) + 1;
    size_t o = 0;
    L.key = o;   o += align256((size_t)n * 4);
    L.count = o; o += align256(nb * 4);
    L.tiles = o; o += align256((nb / kScanTile + 2) * 4);
    L.ctrl = o;  o += 256;
    L.tmp64 = o; o += align256((size_t)n * 6 * 8);     // float64 state
    L.tmp32 = o; o += align256((size_t)n * 15 * 4);    // mixed: 3 int32 + 12 float32 columns
    L.order = o; o += align256((size_t)n * 8);
    L.phase = o; o += align256((size_t)n * 8);
    L.perm = o;  o += align256((size_t)n * 4);    // restore: the inverse of order
    L.total = o;
    return L;
}

static void copy_back(const void* src, void* dst, size_t bytes, const uint32_t* ctrl, int64_t n, cudaStream_t s) {
    const int64_t words = (int64_t)(bytes / 4);
    const int block = 256;
    int64_t g = (words + block - 1) / block;
    const int grid = (int)(g > 148 * 16 ? 148 * 16 : (g < 1 ? 1 : g));
    sort_copy_back<<<grid, block, 0, s>>>(words, static_cast<const uint32_t*>(src), static_cast<uint32_t*>(dst), ctrl,
                                          n);
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
    if (!m.all_uniform) return PPT_OK;  // non-uniform maps: no cheap cell key, keep the order
    SortGeom G;
    uint64_t cells = 1;
    for (int a = 0; a < 3; ++a) {
        G.lo[a] = m.ax[a].lo;
        G.inv_d[a] = m.ax[a].inv_d;
        G.n[a] = m.ax[a].n;
        G.flat[a] = axis_is_flat(m.ax[a]) ? 1 : 0;
        cells *= (uint64_t)(m.ax[a].n - 1);
    }
    G.n_in = (uint32_t)(cells < ((uint64_t)1 << kBucketBits) ? cells : ((uint64_t)1 << kBucketBits));
    G.outside = G.n_in;
    const int64_t nb = (int64_t)G.n_in + 1;

    const int64_t n = st->n;
    SortLayout L = sort_layout(n);
    char* base = static_cast<char*>(scratch);
    uint32_t* key = reinterpret_cast<uint32_t*>(base + L.key);
    uint32_t* count = reinterpret_cast<uint32_t*>(base + L.count);
    uint32_t* tiles = reinterpret_cast<uint32_t*>(base + L.tiles);
    uint32_t* ctrl = reinterpret_cast<uint32_t*>(base + L.ctrl);
    double* tmp64 = reinterpret_cast<double*>(base + L.tmp64);
    uint32_t* tmp32 = reinterpret_cast<uint32_t*>(base + L.tmp32);
    int64_t* order_tmp = reinterpret_cast<int64_t*>(base + L.order);
    double* phase_tmp = reinterpret_cast<double*>(base + L.phase);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int block = 256;

    PPT_CUDA_TRY(cudaMemsetAsync(count, 0, (size_t)nb * 4, s));
    PPT_CUDA_TRY(cudaMemsetAsync(ctrl, 0, 8, s));
    if (st->precision == PPT_PREC_F64)
        sort_keys_f64<<<grid_for(n, block), block, 0, s>>>(n, st->f64, G, key, count, ctrl);
    else
        sort_keys_mixed<<<grid_for(n, block), block, 0, s>>>(n, st->i32, G, key, count, ctrl);
    const int ntiles = (int)((nb + kScanTile - 1) / kScanTile);
    scan_tiles<<<ntiles, kScanTile, 0, s>>>(nb, count, count, tiles, ctrl, n);
    scan_top<<<1, kScanTile, 0, s>>>(ntiles, tiles, ctrl, n);
    scan_add<<<grid_for(nb, block), block, 0, s>>>(nb, count, tiles, ctrl, n);
    if (st->precision == PPT_PREC_F64) {
        sort_scatter<<<grid_for(n, block), block, 0, s>>>(n, key, count, ctrl, 6, st->f64, tmp64, 0, nullptr, 0,
                                                          nullptr, nullptr, order, order_tmp, rf_phase, phase_tmp);
        copy_back(tmp64, st->f64, (size_t)n * 6 * 8, ctrl, n, s);
    } else {
        // 3 int32 cell columns then 12 float32 columns, all 4-byte words
        sort_scatter<<<grid_for(n, block), block, 0, s>>>(
            n, key, count, ctrl, 0, nullptr, nullptr, 3, reinterpret_cast<const uint32_t*>(st->i32), 12,
            reinterpret_cast<const uint32_t*>(st->f32), tmp32, order, order_tmp, rf_phase, phase_tmp);
        copy_back(tmp32, st->i32, (size_t)n * 3 * 4, ctrl, n, s);
        copy_back(tmp32 + 3 * n, st->f32, (size_t)n * 12 * 4, ctrl, n, s);
    }
    copy_back(order_tmp, order, (size_t)n * 8, ctrl, n, s);
    if (rf_phase) copy_back(phase_tmp, rf_phase, (size_t)n * 8, ctrl, n, s);
    PPT_CUDA_TRY(cudaGetLastError());
    return PPT_OK;
}

extern "C" int ppt_restore_order(ppt_state* st, int64_t* order, double* rf_phase, void* scratch, void* stream) {
    int rc = check_state(st);
    if (rc) return rc;
    if (st->n == 0) return PPT_OK;
    if (!order || !scratch) return fail(PPT_ERR_ARG, "order and scratch must not be NULL");
    const int64_t n = st->n;
    SortLayout L = sort_layout(n);
    char* base = static_cast<char*>(scratch);
    double* tmp64 = reinterpret_cast<double*>(base + L.tmp64);
    uint32_t* tmp32 = reinterpret_cast<uint32_t*>(base + L.tmp32);
    double* phase_tmp = reinterpret_cast<double*>(base + L.phase);
    uint32_t* perm = reinterpret_cast<uint32_t*>(base + L.perm);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int block = 256;
    PPT_CUDA_TRY(cudaMemsetAsync(perm, 0xff, (size_t)n * 4, s));   // unclaimed positions: skipped
    restore_inverse<<<grid_for(n, block), block, 0, s>>>(n, order, perm);
    if (st->precision == PPT_PREC_F64) {
        restore_gather<<<grid_for(n, block), block, 0, s>>>(n, perm, 6, st->f64, tmp64, 0, nullptr, 0, nullptr,
                                                            nullptr, rf_phase, phase_tmp);
        PPT_CUDA_TRY(cudaMemcpyAsync(st->f64, tmp64, (size_t)n * 6 * 8, cudaMemcpyDeviceToDevice, s));
    } else {
        restore_gather<<<grid_for(n, block), block, 0, s>>>(
            n, perm, 0, nullptr, nullptr, 3, reinterpret_cast<const uint32_t*>(st->i32), 12,
            reinterpret_cast<const uint32_t*>(st->f32), tmp32, rf_phase, phase_tmp);
        PPT_CUDA_TRY(cudaMemcpyAsync(st->i32, tmp32, (size_t)n * 3 * 4, cudaMemcpyDeviceToDevice, s));
        PPT_CUDA_TRY(cudaMemcpyAsync(st->f32, tmp32 + 3 * n, (size_t)n * 12 * 4, cudaMemcpyDeviceToDevice, s));
    }
    if (rf_phase) PPT_CUDA_TRY(cudaMemcpyAsync(rf_phase, phase_tmp, (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
    iota_rows<<<grid_for(n, block), block, 0, s>>>(n, order);
    PPT_CUDA_TRY(cudaGetLastError());
    return PPT_OK;
}
