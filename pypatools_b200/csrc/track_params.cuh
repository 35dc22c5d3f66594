// Kernel parameter blocks of the two track kernels (passed by value as
// __grid_constant__ parameters) and the host-side launch entry points.
#pragma once

#include "mixed_common.cuh"
#include "surface.cuh"

namespace ppt {

struct TrackDev {
    FieldsDev F;
    int64_t n;
    int64_t step0;
    int64_t nsteps;
    int64_t nsteps_total;
    int64_t rec_every;
    int64_t n_rec;
    int flags;
    double dt;
    double qm;
    double t0;
    double omega;
    const double* rf_phase;
    double* f64;
    double* r_hist;
    double* v_hist;
    const int64_t* order;
    int* status;
    unsigned long long* counters;
    SurfaceDev surf;    // electrode surface (n_tri = 0: none)
    uint8_t* active;    // row order; with a surface, 0 = stopped by it
    const double* dt_rows;   // RK4 / rk4_rel: one dt per particle, row order (NULL: dt)
    int32_t rf_tab_n;        // entries of the per-step RF table a launch builds (0: none)
    int32_t pad_;
};

struct TrackMixDev {
    MapDev map;
    GridF G;
    float e_const[3];
    float b_const[3];
    int const_nz;
    int64_t n;
    int64_t step0;
    int64_t nsteps;
    int64_t nsteps_total;
    int64_t rec_every;
    int64_t n_rec;
    int flags;
    double dt;
    double t0;
    double omega;
    double wdt;      // omega dt
    float qm;        // q/m
    float hqdt;      // 0.5 q/m dt, rounded to float32 (wscale below corrects the rounding)
    float dtf;       // dt
    float kh[3];     // dt / d: cell units per (m/s), as a float-float pair
    float kl[3];
    float inv_d[3];  // 1 / d (RK4 stage positions)
    float cell_max[3];  // n - 1 per axis: last node layer, for the cheap in-map pre-test
    const double* rf_phase;
    int32_t* ci;
    float* fs;
    double* r_hist;
    double* v_hist;
    const int64_t* order;
    int* status;
    unsigned long long* counters;
    int32_t rf_tab_n;   // entries of the per-step RF table a launch builds (0: none)
    float wscale;       // Boris: (0.5 q/m dt) / hqdt - 1, applied to each velocity increment
    int32_t k_elems;    // map elements per z cell: the record width, 0 when the map does not vary along z
    uint32_t inner_span[3];   // n - 3 per axis (0 below 4 nodes): cells 1 .. n-3 have inner corners only
};

// The electrode surface of a mixed-form Boris track (a second kernel
// parameter, so the parameter block of the kernels without one stays as it is).
struct CollDev {
    SurfaceDev surf;
    uint8_t* active;    // row order; 0 = stopped by the surface
};

// One (form, algorithm, RF) class of serving jobs: a block-level work queue
// over items = (job, 128-particle block) pairs.  The job tables, the per-job
// step counters and done flags live in device memory, so a tick needs no
// host data and can be replayed from a captured CUDA graph.
struct JobQueueDev {
    const void* table;        // TrackDev[] (float64 jobs) or TrackMixDev[] (mixed jobs), by table index
    const int* table_index;   // class-local job -> table index
    const int* job_index;     // class-local job -> global job index (steps / done)
    const int* item_start;    // class-local prefix sums of items, n_jobs + 1 entries
    int n_jobs;
    int n_items;
    unsigned* queue;          // work-queue head, zeroed before each tick
    const int64_t* steps;     // steps done per global job
    const int* done;          // 1 once the job's last step ran
    const int64_t* window;    // steps per tick per global job (0: chunk)
    int64_t chunk;            // steps per tick
};

constexpr int kJobBlock = 128;

// The record layout a float64 launch is specialised on: one uniform-grid map
// and no constant field parts; 0 otherwise (the run-time dispatch over any
// number of maps).  Single tracks and serving jobs use the same rule, so a
// job runs the same kernel code alone and in a serving mix.
inline int f64_single_layout(const TrackDev& P) {
    if (P.F.n_maps != 1 || P.F.e_const_nz || P.F.b_const_nz || !P.F.maps[0].all_uniform) return 0;
    return P.F.maps[0].layout;
}

int mixed_grid(const FieldsDev& F, GridF* G);
int check_state(const ppt_state* st);
int launch_track_f64(const TrackDev& P, int algorithm, bool rf, bool surface, cudaStream_t s);
int make_track_mixed(const FieldsDev& F, const ppt_state* st, const ppt_track_args* a, int64_t n_rec,
                     TrackMixDev* P);
int launch_track_mixed(const TrackMixDev& P, int algorithm, bool rf, cudaStream_t s);
int launch_track_mixed_coll(const TrackMixDev& P, const CollDev& C, bool rf, cudaStream_t s);
int launch_f64_jobs(const JobQueueDev& Q, int algorithm, int layout, bool rf, int grid, cudaStream_t s);
int launch_mixed_jobs(const JobQueueDev& Q, int algorithm, int layout, bool rf, int grid, cudaStream_t s);

// Device helper shared by both job kernels: thread 0 takes the next item and
// finds its class-local job by bisection over item_start.
__device__ __forceinline__ void take_item(const JobQueueDev& Q, int* s_item, int* s_job) {
    if (threadIdx.x == 0) {
        const int it = (int)atomicAdd(Q.queue, 1u);
        int lo = 0, hi = Q.n_jobs;   // item_start[lo] <= it < item_start[hi]
        if (it < Q.n_items) {
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (Q.item_start[mid] <= it) lo = mid; else hi = mid;
            }
        }
        *s_item = it;
        *s_job = lo;
    }
    __syncthreads();
}

// Add a block's in-map gathers and particle steps to the two device
// counters: warp sums by shuffle, then one atomic pair per block (per-warp
// atomics on the same two addresses serialised at the end of short launches).
// Every thread of the block calls it.
__device__ __forceinline__ void block_add_counters(unsigned long long* counters, unsigned hits, unsigned steps) {
    __shared__ unsigned long long part[2][32];
    unsigned long long h = hits, s = steps;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        h += __shfl_down_sync(0xffffffffu, h, o);
        s += __shfl_down_sync(0xffffffffu, s, o);
    }
    const int warp = threadIdx.x >> 5, warps = (blockDim.x + 31) >> 5;
    if ((threadIdx.x & 31) == 0) {
        part[0][warp] = h;
        part[1][warp] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < warps; ++w) {
            h += part[0][w];
            s += part[1][w];
        }
        atomicAdd(counters, h);
        atomicAdd(counters + 1, s);
    }
    __syncthreads();   // part[] is reused by the next call in the block
}

// Step window of a job in this tick: [step0, step0 + k) and its flags.
__device__ __forceinline__ void job_window(const JobQueueDev& Q, int gjob, int64_t total, int64_t* step0,
                                           int64_t* k, int* flags) {
    const int64_t s0 = Q.steps[gjob];
    const int64_t w = Q.window[gjob] > 0 ? Q.window[gjob] : Q.chunk;
    int64_t kk = total - s0;
    if (kk > w) kk = w;
    if (kk < 0) kk = 0;
    *step0 = s0;
    *k = kk;
    *flags = (s0 == 0 ? PPT_TRACK_INIT : 0) | (s0 + kk == total ? PPT_TRACK_FINAL : 0);
}

}  // namespace ppt
