// Kernel parameter blocks of the two track kernels (passed by value as
// __grid_constant__ parameters) and the host-side launch entry points.
#pragma once

#include "mixed_common.cuh"

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
    float hqdt;      // 0.5 q/m dt
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
};

int mixed_grid(const FieldsDev& F, GridF* G);
int check_state(const ppt_state* st);
int launch_track_f64(const TrackDev& P, int algorithm, bool rf, cudaStream_t s);
int make_track_mixed(const FieldsDev& F, const ppt_state* st, const ppt_track_args* a, int64_t n_rec,
                     TrackMixDev* P);
int launch_track_mixed(const TrackMixDev& P, int algorithm, bool rf, cudaStream_t s);

}  // namespace ppt
