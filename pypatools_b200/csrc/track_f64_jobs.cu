// Plain form: launchers of the serving job kernels (track_f64_impl.cuh),
// specialised on the record layout exactly as the single-track kernels are
// (f64_single_layout), so a job runs the same code served and alone.
#include "track_f64_impl.cuh"

namespace ppt {

template <int ALG, int L>
static void launch_jobs_layout(const JobQueueDev& Q, bool rf, int grid, cudaStream_t s) {
    constexpr bool kE = L == 0 || layout_has_e(L);
    if (rf && kE) track_f64_jobs_kernel<ALG, kE, L><<<grid, kJobBlock, 0, s>>>(Q);
    else track_f64_jobs_kernel<ALG, false, L><<<grid, kJobBlock, 0, s>>>(Q);
}

template <int ALG>
static cudaError_t launch_jobs_alg(const JobQueueDev& Q, int layout, bool rf, int grid, cudaStream_t s) {
    switch (layout) {
        case kLayFull: launch_jobs_layout<ALG, kLayFull>(Q, rf, grid, s); break;
        case kLayE: launch_jobs_layout<ALG, kLayE>(Q, rf, grid, s); break;
        case kLayB: launch_jobs_layout<ALG, kLayB>(Q, rf, grid, s); break;
        case kLayExEyBz: launch_jobs_layout<ALG, kLayExEyBz>(Q, rf, grid, s); break;
        case kLayEzBz: launch_jobs_layout<ALG, kLayEzBz>(Q, rf, grid, s); break;
        case kLayBz: launch_jobs_layout<ALG, kLayBz>(Q, rf, grid, s); break;
        default: launch_jobs_layout<ALG, 0>(Q, rf, grid, s); break;
    }
    return cudaGetLastError();
}

int launch_f64_jobs(const JobQueueDev& Q, int algorithm, int layout, bool rf, int grid, cudaStream_t s) {
    cudaError_t e;
    switch (algorithm) {
        case PPT_ALG_LEAPFROG: e = launch_jobs_alg<PPT_ALG_LEAPFROG>(Q, layout, rf, grid, s); break;
        case PPT_ALG_BORIS: e = launch_jobs_alg<PPT_ALG_BORIS>(Q, layout, rf, grid, s); break;
        case PPT_ALG_RK4: e = launch_jobs_alg<PPT_ALG_RK4>(Q, layout, rf, grid, s); break;
        case PPT_ALG_YOSHIDA: e = launch_jobs_alg<PPT_ALG_YOSHIDA>(Q, layout, rf, grid, s); break;
        case PPT_ALG_VAY_REL: e = launch_jobs_alg<PPT_ALG_VAY_REL>(Q, layout, rf, grid, s); break;
        case PPT_ALG_RK4_REL: e = launch_jobs_alg<PPT_ALG_RK4_REL>(Q, layout, rf, grid, s); break;
        case PPT_ALG_YOSHIDA_REL: e = launch_jobs_alg<PPT_ALG_YOSHIDA_REL>(Q, layout, rf, grid, s); break;
        case PPT_ALG_BORIS_REL: e = launch_jobs_alg<PPT_ALG_BORIS_REL>(Q, layout, rf, grid, s); break;
        case PPT_ALG_VAY: e = launch_jobs_alg<PPT_ALG_VAY>(Q, layout, rf, grid, s); break;
        default: return fail(PPT_ERR_ARG, "unknown algorithm");
    }
    if (e != cudaSuccess) return cuda_fail(e, "track_f64_jobs_kernel launch");
    return PPT_OK;
}

}  // namespace ppt
