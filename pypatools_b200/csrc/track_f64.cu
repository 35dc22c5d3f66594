// Plain form: launchers of the single-track kernels (track_f64_impl.cuh).
#include "track_f64_impl.cuh"

namespace ppt {

template <int ALG, int L>
static void launch_layout(const TrackDev& P, bool rf, int grid, int block, cudaStream_t s) {
    constexpr bool kE = layout_has_e(L);
    const size_t smem = (size_t)P.rf_tab_n * sizeof(double2);
    if (rf && kE) track_f64_kernel<ALG, kE, false, L><<<grid, block, smem, s>>>(P);
    else track_f64_kernel<ALG, false, false, L><<<grid, block, 0, s>>>(P);
}

template <int ALG>
static cudaError_t launch_alg(const TrackDev& P, bool rf, bool coll, cudaStream_t s) {
    const int block = pick_block(P.n);
    const int grid = grid_for(P.n, block);
    const size_t smem = (size_t)P.rf_tab_n * sizeof(double2);
    if (coll) {
        if (rf) track_f64_kernel<ALG, true, true, 0><<<grid, block, smem, s>>>(P);
        else track_f64_kernel<ALG, false, true, 0><<<grid, block, 0, s>>>(P);
        return cudaGetLastError();
    }
    switch (f64_single_layout(P)) {
        case kLayFull: launch_layout<ALG, kLayFull>(P, rf, grid, block, s); break;
        case kLayE: launch_layout<ALG, kLayE>(P, rf, grid, block, s); break;
        case kLayB: launch_layout<ALG, kLayB>(P, rf, grid, block, s); break;
        case kLayExEyBz: launch_layout<ALG, kLayExEyBz>(P, rf, grid, block, s); break;
        case kLayEzBz: launch_layout<ALG, kLayEzBz>(P, rf, grid, block, s); break;
        case kLayBz: launch_layout<ALG, kLayBz>(P, rf, grid, block, s); break;
        default:
            if (rf) track_f64_kernel<ALG, true, false, 0><<<grid, block, smem, s>>>(P);
            else track_f64_kernel<ALG, false, false, 0><<<grid, block, 0, s>>>(P);
    }
    return cudaGetLastError();
}

int launch_track_f64(const TrackDev& P, int algorithm, bool rf, bool coll, cudaStream_t s) {
    cudaError_t e;
    switch (algorithm) {
        case PPT_ALG_LEAPFROG: e = launch_alg<PPT_ALG_LEAPFROG>(P, rf, coll, s); break;
        case PPT_ALG_BORIS: e = launch_alg<PPT_ALG_BORIS>(P, rf, coll, s); break;
        case PPT_ALG_RK4: e = launch_alg<PPT_ALG_RK4>(P, rf, coll, s); break;
        case PPT_ALG_YOSHIDA: e = launch_alg<PPT_ALG_YOSHIDA>(P, rf, coll, s); break;
        case PPT_ALG_VAY_REL: e = launch_alg<PPT_ALG_VAY_REL>(P, rf, coll, s); break;
        case PPT_ALG_RK4_REL: e = launch_alg<PPT_ALG_RK4_REL>(P, rf, coll, s); break;
        case PPT_ALG_YOSHIDA_REL: e = launch_alg<PPT_ALG_YOSHIDA_REL>(P, rf, coll, s); break;
        case PPT_ALG_BORIS_REL: e = launch_alg<PPT_ALG_BORIS_REL>(P, rf, coll, s); break;
        case PPT_ALG_VAY: e = launch_alg<PPT_ALG_VAY>(P, rf, coll, s); break;
        default: return fail(PPT_ERR_ARG, "unknown algorithm");
    }
    if (e != cudaSuccess) return cuda_fail(e, "track_f64_kernel launch");
    return PPT_OK;
}

}  // namespace ppt
