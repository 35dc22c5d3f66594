// Cylindrical field maps onto a Cartesian node grid: the resampling step of
// the reference's midplane and multi-slice loaders (load_opal_midplane and
// load_aima_agora, src/PyPATools/field_src/field_loaders.py:612-640 and
// :836-899), which there runs scipy's RegularGridInterpolator point by point
// on the CPU.  For every Cartesian node (x_i, y_j):
//   r = sqrt(x^2 + y^2) * r_scale,  theta = degrees(atan2(y, x)) + 360 if < 0
//   (B_r, B_theta, B_z) = bilinear interpolation on the (r, theta) node grid,
//                         0 outside [r_0, r_last] x [theta_0, theta_last]
//   B_x = B_r cos(theta) - B_theta sin(theta),  B_y = B_r sin(theta) + B_theta cos(theta)
// Cell search as the interpolator's: the left node of the bracketing cell
// (searchsorted, side 'left', minus one) clamped to [0, n-2].
#include <cmath>

#include "ppt_internal.cuh"

namespace ppt {

struct PolarArgs {
    const double* r;        // nr node radii (device)
    const double* t;        // nt node angles [deg] (device)
    int64_t nr, nt;
    const double* comp[3];  // (nr, nt) B_r, B_theta, B_z or NULL
    const double* x;        // nx Cartesian node coordinates (device)
    const double* y;
    int64_t nx, ny;
    double r_scale;
    double* out[3];         // (nx, ny) B_x, B_y, B_z or NULL
};

// Left node of the bracketing cell, first index with g[i] >= v minus one.
__device__ __forceinline__ int64_t left_node(const double* g, int64_t n, double v) {
    int64_t lo = 0, hi = n;   // first index with g >= v lies in [lo, hi]
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (g[mid] < v) lo = mid + 1; else hi = mid;
    }
    int64_t i = lo - 1;
    return i < 0 ? 0 : (i > n - 2 ? n - 2 : i);
}

__global__ void polar_to_cartesian_kernel(const __grid_constant__ PolarArgs A) {
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= A.nx * A.ny) return;
    const int64_t i = p / A.ny, j = p - i * A.ny;
    const double x = A.x[i], y = A.y[j];
    // each product and sum rounded on its own, as numpy forms x**2 + y**2
    const double r = __dmul_rn(sqrt(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y))), A.r_scale);
    double th = atan2(y, x) * 57.29577951308232;   // degrees, as numpy's rad2deg
    if (th < 0.0) th += 360.0;
    double v[3] = {0.0, 0.0, 0.0};
    const bool inside = r >= A.r[0] && r <= A.r[A.nr - 1] && th >= A.t[0] && th <= A.t[A.nt - 1];
    if (inside) {
        const int64_t a = left_node(A.r, A.nr, r), b = left_node(A.t, A.nt, th);
        const double tr = (r - A.r[a]) / (A.r[a + 1] - A.r[a]);
        const double tt = (th - A.t[b]) / (A.t[b + 1] - A.t[b]);
        for (int c = 0; c < 3; ++c) {
            const double* f = A.comp[c];
            if (!f) continue;
            const double* row0 = f + a * A.nt;
            const double* row1 = row0 + A.nt;
            const double c0 = row0[b] * (1.0 - tr) + row1[b] * tr;
            const double c1 = row0[b + 1] * (1.0 - tr) + row1[b + 1] * tr;
            v[c] = c0 * (1.0 - tt) + c1 * tt;
        }
    }
    if (A.out[0] || A.out[1]) {
        double s, co;
        sincos(th * 0.017453292519943295, &s, &co);   // numpy's deg2rad factor
        if (A.out[0]) A.out[0][p] = v[0] * co - v[1] * s;
        if (A.out[1]) A.out[1][p] = v[0] * s + v[1] * co;
    }
    if (A.out[2]) A.out[2][p] = v[2];
}

}  // namespace ppt

using namespace ppt;

extern "C" int ppt_polar_to_cartesian(const ppt_polar_grid* grid, const double* const comp[3], int64_t nx,
                                      const double* x, int64_t ny, const double* y, double r_scale,
                                      double* const out[3], void* stream) {
    if (!grid || !comp || !out) return fail(PPT_ERR_ARG, "grid, comp and out must not be NULL");
    if (grid->nr < 2 || grid->nt < 2) return fail(PPT_ERR_ARG, "the polar grid needs >= 2 nodes per axis");
    if (!grid->r || !grid->theta) return fail(PPT_ERR_ARG, "polar node arrays must not be NULL");
    if (nx < 0 || ny < 0) return fail(PPT_ERR_ARG, "nx and ny must be >= 0");
    if (nx * ny == 0) return PPT_OK;
    if (!x || !y) return fail(PPT_ERR_ARG, "x and y must not be NULL");
    PolarArgs A;
    A.r = grid->r;
    A.t = grid->theta;
    A.nr = grid->nr;
    A.nt = grid->nt;
    for (int c = 0; c < 3; ++c) {
        A.comp[c] = comp[c];
        A.out[c] = out[c];
    }
    A.x = x;
    A.y = y;
    A.nx = nx;
    A.ny = ny;
    A.r_scale = r_scale;
    const int block = 256;
    polar_to_cartesian_kernel<<<grid_for(nx * ny, block), block, 0, static_cast<cudaStream_t>(stream)>>>(A);
    PPT_CUDA_TRY(cudaGetLastError());
    return PPT_OK;
}
