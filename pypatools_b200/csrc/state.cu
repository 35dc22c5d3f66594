// Conversion between the reference's (M,3) float64 r / v arrays
// (Pusher.track_batch inputs and outputs, src/PyPATools/pusher.py:894-1012)
// and the device structure-of-arrays particle state the track kernels keep.
#include <algorithm>
#include <cmath>

#include "ppt_internal.cuh"
#include "mixed_common.cuh"

namespace ppt {

__global__ void load_f64_kernel(int64_t n, const double* __restrict__ r, const double* __restrict__ v,
                                double* __restrict__ st, int u_state) {
    int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= n) return;
    double vx = v[3 * s], vy = v[3 * s + 1], vz = v[3 * s + 2];
    if (u_state) {
        double g = 1.0 / sqrt(1.0 - (vx * vx + vy * vy + vz * vz) / (kClight * kClight));
        vx *= g;
        vy *= g;
        vz *= g;
    }
    st[s] = r[3 * s];
    st[n + s] = r[3 * s + 1];
    st[2 * n + s] = r[3 * s + 2];
    st[3 * n + s] = vx;
    st[4 * n + s] = vy;
    st[5 * n + s] = vz;
}

__global__ void store_f64_kernel(int64_t n, const double* __restrict__ st, const int64_t* __restrict__ order,
                                 double* __restrict__ r, double* __restrict__ v, int u_state) {
    int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int64_t row = order ? order[s] : s;
    double wx = st[3 * n + s], wy = st[4 * n + s], wz = st[5 * n + s];
    if (u_state) {
        double ig = 1.0 / sqrt(1.0 + (wx * wx + wy * wy + wz * wz) / (kClight * kClight));
        wx *= ig;
        wy *= ig;
        wz *= ig;
    }
    if (r) {
        r[3 * row] = st[s];
        r[3 * row + 1] = st[n + s];
        r[3 * row + 2] = st[2 * n + s];
    }
    if (v) {
        v[3 * row] = wx;
        v[3 * row + 1] = wy;
        v[3 * row + 2] = wz;
    }
}

__global__ void load_mixed_kernel(int64_t n, const double* __restrict__ r, const double* __restrict__ v,
                                  int32_t* __restrict__ ci, float* __restrict__ fs, GridF G, int u_state,
                                  int* status) {
    int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= n) return;
    double vv[3] = {v[3 * s], v[3 * s + 1], v[3 * s + 2]};
    if (u_state) {
        double g = 1.0 / sqrt(1.0 - (vv[0] * vv[0] + vv[1] * vv[1] + vv[2] * vv[2]) / (kClight * kClight));
        for (int c = 0; c < 3; ++c) vv[c] *= g;
    }
    for (int c = 0; c < 3; ++c) {
        double u = (r[3 * s + c] - G.lo[c]) * G.inv_d[c];
        double fl = floor(u);
        if (!(fabs(fl) < 2.0e9)) {           // cell index must fit int32 (NaN too)
            if (status) atomicOr(status, PPT_STATUS_NONFINITE);
            fl = 0.0;
            u = 0.0;
        }
        int cell = (int)fl;
        const double off = u - fl;           // in [0, 1)
        // the high word on the 2^-22 grid the Boris family's steps keep it on
        // (exact additions, track_mixed.cu add_cells_q), the rest in the low word
        const double fq = rint(off * 0x1p22) * 0x1p-22;
        float f = (float)fq;
        float f_lo = (float)(off - fq);
        if (f >= 1.0f) {                     // off within 2^-23 of 1: the next cell's node
            f = 0.0f;
            cell += 1;
        }
        ci[c * n + s] = cell;
        fs[c * n + s] = f;
        fs[(9 + c) * n + s] = f_lo;
        float hi = (float)vv[c];
        float lo = (float)(vv[c] - (double)hi);
        fs[(3 + c) * n + s] = hi;
        fs[(6 + c) * n + s] = lo;
    }
}

__global__ void store_mixed_kernel(int64_t n, const int32_t* __restrict__ ci, const float* __restrict__ fs,
                                   const int64_t* __restrict__ order, double* __restrict__ r,
                                   double* __restrict__ v, GridF G, int u_state) {
    int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int64_t row = order ? order[s] : s;
    double w[3];
    for (int c = 0; c < 3; ++c) w[c] = (double)fs[(3 + c) * n + s] + (double)fs[(6 + c) * n + s];
    if (u_state) {
        double ig = 1.0 / sqrt(1.0 + (w[0] * w[0] + w[1] * w[1] + w[2] * w[2]) / (kClight * kClight));
        for (int c = 0; c < 3; ++c) w[c] *= ig;
    }
    for (int c = 0; c < 3; ++c) {
        if (r) r[3 * row + c] = G.lo[c] + ((double)ci[c * n + s] + ((double)fs[c * n + s] + (double)fs[(9 + c) * n + s])) * G.d[c];
        if (v) v[3 * row + c] = w[c];
    }
}

int mixed_grid(const FieldsDev& F, GridF* G) {
    if (F.n_maps != 1)
        return fail(PPT_ERR_UNSUPPORTED, "the mixed form needs exactly one field map (E, B or E+B on one grid)");
    const MapDev& m = F.maps[0];
    if (m.dtype != PPT_DTYPE_F32) return fail(PPT_ERR_ARG, "the mixed form needs a float32 map");
    if (!m.all_uniform) return fail(PPT_ERR_UNSUPPORTED, "the mixed form needs uniform grid axes");
    // Along an axis the map does not vary, positions still need cells: a
    // grid of 2^24 cells of the finest spacing of the other axes, centred on
    // 0 (every cell of it reads the map's one layer; make_track_mixed zeroes
    // the map stride of that axis).  Cell indices stay below 2^24, exact in
    // float32 as the kernels need.
    double fine = 0.0;
    for (int c = 0; c < 3; ++c)
        if (!axis_is_flat(m.ax[c])) fine = fine == 0.0 ? m.ax[c].d : std::min(fine, m.ax[c].d);
    for (int c = 0; c < 3; ++c) {
        if (axis_is_flat(m.ax[c])) {
            G->d[c] = fine;
            G->inv_d[c] = 1.0 / fine;
            G->lo[c] = -(double)(1 << 23) * fine;
            G->n[c] = (1 << 24) + 1;
            continue;
        }
        G->lo[c] = m.ax[c].lo;
        G->d[c] = m.ax[c].d;
        G->inv_d[c] = m.ax[c].inv_d;
        G->n[c] = m.ax[c].n;
    }
    return PPT_OK;
}

int check_state(const ppt_state* st) {
    if (!st) return fail(PPT_ERR_ARG, "state is NULL");
    if (st->n < 0) return fail(PPT_ERR_ARG, "state n must be >= 0");
    if (st->algorithm < 0 || st->algorithm >= PPT_ALG_COUNT) return fail(PPT_ERR_ARG, "unknown algorithm");
    if (st->precision == PPT_PREC_F64) {
        if (st->n > 0 && !st->f64) return fail(PPT_ERR_ARG, "float64 state needs the f64 buffer");
    } else if (st->precision == PPT_PREC_MIXED) {
        if (st->n > 0 && (!st->i32 || !st->f32)) return fail(PPT_ERR_ARG, "mixed state needs i32 and f32 buffers");
    } else {
        return fail(PPT_ERR_ARG, "unknown precision");
    }
    return PPT_OK;
}

}  // namespace ppt

using namespace ppt;

extern "C" int ppt_state_load(ppt_state* st, const ppt_fields* fields, const double* r, const double* v,
                              void* stream) {
    int rc = check_state(st);
    if (rc) return rc;
    if (st->n == 0) return PPT_OK;
    if (!r || !v) return fail(PPT_ERR_ARG, "r and v must not be NULL");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int u_state = st->algorithm == PPT_ALG_BORIS_REL || st->algorithm == PPT_ALG_VAY;
    const int block = 256;
    if (st->precision == PPT_PREC_F64) {
        load_f64_kernel<<<grid_for(st->n, block), block, 0, s>>>(st->n, r, v, st->f64, u_state);
    } else {
        FieldsDev F;
        rc = build_fields(fields, &F);
        if (rc) return rc;
        GridF G;
        rc = mixed_grid(F, &G);
        if (rc) return rc;
        load_mixed_kernel<<<grid_for(st->n, block), block, 0, s>>>(st->n, r, v, st->i32, st->f32, G, u_state,
                                                                   nullptr);
    }
    PPT_CUDA_TRY(cudaGetLastError());
    return PPT_OK;
}

extern "C" int ppt_state_store(const ppt_state* st, const ppt_fields* fields, const int64_t* order, double* r,
                               double* v, void* stream) {
    int rc = check_state(st);
    if (rc) return rc;
    if (st->n == 0) return PPT_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int u_state = st->algorithm == PPT_ALG_BORIS_REL || st->algorithm == PPT_ALG_VAY;
    const int block = 256;
    if (st->precision == PPT_PREC_F64) {
        store_f64_kernel<<<grid_for(st->n, block), block, 0, s>>>(st->n, st->f64, order, r, v, u_state);
    } else {
        FieldsDev F;
        rc = build_fields(fields, &F);
        if (rc) return rc;
        GridF G;
        rc = mixed_grid(F, &G);
        if (rc) return rc;
        store_mixed_kernel<<<grid_for(st->n, block), block, 0, s>>>(st->n, st->i32, st->f32, order, r, v, G,
                                                                    u_state);
    }
    PPT_CUDA_TRY(cudaGetLastError());
    return PPT_OK;
}
