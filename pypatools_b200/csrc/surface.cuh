// Electrode surfaces: a triangle mesh that stops particles whose step segment
// crosses it.
//
// Reference: Pusher.track_batch tests each step's segment (position before
// -> after the push) of every active particle against the electrode assembly
// and deactivates the ones that hit (src/PyPATools/pusher.py:970-990, calling
// PyElectrodeAssembly.segment_intersects_surface of the external py_electrodes
// package).  Here the surface is a triangle mesh on the device, binned into a
// uniform grid of cells; a segment is tested against the triangles of the
// cells its bounding box overlaps with the Moller-Trumbore ray-triangle test
// (T. Moller, B. Trumbore, "Fast, minimum storage ray-triangle
// intersection", J. Graphics Tools 2(1), 1997), restricted to the segment
// (0 <= t <= 1, edges and end points included).
//
// The test's arithmetic is written with explicitly rounded operations (no
// fused multiply-adds) in a fixed order, so every hit decision is the same
// as the NumPy restatement's, bit for bit.
#pragma once

#include "ppt_internal.cuh"

namespace ppt {

struct SurfaceDev {
    const double* tri;          // 9 per triangle: v0, e1 = v1 - v0, e2 = v2 - v0
    const int32_t* cell_start;  // cells + 1 offsets into cell_tri
    const int32_t* cell_tri;    // triangle indices, binned by cell ([i][j][k], k fastest)
    double lo[3];               // grid origin
    double inv_h[3];            // 1 / cell size
    int32_t dims[3];
    int32_t n_tri;
    const int32_t* trange;      // 6 per triangle: its first and last cell per axis (x0 x1 y0 y1 z0 z1)
};

__device__ __forceinline__ double rn_dot(double ax, double ay, double az, double bx, double by, double bz) {
    return __dadd_rn(__dadd_rn(__dmul_rn(ax, bx), __dmul_rn(ay, by)), __dmul_rn(az, bz));
}

__device__ __forceinline__ V3 rn_cross(V3 a, V3 b) {
    return v3(__dsub_rn(__dmul_rn(a.y, b.z), __dmul_rn(a.z, b.y)),
              __dsub_rn(__dmul_rn(a.z, b.x), __dmul_rn(a.x, b.z)),
              __dsub_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}

// Segment p0 + t d, t in [0, 1], against one triangle.
__device__ __forceinline__ bool segment_hits_triangle(const double* __restrict__ T, V3 p0, V3 d) {
    const V3 v0 = v3(T[0], T[1], T[2]);
    const V3 e1 = v3(T[3], T[4], T[5]);
    const V3 e2 = v3(T[6], T[7], T[8]);
    const V3 pv = rn_cross(d, e2);
    const double det = rn_dot(e1.x, e1.y, e1.z, pv.x, pv.y, pv.z);
    if (det == 0.0) return false;   // the segment is parallel to the triangle's plane
    const double inv = 1.0 / det;
    const V3 tv = v3(__dsub_rn(p0.x, v0.x), __dsub_rn(p0.y, v0.y), __dsub_rn(p0.z, v0.z));
    const double u = __dmul_rn(rn_dot(tv.x, tv.y, tv.z, pv.x, pv.y, pv.z), inv);
    if (!(u >= 0.0 && u <= 1.0)) return false;
    const V3 qv = rn_cross(tv, e1);
    const double v = __dmul_rn(rn_dot(d.x, d.y, d.z, qv.x, qv.y, qv.z), inv);
    if (!(v >= 0.0 && __dadd_rn(u, v) <= 1.0)) return false;
    const double t = __dmul_rn(rn_dot(e2.x, e2.y, e2.z, qv.x, qv.y, qv.z), inv);
    return t >= 0.0 && t <= 1.0;
}

// Does the segment p0 -> p1 meet any triangle of the surface?  The cells of
// the segment's bounding box are visited (one for the short steps of a
// tracking run); a triangle listed in several of them may be tested twice.
__device__ __forceinline__ bool segment_hits_surface(const SurfaceDev& S, V3 p0, V3 p1) {
    const double a0[3] = {p0.x, p0.y, p0.z}, a1[3] = {p1.x, p1.y, p1.z};
    int lo[3], hi[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const double u0 = (fmin(a0[a], a1[a]) - S.lo[a]) * S.inv_h[a];
        const double u1 = (fmax(a0[a], a1[a]) - S.lo[a]) * S.inv_h[a];
        if (!(u1 >= 0.0 && u0 < (double)S.dims[a])) return false;   // beyond the mesh (or NaN)
        lo[a] = u0 <= 0.0 ? 0 : (int)u0;
        hi[a] = u1 >= (double)(S.dims[a] - 1) ? S.dims[a] - 1 : (int)u1;
    }
    const V3 d = v3(__dsub_rn(p1.x, p0.x), __dsub_rn(p1.y, p0.y), __dsub_rn(p1.z, p0.z));
    for (int i = lo[0]; i <= hi[0]; ++i)
        for (int j = lo[1]; j <= hi[1]; ++j)
            for (int k = lo[2]; k <= hi[2]; ++k) {
                const int cell = (i * S.dims[1] + j) * S.dims[2] + k;
                const int end = S.cell_start[cell + 1];
                for (int q = S.cell_start[cell]; q < end; ++q)
                    if (segment_hits_triangle(S.tri + 9 * (int64_t)S.cell_tri[q], p0, d)) return true;
            }
    return false;
}

// Ray p + t d (t >= 0) against one triangle: the hit's t, or -1.  The same
// rounded operations as segment_hits_triangle.
__device__ __forceinline__ double ray_triangle_t(const double* __restrict__ T, V3 p0, V3 d) {
    const V3 v0 = v3(T[0], T[1], T[2]);
    const V3 e1 = v3(T[3], T[4], T[5]);
    const V3 e2 = v3(T[6], T[7], T[8]);
    const V3 pv = rn_cross(d, e2);
    const double det = rn_dot(e1.x, e1.y, e1.z, pv.x, pv.y, pv.z);
    if (det == 0.0) return -1.0;
    const double inv = 1.0 / det;
    const V3 tv = v3(__dsub_rn(p0.x, v0.x), __dsub_rn(p0.y, v0.y), __dsub_rn(p0.z, v0.z));
    const double u = __dmul_rn(rn_dot(tv.x, tv.y, tv.z, pv.x, pv.y, pv.z), inv);
    if (!(u >= 0.0 && u <= 1.0)) return -1.0;
    const V3 qv = rn_cross(tv, e1);
    const double v = __dmul_rn(rn_dot(d.x, d.y, d.z, qv.x, qv.y, qv.z), inv);
    if (!(v >= 0.0 && __dadd_rn(u, v) <= 1.0)) return -1.0;
    const double t = __dmul_rn(rn_dot(e2.x, e2.y, e2.z, qv.x, qv.y, qv.z), inv);
    return t >= 0.0 ? t : -1.0;
}

// Crossings of the axis-parallel ray from p in direction dir (0..5 = +x -x
// +y -y +z -z) with the surface: their number and the nearest one's distance
// (INFINITY without any).  The ray walks the column of grid cells it lies in;
// a triangle listed in several cells of the column is tested in the first of
// them the walk reaches.
__device__ __forceinline__ void axis_ray_hits(const SurfaceDev& S, V3 p, int dir, int& count, double& dist) {
    const int ax = dir >> 1;
    const double sgn = (dir & 1) ? -1.0 : 1.0;
    const double pc[3] = {p.x, p.y, p.z};
    count = 0;
    dist = INFINITY;
    int cell[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const double u = (pc[a] - S.lo[a]) * S.inv_h[a];
        if (!(u == u)) return;                                            // NaN
        if (a != ax && !(u >= 0.0 && u < (double)S.dims[a])) return;   // the column misses the mesh
        cell[a] = u < 0.0 ? -1 : (u >= (double)S.dims[a] ? S.dims[a] : (int)u);
    }
    const V3 d = v3(ax == 0 ? sgn : 0.0, ax == 1 ? sgn : 0.0, ax == 2 ? sgn : 0.0);
    int c0 = cell[ax], step = (dir & 1) ? -1 : 1;
    if (step > 0) c0 = c0 < 0 ? 0 : c0;
    else c0 = c0 >= S.dims[ax] ? S.dims[ax] - 1 : c0;
    for (int c = c0; c >= 0 && c < S.dims[ax]; c += step) {
        cell[ax] = c;
        const int lin = (cell[0] * S.dims[1] + cell[1]) * S.dims[2] + cell[2];
        const int end = S.cell_start[lin + 1];
        for (int q = S.cell_start[lin]; q < end; ++q) {
            const int tri = S.cell_tri[q];
            const int lo = S.trange[6 * tri + 2 * ax], hi = S.trange[6 * tri + 2 * ax + 1];
            const int first = step > 0 ? (c0 > lo ? c0 : lo) : (c0 < hi ? c0 : hi);
            if (c != first) continue;     // tested in an earlier cell of the walk
            const double t = ray_triangle_t(S.tri + 9 * (int64_t)tri, p, d);
            if (t >= 0.0) {
                ++count;
                dist = t < dist ? t : dist;
            }
        }
    }
}

}  // namespace ppt

struct ppt_surface {
    int device;
    ppt::SurfaceDev dev;
    void* buf;          // one device allocation: triangles, cell offsets, cell lists
    size_t bytes;
};
