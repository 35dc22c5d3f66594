// Internal declarations shared by the libppt CUDA sources.
//
// Device-side field-map layout (what the hot kernels gather from):
//   one record per node, nodes in [i][j][k] order (k fastest, the 'ij'
//   meshgrid order of the reference's NumbaInterpolator values,
//   src/PyPATools/field_src/interpolators.py:118-125);
//   record = [Fx Fy Fz 0] for a map that stores one field (E or B), or
//            [Ex Ey Ez 0 | Bx By Bz 0] for a map that stores both,
//   in float64 (plain form, 32 B per field per node, one 256-bit load) or
//   float32 (mixed form, 16 B per field per node, one 128-bit load).
//   The 4th slot is padding so every field of every node starts on a 16/32-B
//   boundary; the algorithmic byte counts exclude it.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>

#include "../../include/ppt.h"

namespace ppt {

constexpr double kClight = 299792458.0;   // scipy.constants.speed_of_light

// ---------------------------------------------------------------------------
// error reporting (thread-local message behind ppt_last_error)
// ---------------------------------------------------------------------------
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t err, const char* what);

#define PPT_CUDA_TRY(expr)                                              \
    do {                                                                \
        cudaError_t _e = (expr);                                        \
        if (_e != cudaSuccess) return ::ppt::cuda_fail(_e, #expr);      \
    } while (0)

// ---------------------------------------------------------------------------
// host-side map object (behind the opaque ppt_fieldmap handle)
// ---------------------------------------------------------------------------
struct AxisDev {
    double lo;        // first node (exact, bounds test x < lo)
    double hi;        // last node  (exact, bounds test x > hi)
    double inv_d;     // (n-1)/(hi-lo), uniform axes
    double d;         // (hi-lo)/(n-1)
    const double* nodes;  // device copy of the node coordinates
    int n;
    int uniform;
};

// An axis along which a map does not vary (the reference's 1D fields vary
// along z only, its 2D fields along x and y: field.py:457-489) is stored as
// two identical node layers at -2^996 and +2^996: every finite coordinate is
// inside, the uniform cell search gives cell 0 and weight exactly 1/2, and
// the lerp of two equal values is exact, so the 3D interpolation reduces
// bit for bit to the 1D / 2D one without a branch in the kernels.
constexpr double kFlatHalf = 0x1p996;

__host__ __device__ __forceinline__ bool axis_is_flat(const AxisDev& a) {
    return a.n == 2 && a.lo == -kFlatHalf && a.hi == kFlatHalf;
}

// Record layouts, named by the component mask they store (bit c = Ex, Ey,
// Ez, Bx, By, Bz).  Up to three components are packed in Ex..Bz order in
// records of 1, 2 or 4 elements; all six use [Ex Ey Ez 0 | Bx By Bz 0].
constexpr int kLayFull = 0x3F;
constexpr int kLayE = 0x07;
constexpr int kLayB = 0x38;
constexpr int kLayExEyBz = 0x23;
constexpr int kLayEzBz = 0x24;
constexpr int kLayBz = 0x20;

__host__ __device__ constexpr int layout_width(int layout) {
    return layout == kLayFull ? 8 : (layout == kLayEzBz ? 2 : (layout == kLayBz ? 1 : 4));
}
__host__ __device__ constexpr bool layout_has_e(int layout) { return (layout & 0x07) != 0; }
__host__ __device__ constexpr bool layout_has_b(int layout) { return (layout & 0x38) != 0; }

// Components a record layout can make non-zero: bit a of e_bits (b_bits)
// is E_a (B_a); the six-component layout also carries the constant parts.
// x * 0 and x + 0 are not identities in IEEE arithmetic (NaN, signed
// zeros), so the compiler keeps every operation on a component that is
// zero by construction unless the code leaves it out: the Boris kernels of
// both precision forms do, at compile time, from these masks.
__host__ __device__ constexpr int e_bits(int L) { return L & 7; }
__host__ __device__ constexpr int b_bits(int L) { return (L >> 3) & 7; }
__host__ __device__ constexpr bool bit(int m, int a) { return ((m >> a) & 1) != 0; }
// components of p x q that can be non-zero when q has the components of qm
__host__ __device__ constexpr int cross_bits(int qm) {
    return ((bit(qm, 1) || bit(qm, 2)) ? 1 : 0) | ((bit(qm, 2) || bit(qm, 0)) ? 2 : 0) |
           ((bit(qm, 0) || bit(qm, 1)) ? 4 : 0);
}
// velocity components a Boris step can change under layout L
__host__ __device__ constexpr int boris_bits(int L) { return e_bits(L) | cross_bits(b_bits(L)); }


struct MapDev {
    const void* data;
    int64_t sx;       // node stride of i  (= ny*nz)
    int64_t sy;       // node stride of j  (= nz)
    int stride;       // elements per node record (1, 2, 4 or 8)
    int layout;       // the kLay* component mask the records store
    int has_e;
    int has_b;
    int b_off;        // element offset of B in a full-layout record (4)
    int dtype;        // PPT_DTYPE_F64 / PPT_DTYPE_F32
    int all_uniform;
    int idx32;        // every element offset (nodes x stride) fits in int32
    AxisDev ax[3];
};

}  // namespace ppt

struct ppt_fieldmap {
    int device;
    ppt::MapDev dev;
    double* axis_buf;     // device node coordinates of all three axes
    void* data;
    size_t bytes;
    int64_t n[3];     // stored node layers per axis (2 for an axis the map does not vary along)
    int64_t src_n[3]; // node counts of the caller's arrays (1 for such an axis)
};

namespace ppt {

struct FieldsDev {
    MapDev maps[PPT_MAX_MAPS];
    int n_maps;
    int e_maps;       // number of maps carrying E
    int b_maps;
    int e_const_nz;   // e_const not all zero
    int b_const_nz;
    double e_const[3];
    double b_const[3];
    double box_lo[3];   // union of the maps' node boxes: a point outside it is outside every map
    double box_hi[3];
};

int build_fields(const ppt_fields* f, FieldsDev* out);

// ---------------------------------------------------------------------------
// small vector helpers
// ---------------------------------------------------------------------------
struct V3 {
    double x, y, z;
};

__host__ __device__ __forceinline__ V3 v3(double x, double y, double z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ V3 operator*(double s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ V3 operator*(V3 a, double s) { return v3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ V3 operator/(V3 a, double s) { return v3(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
    // a x b, component order of the reference's cross_product (pusher.py:99-106)
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

// 256-bit read-only load of four float64 values (32-B aligned address).
__device__ __forceinline__ void ldg_f64x4(const double* p, double& a, double& b, double& c, double& d) {
    asm volatile("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];"
                 : "=d"(a), "=d"(b), "=d"(c), "=d"(d)
                 : "l"(p));
}

// ---------------------------------------------------------------------------
// cell location on one axis (float64)
// ---------------------------------------------------------------------------
// In-domain test, cell index and weight on one axis, following
// interpolators.py:93-115: outside when x < g[0] or x > g[n-1] (so the last
// node is inside); cell = bracketing left node clamped to [0, n-2];
// weight t = (x - g[i]) / (g[i+1] - g[i]) clamped to [0, 1].
// Uniform axes get the cell by (x - lo) * inv_d instead of a binary search:
// the interpolant is continuous across cells, so a cell picked one off at a
// node changes the result only by rounding.
__device__ __forceinline__ bool locate_axis(const AxisDev& a, double x, int& i, double& t) {
    if (!(x >= a.lo && x <= a.hi)) return false;   // NaN counts as outside
    if (a.uniform) {
        double u = (x - a.lo) * a.inv_d;
        int c = (int)floor(u);
        c = c < 0 ? 0 : (c > a.n - 2 ? a.n - 2 : c);
        double tt = u - (double)c;
        t = tt < 0.0 ? 0.0 : (tt > 1.0 ? 1.0 : tt);
        i = c;
    } else {
        // interpolators.py:44-60: left/right bisection with g[mid] <= x
        const double* g = a.nodes;
        int left = 0, right = a.n - 1;
        if (x >= g[a.n - 1]) {
            left = a.n - 2;
        } else {
            while (left < right - 1) {
                int mid = (left + right) >> 1;
                if (g[mid] <= x) left = mid; else right = mid;
            }
        }
        double g0 = g[left], g1 = g[left + 1];
        double tt = (x - g0) / (g1 - g0);
        t = tt < 0.0 ? 0.0 : (tt > 1.0 ? 1.0 : tt);
        i = left;
    }
    return true;
}

struct Cell {
    int64_t base;     // node index of corner (i, j, k)
    double tx, ty, tz;
};

__device__ __forceinline__ bool axis_contains(const AxisDev& a, double x) { return x >= a.lo && x <= a.hi; }

__device__ __forceinline__ bool locate(const MapDev& m, V3 r, Cell& c) {
    int i, j, k;
    // the three bounds tests first: a point outside on any axis costs no cell search
    if (!(axis_contains(m.ax[0], r.x) & axis_contains(m.ax[1], r.y) & axis_contains(m.ax[2], r.z))) return false;
    if (!locate_axis(m.ax[0], r.x, i, c.tx)) return false;
    if (!locate_axis(m.ax[1], r.y, j, c.ty)) return false;
    if (!locate_axis(m.ax[2], r.z, k, c.tz)) return false;
    c.base = (int64_t)i * m.sx + (int64_t)j * m.sy + k;
    return true;
}

// Reference lerp order (interpolators.py:127-135): x first, then y, then z.
__device__ __forceinline__ double tri(double c000, double c100, double c010, double c110,
                                      double c001, double c101, double c011, double c111,
                                      double tx, double ty, double tz) {
    double ux = 1.0 - tx, uy = 1.0 - ty, uz = 1.0 - tz;
    double c00 = c000 * ux + c100 * tx;
    double c01 = c001 * ux + c101 * tx;
    double c10 = c010 * ux + c110 * tx;
    double c11 = c011 * ux + c111 * tx;
    double c0 = c00 * uy + c10 * ty;
    double c1 = c01 * uy + c11 * ty;
    return c0 * uz + c1 * tz;
}

// Gather the 8 corners of one field (record offset `off`) of a float64 map
// and interpolate its 3 components.
__device__ __forceinline__ V3 gather_f64(const MapDev& m, const Cell& c, int off) {
    const double* base = static_cast<const double*>(m.data);
    const int S = m.stride;
    double v[8][4];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int di = (q >> 2) & 1, dj = (q >> 1) & 1, dk = q & 1;
        const int64_t node = c.base + di * m.sx + dj * m.sy + dk;
        ldg_f64x4(base + node * S + off, v[q][0], v[q][1], v[q][2], v[q][3]);
    }
    // corner q = di*4 + dj*2 + dk
    V3 o;
    o.x = tri(v[0][0], v[4][0], v[2][0], v[6][0], v[1][0], v[5][0], v[3][0], v[7][0], c.tx, c.ty, c.tz);
    o.y = tri(v[0][1], v[4][1], v[2][1], v[6][1], v[1][1], v[5][1], v[3][1], v[7][1], c.tx, c.ty, c.tz);
    o.z = tri(v[0][2], v[4][2], v[2][2], v[6][2], v[1][2], v[5][2], v[3][2], v[7][2], c.tx, c.ty, c.tz);
    return o;
}

// gather_f64 for a record stride S known at compile time.
template <int S>
__device__ __forceinline__ V3 gather_f64s(const MapDev& m, const Cell& c, int off) {
    const double* base = static_cast<const double*>(m.data);
    double v[8][4];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int di = (q >> 2) & 1, dj = (q >> 1) & 1, dk = q & 1;
        const int64_t node = c.base + di * m.sx + dj * m.sy + dk;
        ldg_f64x4(base + node * S + off, v[q][0], v[q][1], v[q][2], v[q][3]);
    }
    V3 o;
    o.x = tri(v[0][0], v[4][0], v[2][0], v[6][0], v[1][0], v[5][0], v[3][0], v[7][0], c.tx, c.ty, c.tz);
    o.y = tri(v[0][1], v[4][1], v[2][1], v[6][1], v[1][1], v[5][1], v[3][1], v[7][1], c.tx, c.ty, c.tz);
    o.z = tri(v[0][2], v[4][2], v[2][2], v[6][2], v[1][2], v[5][2], v[3][2], v[7][2], c.tx, c.ty, c.tz);
    return o;
}

__device__ __forceinline__ void ldg_f64x2(const double* p, double& a, double& b) {
    asm volatile("ld.global.nc.v2.f64 {%0,%1}, [%2];" : "=d"(a), "=d"(b) : "l"(p));
}

// The K interpolated slots of a float64 map with 1- or 2-element records.
template <int W>
__device__ __forceinline__ void gather_slots_f64(const MapDev& m, const Cell& c, double out[W]) {
    const double* base = static_cast<const double*>(m.data);
    double v[8][W];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int di = (q >> 2) & 1, dj = (q >> 1) & 1, dk = q & 1;
        const int64_t node = c.base + di * m.sx + dj * m.sy + dk;
        if constexpr (W == 2) ldg_f64x2(base + node * 2, v[q][0], v[q][1]);
        else v[q][0] = __ldg(base + node);
    }
#pragma unroll
    for (int k = 0; k < W; ++k)
        out[k] = tri(v[0][k], v[4][k], v[2][k], v[6][k], v[1][k], v[5][k], v[3][k], v[7][k], c.tx, c.ty, c.tz);
}

// Add one float64 map's E and B at a located cell; components the layout
// does not store are identically zero and are not gathered.
__device__ __forceinline__ void gather_map_f64(const MapDev& m, const Cell& c, V3& E, V3& B) {
    switch (m.layout) {
        case kLayFull:
            E = E + gather_f64(m, c, 0);
            B = B + gather_f64(m, c, m.b_off);
            break;
        case kLayE:
            E = E + gather_f64(m, c, 0);
            break;
        case kLayB:
            B = B + gather_f64(m, c, 0);
            break;
        case kLayExEyBz: {
            const V3 o = gather_f64(m, c, 0);
            E.x += o.x;
            E.y += o.y;
            B.z += o.z;
            break;
        }
        case kLayEzBz: {
            double o[2];
            gather_slots_f64<2>(m, c, o);
            E.z += o[0];
            B.z += o[1];
            break;
        }
        default: {   // kLayBz
            double o[1];
            gather_slots_f64<1>(m, c, o);
            B.z += o[0];
            break;
        }
    }
}

// E and B at r from all maps plus the constant parts (float64).  Returns the
// number of maps whose grid contained r.
__device__ __forceinline__ int eval_fields_f64(const FieldsDev& F, V3 r, V3& E, V3& B) {
    E = v3(F.e_const[0], F.e_const[1], F.e_const[2]);
    B = v3(F.b_const[0], F.b_const[1], F.b_const[2]);
    int hits = 0;
    for (int mi = 0; mi < F.n_maps; ++mi) {
        const MapDev& m = F.maps[mi];
        Cell c;
        if (!locate(m, r, c)) continue;
        ++hits;
        gather_map_f64(m, c, E, B);
    }
    return hits;
}

// launch helpers
int grid_for(int64_t n, int block);
int pick_block(int64_t n);

}  // namespace ppt
