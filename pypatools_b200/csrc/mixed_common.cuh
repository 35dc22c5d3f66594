// Helpers for the mixed-precision form.
//
// Position: an int32 cell index per axis plus an in-cell offset in cell units
// on the map's uniform grid, held as an unevaluated float32 pair (hi + lo),
// so x = lo_grid + (cell + hi + lo) d.  After a step that may see a field the
// high word is in [0, 1] and IS the trilinear weight of the reference's
// interpolation (interpolators.py:109-115), so no floor or division happens
// per step.  Each such step adds its increment with nothing rounded away
// (add_cells_ff): the float32 sum of offset and increment would round at
// 2^-24 cells per step, and the increment's low part, which holds the fixed-
// sign float32 rounding of dt / d, would never reach the offset at all -- a
// bias of ~1e-8 of every step.  Field-free Boris-family steps advance the high
// word alone and carry whole cells only every sixteenth global step, so
// between those the high word may run past 1 (the represented position is
// exact either way).
// Velocity: an unevaluated float32 pair (hi + lo).  Per-step increments are
// computed in float32 and added with an error-free two-sum, so rounding does
// not random-walk the state at float32 precision.
#pragma once

#include "ppt_internal.cuh"

namespace ppt {

// Packed float32 pairs (sm_100 FFMA2 and the f32x2 subtract): one
// instruction issues both lanes, and each lane is rounded exactly as the
// scalar operation, so a pair computes the same bits as two scalar
// operations.  The trilinear interpolation of two record components at once
// goes through these (half the issue slots of the scalar form).
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "sub.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}

struct GridF {
    double lo[3];
    double d[3];
    double inv_d[3];
    int n[3];
};

// (a_hi, a_lo) += b, error-free (Knuth two-sum, then renormalise).
__device__ __forceinline__ void ff_add(float& hi, float& lo, float b) {
    float s = hi + b;
    float bb = s - hi;
    float err = (hi - (s - bb)) + (b - bb);
    float l = lo + err;
    float h = s + l;
    lo = l - (h - s);
    hi = h;
}

// (cell, f + fl) += p + q cells (p the leading part of the increment, q a
// correction below it): the sum f + p split exactly into its rounded value and
// error (Knuth's two-sum), the error and q into the low word fl, the pair
// renormalised, and whole cells carried out of the high word.  h - floor(h)
// rounds only for a negative h (a step backwards over a cell face), and that
// error, exact by Dekker's fast two-sum (|floor h| >= |h|), goes into fl too.
// Leaves f in [0, 1].  The caller's cell is a float (exact integers) or int.
template <typename C>
__device__ __forceinline__ void add_cells_ff(C& cell, float& f, float& fl, float p, float q, bool renorm) {
    const float s = f + p;
    const float bb = s - f;
    const float e = (f - (s - bb)) + (p - bb);
    float lo = fl + (e + q);
    float h = s;
    if (renorm) {
        h = s + lo;
        lo = lo - (h - s);
    }
    const float cc = floorf(h);
    const float t = h - cc;
    lo = lo + (h - (t + cc));
    f = t;
    fl = lo;
    cell += (C)cc;
}

// Advance one position axis by v * k cell units, v = (vh + vl), k = (kh + kl),
// on the float-float offset (add_cells_ff).  corr: a further displacement in
// cells, small against the offset (RK4's stage correction).
__device__ __forceinline__ void advance_axis(int& cell, float& f, float& fl, float vh, float vl, float kh, float kl,
                                             float corr = 0.0f) {
    const float p = vh * kh;
    const float e = fmaf(vh, kh, -p);                  // exact low part of vh*kh
    const float tail = fmaf(vh, kl, fmaf(vl, kh, e)) + corr;
    add_cells_ff(cell, f, fl, p, tail, true);
}

// In-domain test + cell/weight on one axis for the position cell + f + fl
// (f the offset's high word in [0, 1], fl its low word), with the
// reference's rule: outside when x < g0 or x > g_last, the last node itself
// inside (interpolators.py:93-97).  The faces are decided on f + fl exactly
// (fl < -f, fl > 1 - f: 1 - f is exact for f in [0.5, 1]): a decision on f
// alone errs for positions within |fl| (~1e-8 of a cell) of a face, and the
// field drops to 0 there, so such a step would be pushed differently from
// the float64 form.
__device__ __forceinline__ bool mixed_axis(int cell, float f, float fl, int n, int& i, float& t) {
    const int inner = n > 3 ? n - 3 : 0;                  // cells 1 .. n-3: no face within reach
    if ((unsigned)(cell - 1) < (unsigned)inner) {
        i = cell;
        t = f;
        return true;
    }
    if (cell == 0 || cell == n - 2) {                     // next to a face (both for n = 2)
        if ((cell == 0 && fl < -f) || (cell == n - 2 && fl > 1.0f - f)) return false;
        i = cell;
        t = f;
        return true;
    }
    if (cell == n - 1 && fl <= -f) {                      // at the last node (or a hair below it)
        i = n - 2;
        t = 1.0f;
        return true;
    }
    return false;
}

__device__ __forceinline__ float lerp_f(float a, float b, float t) { return fmaf(t, b - a, a); }

struct F3 {
    float x, y, z;
};
__device__ __forceinline__ F3 f3(float x, float y, float z) { return F3{x, y, z}; }
__device__ __forceinline__ F3 operator+(F3 a, F3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ F3 operator-(F3 a, F3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ F3 operator*(float s, F3 a) { return f3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float dotf(F3 a, F3 b) { return fmaf(a.x, b.x, fmaf(a.y, b.y, a.z * b.z)); }
__device__ __forceinline__ F3 crossf(F3 a, F3 b) {
    return f3(fmaf(a.y, b.z, -a.z * b.y), fmaf(a.z, b.x, -a.x * b.z), fmaf(a.x, b.y, -a.y * b.x));
}

}  // namespace ppt
