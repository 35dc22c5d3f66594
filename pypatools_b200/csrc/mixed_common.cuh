// Helpers for the mixed-precision form.
//
// Position: an int32 cell index per axis plus a float32 offset in cell units
// on the map's uniform grid, so x = lo + (cell + offset) d.  After a step
// that may see a field the offset is in [0, 1] and IS the trilinear weight of
// the reference's interpolation (interpolators.py:109-115), so no floor or
// division happens per step; field-free Boris-family steps carry whole cells
// only every fourth global step, so between those the offset may run past 1
// (the represented position is exact either way).
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

// Advance one position axis by v * k cell units, v = (vh + vl), k = (kh + kl),
// keeping the float32 offset in [0, 1) and carrying whole cells into the index.
__device__ __forceinline__ void advance_axis(int& cell, float& f, float vh, float vl, float kh, float kl) {
    float p = vh * kh;
    float e = fmaf(vh, kh, -p);                  // exact low part of vh*kh
    float tail = fmaf(vh, kl, fmaf(vl, kh, e));
    float fn = f + p;
    fn = fn + tail;
    float c = floorf(fn);
    fn -= c;
    cell += (int)c;
    if (fn >= 1.0f) {
        fn -= 1.0f;
        cell += 1;
    }
    f = fn;
}

// In-domain test + cell/weight on one axis (the reference's x < g0 or
// x > g_last test: the last node itself is inside).
__device__ __forceinline__ bool mixed_axis(int cell, float f, int n, int& i, float& t) {
    if ((unsigned)cell <= (unsigned)(n - 2)) {
        i = cell;
        t = f;
        return true;
    }
    if (cell == n - 1 && f == 0.0f) {
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
