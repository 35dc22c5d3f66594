// Mixed-precision form of the fused push + trilinear gather.
//
// Same step structure and reference semantics as the float64 kernel
// (Boris pusher.py:124-165, Vay 'vay_rel' :216-279, RK4 :803-892, leapfrog
// :730-739, record indices :966-1007, fill 0 outside the map
// interpolators.py:93-97), with:
//   * positions as int32 cell + in-cell offset, the offset a float32 pair
//     whose high word is the trilinear weight (no per-step cell search) and
//     moves by exact quanta (add_cells_q, drift_quanta), so that a run of
//     field-free steps takes O(1) work with the bits of the steps taken one
//     by one (drift_steps, carry_periods),
//   * float32 node records (one vector load per corner), float32
//     interpolation and float32 rotation, computing the velocity INCREMENT
//     of the step, the E path's roundings kept in low words,
//   * velocity state as a float32 hi/lo pair updated by an error-free sum,
//   * float64 for the RF factor cos(omega t + phi) (a per-particle phasor
//     times a per-step table, on the FP64 pipe this kernel otherwise leaves
//     idle) and for the field time of RK4 stages.
#include <cmath>

#include "track_params.cuh"

namespace ppt {


constexpr double kTwoPi = 6.283185307179586;
constexpr double kInvTwoPi = 0.15915494309189535;

struct MixCtx {
    const TrackMixDev* P;
    double phase;            // omega t0 + phi_i
    unsigned hits;
    double c0, s0;           // cos and sin of the phase
    const double2* tab;      // (cos, sin) of g omega dt for every g of the launch, or NULL
    int64_t tab0;            // the launch's first step
};

// Per-step RF table length limit: the sorted launches of a bunch crossing
// its map are ~100 steps; longer launches compute the same values directly.
constexpr int kRfTable = 512;

// (cos, sin) of g omega dt in float64: the per-step factor of the RF phase,
// the same for every particle, so a block tabulates it once per launch.
__device__ __forceinline__ void rf_turn(int64_t g, double wdt, double& cg, double& sg) {
    sincos((double)g * wdt, &sg, &cg);
}

// (cos, sin) of g omega dt in float64
__device__ __forceinline__ double2 rf_turn2(int64_t g, double wdt) {
    double cg, sg;
    rf_turn(g, wdt, cg, sg);
    return make_double2(cg, sg);
}

// cos(omega (t0 + g dt) + phi_i) = cos a cos b - sin a sin b with a = omega
// t0 + phi_i per particle and b = g omega dt per step, in float64 (one
// product and one FMA on the FP64 pipe, which this float32 kernel leaves
// idle).  The value depends on g and the particle only, table or not, so
// tracks split into launches differently agree bit for bit.
__device__ __forceinline__ double rf_cos(const MixCtx& c, int64_t g) {
    const double2 t = c.tab != nullptr ? c.tab[(int)(g - c.tab0)] : rf_turn2(g, c.P->wdt);
    return fma(c.c0, t.x, -(c.s0 * t.y));
}

// Fill the block's RF table for steps step0 .. step0 + n - 1 (all threads
// of the block call it; n <= kRfTable).
__device__ __forceinline__ void build_rf_table(double2* tab, int64_t step0, int n, double wdt) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) tab[i] = rf_turn2(step0 + i, wdt);
    __syncthreads();
}

// 256-bit read-only load of one [E | B] node record (32-B aligned).
__device__ __forceinline__ void ldg_f32x8(const float* p, float (&v)[8]) {
    asm volatile("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]),
                   "=f"(v[7])
                 : "l"(p));
}

// One component from 8 corners (corner q = di*4 + dj*2 + dk), x first, then
// y, then z (interpolators.py:127-135), each lerp a + t (b - a).
template <typename Get>
__device__ __forceinline__ float tri8(Get get, float tx, float ty, float tz) {
    float c00 = lerp_f(get(0), get(4), tx), c01 = lerp_f(get(1), get(5), tx);
    float c10 = lerp_f(get(2), get(6), tx), c11 = lerp_f(get(3), get(7), tx);
    return lerp_f(lerp_f(c00, c10, ty), lerp_f(c01, c11, ty), tz);
}

// The same for two components at once, lane by lane (packed pairs: one
// issue slot per lerp step for both, each lane rounded as tri8 rounds).
__device__ __forceinline__ float2 lerp2(float2 a, float2 b, float2 t) { return fma2(t, sub2(b, a), a); }

__device__ __forceinline__ float2 tri8_pair(const float2 q[8], float2 tx, float2 ty, float2 tz) {
    const float2 c00 = lerp2(q[0], q[4], tx), c01 = lerp2(q[1], q[5], tx);
    const float2 c10 = lerp2(q[2], q[6], tx), c11 = lerp2(q[3], q[7], tx);
    return lerp2(lerp2(c00, c10, ty), lerp2(c01, c11, ty), tz);
}

// tri8_pair whose last (z) level is split exactly: the result as (head,
// tail) per lane.  The x and y levels round as in tri8_pair; the z level --
// head = c0 + t (c1 - c0) -- rounds at half an ulp of the field, which for a
// map that varies along z is the largest rounding of the interpolation and
// reaches every velocity through the kick, so it is kept: t (c1 - c0) split
// by an FMA, the sum by Knuth's two-sum.
__device__ __forceinline__ float2 tri8_pair_ff(const float2 q[8], float2 tx, float2 ty, float2 tz, float2& lo) {
    const float2 c00 = lerp2(q[0], q[4], tx), c01 = lerp2(q[1], q[5], tx);
    const float2 c10 = lerp2(q[2], q[6], tx), c11 = lerp2(q[3], q[7], tx);
    const float2 c0 = lerp2(c00, c10, ty), c1 = lerp2(c01, c11, ty);
    const float2 d = sub2(c1, c0);
    const float2 p = __fmul2_rn(tz, d);
    const float2 pe = fma2(tz, d, make_float2(-p.x, -p.y));
    const float2 h = __fadd2_rn(c0, p);
    const float2 bb = sub2(h, c0);
    const float2 e = __fadd2_rn(sub2(c0, sub2(h, bb)), sub2(p, bb));
    lo = __fadd2_rn(e, pe);
    return h;
}

// Trilinear E/B at (cell, offset) from the float32 map of record layout L;
// returns false when outside.  Components L does not store are compile-time
// zeros, so the arithmetic that would multiply them vanishes from the
// kernel.  Only the six-component layout carries the constant field parts
// (the host creates that layout whenever they are not zero).
// El: the low parts of E's components (tri8_pair_ff).
// fl: the offset's low words (zeros where only the high words are known).
template <int L>
__device__ __forceinline__ void gather_cell(const TrackMixDev& P, int i, int j, int k, float tx, float ty, float tz,
                                            F3& E, F3& B, F3& El);

template <int L>
__device__ __forceinline__ void field_init(const TrackMixDev& P, F3& E, F3& B, F3& El) {
    El = f3(0.0f, 0.0f, 0.0f);
    if constexpr (L == kLayFull) {
        E = f3(P.e_const[0], P.e_const[1], P.e_const[2]);
        B = f3(P.b_const[0], P.b_const[1], P.b_const[2]);
    } else {
        E = f3(0.0f, 0.0f, 0.0f);
        B = f3(0.0f, 0.0f, 0.0f);
    }
}

template <int L>
__device__ __forceinline__ bool gather_mixed(const TrackMixDev& P, const int cell[3], const float f[3],
                                             const float fl[3], F3& E, F3& B, F3& El) {
    field_init<L>(P, E, B, El);
    int i, j, k;
    float tx, ty, tz;
    if (!mixed_axis(cell[0], f[0], fl[0], P.G.n[0], i, tx)) return false;
    if (!mixed_axis(cell[1], f[1], fl[1], P.G.n[1], j, ty)) return false;
    if (!mixed_axis(cell[2], f[2], fl[2], P.G.n[2], k, tz)) return false;
    gather_cell<L>(P, i, j, k, tx, ty, tz, E, B, El);
    return true;
}

// The trilinear fields of cell (i, j, k) at weights (tx, ty, tz), added to
// the E, B field_init set.
template <int L>
__device__ __forceinline__ void gather_cell(const TrackMixDev& P, int i, int j, int k, float tx, float ty, float tz,
                                            F3& E, F3& B, F3& El) {
    const MapDev& m = P.map;
    const float2 tx2 = make_float2(tx, tx), ty2 = make_float2(ty, ty), tz2 = make_float2(tz, tz);
    constexpr int W = layout_width(L);
    // corner (di, dj) = (0,0) (0,1) (1,0) (1,1); the k+1 corner is the next
    // record; 32-bit offsets when the map's elements allow (maps below 2^31
    // that vary along z: a map constant along z takes the 64-bit path, whose
    // z stride k_elems is 0 for it, so the common path keeps k * W)
    const float* p00;
    const float* p10;
    const float* p01;
    if (m.idx32) {
        const int sx = (int)m.sx * W, sy = (int)m.sy * W;
        p00 = static_cast<const float*>(m.data) + (i * sx + j * sy + k * W);
        p10 = p00 + sx;
        p01 = p00 + sy;
    } else {
        const int64_t off = ((int64_t)i * m.sx + (int64_t)j * m.sy) * W + (int64_t)k * P.k_elems;
        p00 = static_cast<const float*>(m.data) + off;
        p10 = p00 + m.sx * W;
        p01 = p00 + m.sy * W;
    }
    const float* p11 = p01 + (p10 - p00);
    const float* pc[4] = {p00, p01, p10, p11};
    // Components adjacent in the record are interpolated as packed pairs
    // (tri8_pair); a lone component takes tri8, the same operations.
    if constexpr (L == kLayFull) {
        // [Ex Ey Ez 0 | Bx By Bz 0]: one 256-bit load per corner, four pairs
        float q[8][8];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            ldg_f32x8(pc[c], q[2 * c]);
            ldg_f32x8(pc[c] + 8, q[2 * c + 1]);
        }
        float2 o[4], ol[2];
#pragma unroll
        for (int h = 0; h < 4; ++h) {
            float2 qp[8];
#pragma unroll
            for (int c = 0; c < 8; ++c) qp[c] = make_float2(q[c][2 * h], q[c][2 * h + 1]);
            if (h < 2) o[h] = tri8_pair_ff(qp, tx2, ty2, tz2, ol[h]);
            else o[h] = tri8_pair(qp, tx2, ty2, tz2);
        }
        E = E + f3(o[0].x, o[0].y, o[1].x);
        El = f3(ol[0].x, ol[0].y, ol[1].x);
        B = B + f3(o[2].x, o[2].y, o[3].x);
    } else if constexpr (W == 4) {
        // three packed components and a pad: one 128-bit load per corner, two pairs
        float4 q[8];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            q[2 * c] = __ldg(reinterpret_cast<const float4*>(pc[c]));
            q[2 * c + 1] = __ldg(reinterpret_cast<const float4*>(pc[c] + 4));
        }
        float2 qa[8], qb[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            qa[c] = make_float2(q[c].x, q[c].y);
            qb[c] = make_float2(q[c].z, q[c].w);
        }
        if constexpr (L == kLayE) {
            float2 la, lb;
            const float2 oa = tri8_pair_ff(qa, tx2, ty2, tz2, la), ob = tri8_pair_ff(qb, tx2, ty2, tz2, lb);
            E = f3(oa.x, oa.y, ob.x);
            El = f3(la.x, la.y, lb.x);
        } else if constexpr (L == kLayB) {
            const float2 oa = tri8_pair(qa, tx2, ty2, tz2), ob = tri8_pair(qb, tx2, ty2, tz2);
            B = f3(oa.x, oa.y, ob.x);
        } else {   // kLayExEyBz
            float2 la;
            const float2 oa = tri8_pair_ff(qa, tx2, ty2, tz2, la), ob = tri8_pair(qb, tx2, ty2, tz2);
            E = f3(oa.x, oa.y, 0.0f);
            El = f3(la.x, la.y, 0.0f);
            B = f3(0.0f, 0.0f, ob.x);
        }
    } else if constexpr (W == 2) {
        // kLayEzBz: one 64-bit load per corner, one pair
        float2 q[8];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            q[2 * c] = __ldg(reinterpret_cast<const float2*>(pc[c]));
            q[2 * c + 1] = __ldg(reinterpret_cast<const float2*>(pc[c] + 2));
        }
        float2 ol;
        const float2 o = tri8_pair_ff(q, tx2, ty2, tz2, ol);
        E = f3(0.0f, 0.0f, o.x);
        El = f3(0.0f, 0.0f, ol.x);
        B = f3(0.0f, 0.0f, o.y);
    } else {
        // kLayBz: one 32-bit load per corner
        float q[8];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            q[2 * c] = __ldg(pc[c]);
            q[2 * c + 1] = __ldg(pc[c] + 1);
        }
        B = f3(0.0f, 0.0f, tri8([&](int c) { return q[c]; }, tx, ty, tz));
    }
}

// Constant field parts exist only with the six-component layout.
template <int L>
__device__ __forceinline__ bool const_fields(const TrackMixDev& P) {
    if constexpr (L == kLayFull) return P.const_nz != 0;
    else return false;
}

// Fields at the step's field time t0 + g dt (+ toff for RK4 stages); the
// float64 time and phase are formed only when E is non-zero.
// (head, tail) of cf (eh + el), formed in float64 and split
__device__ __forceinline__ void mul_pair(double cf, float& eh, float& el) {
    const double e = fma((double)el, cf, (double)eh * cf);
    eh = (float)e;
    el = (float)(e - (double)eh);
}

// El: the low parts of E's components (the interpolation's last level and,
// with RF, the factor's and the product's), for the Boris kick correction.
template <bool RF, int L>
__device__ __forceinline__ void rf_modulate(MixCtx& c, int64_t g, double toff, F3& E, F3& El);

template <bool RF, int L>
__device__ __forceinline__ bool fields_mixed(MixCtx& c, const int cell[3], const float f[3], const float fl[3],
                                             int64_t g, double toff, F3& E, F3& B, F3& El) {
    bool in = gather_mixed<L>(*c.P, cell, f, fl, E, B, El);
    c.hits += in;
    rf_modulate<RF, L>(c, g, toff, E, El);
    return in || const_fields<L>(*c.P);
}

// E times the RF factor at the step's field time t0 + g dt (+ toff), the
// products' roundings into El; the float64 time and phase are formed only
// when E is non-zero.
template <bool RF, int L>
__device__ __forceinline__ void rf_modulate(MixCtx& c, int64_t g, double toff, F3& E, F3& El) {
    if (RF) {
        constexpr int EM = e_bits(L);
        if ((bit(EM, 0) && E.x != 0.0f) || (bit(EM, 1) && E.y != 0.0f) || (bit(EM, 2) && E.z != 0.0f)) {
            // omega (t0 + g dt + toff) + phi_i = (omega t0 + phi_i) + g (omega dt) + omega toff, in float64
            double cf;
            if (toff == 0.0) {
                cf = rf_cos(c, g);
            } else {
                // RK4 stage times t + dt/2, t + dt: the phase reduced to
                // [-pi, pi] in float64, then cosf (the hardware __cosf,
                // absolute error 2^-21.4, doubled the error tail)
                double ph = fma((double)g, c.P->wdt, c.phase);
                ph = fma(c.P->omega, toff, ph);
                const double red = fma(-rint(ph * kInvTwoPi), kTwoPi, ph);
                cf = (double)cosf((float)red);
            }
            if constexpr (bit(EM, 0)) mul_pair(cf, E.x, El.x);
            if constexpr (bit(EM, 1)) mul_pair(cf, E.y, El.y);
            if constexpr (bit(EM, 2)) mul_pair(cf, E.z, El.z);
        }
    }
}

// The same without the low parts (the pushers other than the Boris family's).
template <bool RF, int L>
__device__ __forceinline__ bool fields_mixed(MixCtx& c, const int cell[3], const float f[3], const float fl[3],
                                             int64_t g, double toff, F3& E, F3& B) {
    F3 El;
    return fields_mixed<RF, L>(c, cell, f, fl, g, toff, E, B, El);
}


// Boris velocity increment in float32 (pusher.py:149-163 rearranged):
// v_new - v = 2 a + (v- + v- x t) x s,  a = (q/m) E dt/2,  v- = v + a,
// t = (q/m) B dt/2, s = 2 t / (1 + t.t), with the components outside EM
// (E) and BM (B) left out; the components of the result outside
// EM | cross_bits(BM) are zero.
template <int QM, int I>
__device__ __forceinline__ float cross_m(const float p[3], const float q[3]) {
    // (p x q)_I without q's zero components (crossf's form when both terms are there)
    constexpr int J = (I + 1) % 3, K = (I + 2) % 3;
    if constexpr (bit(QM, K) && bit(QM, J)) return fmaf(p[J], q[K], -p[K] * q[J]);
    else if constexpr (bit(QM, K)) return p[J] * q[K];
    else if constexpr (bit(QM, J)) return -(p[K] * q[J]);
    else return 0.0f;
}

template <int M>
__device__ __forceinline__ float self_dot_m(const float t[3]) {
    // dotf(t, t) without the zero components (z, then y, then x)
    float acc = 0.0f;
    if constexpr (bit(M, 2)) acc = t[2] * t[2];
    if constexpr (bit(M, 1)) acc = bit(M, 2) ? fmaf(t[1], t[1], acc) : t[1] * t[1];
    if constexpr (bit(M, 0)) acc = (bit(M, 1) || bit(M, 2)) ? fmaf(t[0], t[0], acc) : t[0] * t[0];
    return acc;
}

template <int EM, int BM>
__device__ __forceinline__ F3 boris_dv_m(F3 vv, F3 E, F3 B, float hqdt) {
    constexpr int CM = cross_bits(BM);
    const float v[3] = {vv.x, vv.y, vv.z}, e[3] = {E.x, E.y, E.z}, b[3] = {B.x, B.y, B.z};
    float a[3], vm[3], t[3], s[3], vp[3], dv[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        a[i] = bit(EM, i) ? hqdt * e[i] : 0.0f;
        vm[i] = bit(EM, i) ? v[i] + a[i] : v[i];
        t[i] = bit(BM, i) ? hqdt * b[i] : 0.0f;
    }
    const float s_f = __fdividef(2.0f, 1.0f + self_dot_m<BM>(t));
#pragma unroll
    for (int i = 0; i < 3; ++i) s[i] = bit(BM, i) ? s_f * t[i] : 0.0f;
    vp[0] = bit(CM, 0) ? vm[0] + cross_m<BM, 0>(vm, t) : vm[0];
    vp[1] = bit(CM, 1) ? vm[1] + cross_m<BM, 1>(vm, t) : vm[1];
    vp[2] = bit(CM, 2) ? vm[2] + cross_m<BM, 2>(vm, t) : vm[2];
    const float c2[3] = {cross_m<BM, 0>(vp, s), cross_m<BM, 1>(vp, s), cross_m<BM, 2>(vp, s)};
#pragma unroll
    for (int i = 0; i < 3; ++i)
        dv[i] = bit(EM, i) ? (bit(CM, i) ? fmaf(2.0f, a[i], c2[i]) : 2.0f * a[i]) : (bit(CM, i) ? c2[i] : 0.0f);
    return f3(dv[0], dv[1], dv[2]);
}

template <int L>
__device__ __forceinline__ F3 boris_dv(F3 v, F3 E, F3 B, float hqdt) {
    return boris_dv_m<e_bits(L), b_bits(L)>(v, E, B, hqdt);
}

constexpr float kCf = 299792458.0f;

__device__ __forceinline__ float rel_gamma_f(F3 v) {
    float bsq = dotf(v, v) * (1.0f / (kCf * kCf));
    bsq = bsq >= 0.9999f ? 0.9999f : bsq;
    return rsqrtf(1.0f - bsq);
}

__device__ __forceinline__ F3 lorentz_f(F3 v, F3 E, F3 B, float qm) { return qm * (E + crossf(v, B)); }

__device__ __forceinline__ F3 rk4_rel_deriv_f(F3 v, F3 E, F3 B, float qm) {
    float g = rel_gamma_f(v);
    F3 F = qm * (E + crossf(v, B));
    float ig = 1.0f / g;
    float k = dotf(v, F) * ig * (1.0f / (kCf * kCf));
    return f3(fmaf(F.x, ig, -k * v.x), fmaf(F.y, ig, -k * v.y), fmaf(F.z, ig, -k * v.z));
}

// pusher.py:216-279 in float32; returns the new velocity (not an increment).
__device__ __forceinline__ F3 vay_rel_f(F3 v, F3 E, F3 B, float qm, float dt) {
    float g = rel_gamma_f(v);
    F3 u = g * v;
    F3 tau = (0.5f * qm * dt) * B;
    F3 up = u + (qm * dt) * E;
    float upm2 = dotf(up, up);
    float tau2 = dotf(tau, tau);
    float udt = dotf(up, tau);
    float gis = 1.0f - upm2 * (1.0f / (kCf * kCf));
    gis = gis < 1e-10f ? 1e-10f : gis;
    float sigma = gis - tau2;
    float q = udt * (1.0f / kCf);
    float gn = sqrtf(0.5f * (sigma + sqrtf(fmaf(sigma, sigma, 4.0f * (tau2 + q * q)))));
    float ig = 1.0f / gn;
    F3 t = ig * tau;
    float sf = 2.0f / (1.0f + tau2 * ig * ig);
    F3 s = sf * t;
    F3 us = up + crossf(up, t);
    F3 un = up + crossf(us, s);
    F3 vn = ig * un;
    float vm = sqrtf(dotf(vn, vn));
    if (vm >= 0.9999f * kCf) vn = ((0.9999f * kCf) / vm) * vn;
    return vn;
}

__device__ __forceinline__ void vel_add(float vh[3], float vl[3], F3 d) {
    ff_add(vh[0], vl[0], d.x);
    ff_add(vh[1], vl[1], d.y);
    ff_add(vh[2], vl[2], d.z);
}

// A Boris increment d, scaled by (1 + ws) into the float-float velocity.
// hqdt = q/m dt/2 rounded to float32 carries one fixed relative error ws
// (2.6e-8 for 5 MeV protons at dt = 1e-10 s) into a and t on every step: a
// bias of the rotation angle that grows with the number of turns, where the
// other roundings vary from step to step.  d (1 + ws) is exact for the 2a
// part and for the rotation to first order (the neglected part is ~ t^2 of
// the correction); d ws is below half an ulp of d, so it goes into the low
// word, and costs three FMAs off the step's critical path.
// (Components outside the mask M stay unchanged: d is zero there.)
template <int M>
__device__ __forceinline__ void vel_add_boris(float vh[3], float vl[3], F3 d, float ws) {
    const float dd[3] = {d.x, d.y, d.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (!bit(M, a)) continue;
        ff_add(vh[a], vl[a], dd[a]);
        vl[a] = fmaf(dd[a], ws, vl[a]);
    }
}

// The same for the Boris steps of a track, at a third of the cost: a fast
// two-sum (exact when |vh| >= |d|, which holds but for a component passing
// through zero, where its error stays below an ulp of d) whose rounding
// error, and the correction d ws, go into the low word without renormalising
// the pair.  vel_renorm renormalises it after global steps g with
// (g + 1) % 4 == 0 that see a field, so the low word stays within a few ulps
// of the high one and a track's bits do not depend on how it is split into
// launches.  vh + vl stays the accumulated velocity throughout.
template <int M>
__device__ __forceinline__ void vel_add_fast(float vh[3], float vl[3], F3 d, float ws) {
    const float dd[3] = {d.x, d.y, d.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (!bit(M, a)) continue;
        const float s = vh[a] + dd[a];
        const float err = dd[a] - (s - vh[a]);
        vl[a] = fmaf(dd[a], ws, vl[a] + err);
        vh[a] = s;
    }
}

// The E kick's low-word correction: 2 ((q/m) dt/2 E exactly - its float32
// product) for the components of EM, from E's low parts El (fields_mixed).
template <int EM>
__device__ __forceinline__ F3 kick_correction(F3 E, F3 El, float hqdt) {
    const float e[3] = {E.x, E.y, E.z}, el[3] = {El.x, El.y, El.z};
    float k[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        if (bit(EM, i)) {
            const float a = hqdt * e[i];
            k[i] = 2.0f * (fmaf(hqdt, e[i], -a) + hqdt * el[i]);
        } else {
            k[i] = 0.0f;
        }
    }
    return f3(k[0], k[1], k[2]);
}

// vel_add_fast with the kick correction kc added to the low word.
template <int M>
__device__ __forceinline__ void vel_add_fast_kc(float vh[3], float vl[3], F3 d, float ws, F3 kc) {
    const float dd[3] = {d.x, d.y, d.z}, kk[3] = {kc.x, kc.y, kc.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (!bit(M, a)) continue;
        const float s = vh[a] + dd[a];
        const float err = dd[a] - (s - vh[a]);
        vl[a] = fmaf(dd[a], ws, (vl[a] + err) + kk[a]);
        vh[a] = s;
    }
}

template <int M>
__device__ __forceinline__ void vel_renorm(float vh[3], float vl[3]) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (!bit(M, a)) continue;
        const float s = vh[a] + vl[a];
        vl[a] = vl[a] - (s - vh[a]);
        vh[a] = s;
    }
}

__device__ __forceinline__ void vel_set(float vh[3], float vl[3], F3 v) {
    // replace the state by a float32 value (clamped / recomputed velocity)
    vh[0] = v.x; vh[1] = v.y; vh[2] = v.z;
    vl[0] = vl[1] = vl[2] = 0.0f;
}

// Per-step position increment v dt / d in cell units, recomputed only when
// the velocity changes, as (q, r): q = the increment rounded to a multiple
// of 2^-22 cells, r the rest (v = vh + vl, dt / d = kh + kl; r is formed from
// the exact residual of vh kh - q by an FMA).  The offset's high word is a
// multiple of 2^-22 in [0, 1] in a map, so hi + q is exact there for steps
// below three cells (|hi + q| < 4: add_cells_q).
__device__ __forceinline__ void split_q(float p, float vh, float vl, float kh, float kl, float& q, float& r) {
    q = rintf(p * 0x1p22f) * 0x1p-22f;
    r = fmaf(vh, kh, -q) + fmaf(vh, kl, vl * kh);
}

// ---------------------------------------------------------------------------
// u-state Boris family of the mixed form: relativistic Boris and Vay (2008)
// on u = gamma v (the float64 form's boris_rel_u / vay_u).  The increment of
// u is formed in float32 as for the Boris above; gamma enters through its
// reciprocal as a float pair (ih + il) good to ~1e-14, because a float32
// gamma would round the same way at every step of a gyration (|u| constant):
// a fixed bias of the rotation angle and of the speed.  The rotation part of
// an increment is scaled by (1 + il / ih), like the (1 + ws) scaling of the
// float32 q dt / 2m, through the velocity's low word.
// ---------------------------------------------------------------------------
constexpr float kInvC2f = 1.1126500560536184e-17f;   // 1 / c^2 [s^2/m^2]

// u.u / c^2 of the float32 head of u (its rounding varies from step to step)
__device__ __forceinline__ float u2_over_c2(const float u[3]) {
    return fmaf(u[0], u[0], fmaf(u[1], u[1], u[2] * u[2])) * kInvC2f;
}

// 1 / sqrt(gh + gl) as a float pair: an rsqrt estimate and one Newton step
// whose residual 1 - g i0^2 is formed from exact products (m is within a few
// ulps of 1, so 1 - m is exact).
__device__ __forceinline__ void inv_sqrt_pair(float gh, float gl, float& ih, float& il) {
    const float i0 = rsqrtf(gh);
    const float p = i0 * i0, pe = fmaf(i0, i0, -p);
    const float m = gh * p, me = fmaf(gh, p, -m);
    const float r = ((1.0f - m) - me) - fmaf(gh, pe, gl * p);
    ih = i0;
    il = 0.5f * i0 * r;
}

// 1 / gamma = 1 / sqrt(1 + x), with 1 + x split exactly (Knuth's two-sum):
// for the small x of ions 1 + x alone would round identically at every step.
__device__ __forceinline__ void inv_gamma_pair(float x, float& ih, float& il) {
    const float gh = 1.0f + x;
    const float bb = gh - 1.0f;
    const float gl = (1.0f - (gh - bb)) + (x - bb);
    inv_sqrt_pair(gh, gl, ih, il);
}

// Relativistic Boris increment of u (boris_rel_u in the float64 form):
// a = (q/m) E dt/2, u- = u + a, t = (q/m) B dt/2 / gamma(u-), s = 2 t / (1 + t.t),
// du = 2 a + (u- + u- x t) x s; corr: the low-word correction of du
// (ws for the float32 q dt / 2m, il / ih for gamma's low part, rotation only).
template <int EM, int BM>
__device__ __forceinline__ void boris_rel_du(const float u[3], F3 E, F3 B, float hqdt, float ws, float du[3],
                                             float corr[3]) {
    constexpr int CM = cross_bits(BM);
    const float e[3] = {E.x, E.y, E.z}, b[3] = {B.x, B.y, B.z};
    float a[3], um[3], t[3], sv[3], up[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        a[i] = bit(EM, i) ? hqdt * e[i] : 0.0f;
        um[i] = bit(EM, i) ? u[i] + a[i] : u[i];
    }
    float ih, il;
    inv_gamma_pair(u2_over_c2(um), ih, il);
    const float th = hqdt * ih;
#pragma unroll
    for (int i = 0; i < 3; ++i) t[i] = bit(BM, i) ? th * b[i] : 0.0f;
    float tt = 0.0f;
#pragma unroll
    for (int i = 0; i < 3; ++i)
        if (bit(BM, i)) tt = fmaf(t[i], t[i], tt);
    const float sf = __fdividef(2.0f, 1.0f + tt);
#pragma unroll
    for (int i = 0; i < 3; ++i) sv[i] = bit(BM, i) ? sf * t[i] : 0.0f;
    up[0] = bit(CM, 0) ? um[0] + cross_m<BM, 0>(um, t) : um[0];
    up[1] = bit(CM, 1) ? um[1] + cross_m<BM, 1>(um, t) : um[1];
    up[2] = bit(CM, 2) ? um[2] + cross_m<BM, 2>(um, t) : um[2];
    const float rot[3] = {cross_m<BM, 0>(up, sv), cross_m<BM, 1>(up, sv), cross_m<BM, 2>(up, sv)};
    const float wr = ws + __fdividef(il, ih);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float kick = bit(EM, i) ? 2.0f * a[i] : 0.0f;
        const float r = bit(CM, i) ? rot[i] : 0.0f;
        du[i] = kick + r;
        corr[i] = fmaf(r, wr, kick * ws);
    }
}

// Vay (2008) increment of u (vay_u in the float64 form):
// u' = u + (q/m) dt (E + v x B / 2) with v = u / gamma(u); tau = (q/m) B dt/2;
// gamma_new^2 = G = (sigma + sqrt(sigma^2 + 4 (tau^2 + (u'.tau / c)^2))) / 2,
// sigma = 1 + u'^2/c^2 - tau^2 (both as float pairs); t = tau / gamma_new,
// s = 1 / (1 + t^2); u_new = s (u' + (u'.t) t + u' x t), written as the
// increment du = (u' - u) + s ((u'.t) t + u' x t - t^2 u').
template <int EM, int BM>
__device__ __forceinline__ void vay_du(const float u[3], F3 E, F3 B, float hqdt, float ws, float du[3],
                                       float corr[3]) {
    const float e[3] = {E.x, E.y, E.z}, b[3] = {B.x, B.y, B.z};
    float ih, il;
    inv_gamma_pair(u2_over_c2(u), ih, il);
    const float v[3] = {u[0] * ih, u[1] * ih, u[2] * ih};
    const float vxb[3] = {cross_m<BM, 0>(v, b), cross_m<BM, 1>(v, b), cross_m<BM, 2>(v, b)};
    float d1[3], up[3], tau[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        // (q/m) dt (E + v x B / 2) = 2 hqdt E + hqdt (v x B)
        const float ke = bit(EM, i) ? 2.0f * hqdt * e[i] : 0.0f;
        const float kb = hqdt * vxb[i];
        d1[i] = ke + kb;
        up[i] = u[i] + d1[i];
        tau[i] = bit(BM, i) ? hqdt * b[i] : 0.0f;
        corr[i] = fmaf(kb, __fdividef(il, ih), d1[i] * ws);
    }
    float tau2 = 0.0f, ut = 0.0f;
#pragma unroll
    for (int i = 0; i < 3; ++i)
        if (bit(BM, i)) {
            tau2 = fmaf(tau[i], tau[i], tau2);
            ut = fmaf(up[i], tau[i], ut);
        }
    const float us = ut * (1.0f / kCf);
    const float w = fmaf(us, us, tau2);                      // tau^2 + u*^2
    // sigma = 1 + x' - tau^2 as a pair
    const float x = u2_over_c2(up);
    const float sh0 = 1.0f + x, bb = sh0 - 1.0f;
    const float sl0 = (1.0f - (sh0 - bb)) + (x - bb);
    const float sh = sh0 - tau2;                             // tau^2 << 1: exact to the pair
    const float sl = sl0 - ((sh - sh0) + tau2);
    // D = sigma^2 + 4 w as a pair, sqrt(D) as a pair
    const float d0 = sh * sh, d0e = fmaf(sh, sh, -d0);
    const float dh = fmaf(4.0f, w, d0);
    const float dl = ((d0 - dh) + 4.0f * w) + fmaf(2.0f * sh, sl, d0e);
    const float rd = sqrtf(dh);
    const float rr = rd * rd, rre = fmaf(rd, rd, -rr);
    const float rdl = __fdividef(((dh - rr) - rre) + dl, 2.0f * rd);
    // G = (sigma + sqrt D) / 2, then 1 / gamma_new = 1 / sqrt(G)
    const float gh = 0.5f * (sh + rd);
    const float gl = 0.5f * (((sh - 2.0f * gh) + rd) + (sl + rdl));
    float jh, jl;
    inv_sqrt_pair(gh, gl, jh, jl);
    float t[3];
    float tt = 0.0f, upt = 0.0f;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        t[i] = bit(BM, i) ? tau[i] * jh : 0.0f;
        if (bit(BM, i)) {
            tt = fmaf(t[i], t[i], tt);
            upt = fmaf(up[i], t[i], upt);
        }
    }
    const float sf = __fdividef(1.0f, 1.0f + tt);
    const float wr = ws + __fdividef(jl, jh);
    const float uxt[3] = {cross_m<BM, 0>(up, t), cross_m<BM, 1>(up, t), cross_m<BM, 2>(up, t)};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float rot = sf * (fmaf(upt, t[i], uxt[i]) - tt * up[i]);
        du[i] = d1[i] + rot;
        corr[i] = fmaf(rot, wr, corr[i]);
    }
}

// u += du with its correction: a fast two-sum into the low word, renormalised
// with the other Boris steps after global steps g with (g + 1) % 4 == 0.
__device__ __forceinline__ void vel_add_corr(float vh[3], float vl[3], const float du[3], const float corr[3]) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float s = vh[a] + du[a];
        const float err = du[a] - (s - vh[a]);
        vl[a] = (vl[a] + err) + corr[a];
        vh[a] = s;
    }
}

// Position increment (dh + dl) = (u / gamma(u)) dt / d of the u state, with
// 1 / gamma as a pair and the products split exactly.
__device__ __forceinline__ void increment_u(const TrackMixDev& P, const float uh[3], const float ul[3], float dh[3],
                                            float dl[3]) {
    float ih, il;
    inv_gamma_pair(u2_over_c2(uh), ih, il);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float p = uh[a] * ih;
        const float pe = fmaf(uh[a], ih, -p);
        const float pl = fmaf(uh[a], il, fmaf(ul[a], ih, pe));   // v = p + pl
        split_q(p * P.kh[a], p, pl, P.kh[a], P.kl[a], dh[a], dl[a]);
    }
}

__device__ __forceinline__ void advance(const TrackMixDev& P, int cell[3], float f[3], float fl[3], const float vh[3],
                                        const float vl[3]) {
#pragma unroll
    for (int a = 0; a < 3; ++a) advance_axis(cell[a], f[a], fl[a], vh[a], vl[a], P.kh[a], P.kl[a]);
}

// Cell + offset of the point (cell, f) + d (d in metres), for RK4 stages.
__device__ __forceinline__ void offset_point(const TrackMixDev& P, const int cell[3], const float f[3], F3 d,
                                             int oc[3], float of[3]) {
    const float dd[3] = {d.x, d.y, d.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float g = fmaf(dd[a], P.inv_d[a], f[a]);
        float c = floorf(g);
        of[a] = g - c;
        oc[a] = cell[a] + (int)c;
        if (of[a] >= 1.0f) { of[a] -= 1.0f; oc[a] += 1; }
    }
}

template <int M = 7>
__device__ __forceinline__ void increment(const TrackMixDev& P, const float vh[3], const float vl[3], float dh[3],
                                          float dl[3]) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (!bit(M, a)) continue;
        split_q(vh[a] * P.kh[a], vh[a], vl[a], P.kh[a], P.kl[a], dh[a], dl[a]);
    }
}

// (cell, hi + lo) += q + r cells for the Boris family's steps that may see a
// field: hi + q exact (both multiples of 2^-22 and |hi + q| < 4), r into lo;
// with `fold` (after global steps g with (g + 1) % 4 == 0) lo's whole
// multiples of 2^-22 move into hi (exact), so hi stays within ~2^-23 of the
// position (the faces are decided on hi + lo: mixed_axis); whole cells out of
// hi (exact).  Leaves hi in [0, 1).
__device__ __forceinline__ void add_cells_q(float& cell, float& hi, float& lo, float q, float r, bool fold) {
    float h = hi + q;
    lo += r;
    if (fold) {
        const float qq = rintf(lo * 0x1p22f) * 0x1p-22f;
        h += qq;
        lo -= qq;
    }
    const float cc = floorf(h);
    hi = h - cc;
    cell += cc;
}

// Per-particle loop state of the Boris family: the position increment, the
// (q, r) pair of increment() / increment_u().
struct Drift {
    float dh[3];
    float dl[3];
};

// Field-free steps of the Boris family (Boris, leapfrog).  Outside the map
// with no constant field both updates leave v exactly unchanged (every added
// term is zero), so such a step is the position advance alone.  The offset
// is a (hi, lo) pair per axis; a field-free step adds the drift quanta (q, r)
// of the increment (drift_quanta) to it, and hi + q is exact, so the drift
// does not round the position step after step (and drift_steps takes a run
// of such steps as one multiply-add).  The
// whole-cell carry is taken after global steps g with (g + 1) % kCarry == 0
// only; in between hi runs up to 1 + kCarry |dh| cells.  Because the carry
// points depend on the global step index alone, a track gives the same bits
// however its steps are split into launches, runs or serving ticks.
// Normalising a non-negative hi (cf + floor hi, hi - floor hi) is exact, and
// so is it for a negative hi that is a multiple of the quantum.
constexpr int kCarry = 32;
constexpr unsigned kCarryMask = kCarry - 1;

// The increment (dh + dl) of field-free steps as q + r: q the increment
// rounded to a multiple of u, the float32 spacing at the largest |hi| a carry
// period reaches (|hi| < 2 + kCarry |dh|); r = (dh - q) + dl the rest,
// rounded to a multiple of u 2^-19.  Once hi is a multiple of u (after at
// most a few roundings at the start of a drift), hi + q is exact; and the low
// word, a multiple of u 2^-19 below 32 u (after a carry it lies in [0, u),
// and a period adds at most kCarry |r| <= 16.5 u), changes by exact additions
// only, so
// whether r is added at every step or kCarry r at a carry point gives the
// same bits.  Without the split, the float32 sum hi + dh rounds dh to the
// spacing of hi's binade, the same amount every step: a fixed-sign error of
// up to 2^-23 cells per step; the rounding of r costs at most u 2^-20 per
// step (1e-12 of a cell for the RF-gap protons).  U[a] = (u, 1 / u) per axis,
// for the carries.
__device__ __forceinline__ void drift_quanta(const Drift& d, float2 Q[3], float2 U[3]) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float bound = fmaf((float)kCarry, fabsf(d.dh[a]), 2.0f);
        // bound in [2^(eb-127), 2^(eb-126)); held to u <= 1 cell (carry_periods'
        // shifts), which only increments of 2^19 cells per step and more reach:
        // those leave the 2^24-cell range within a carry period, where the
        // launch's range check flags them
        const int eb = min((__float_as_int(bound) >> 23) & 0xff, 150);
        const float u = __int_as_float((eb - 23) << 23);        // float32 spacing below 2^(eb-126)
        const float ui = __int_as_float((277 - eb) << 23);      // 1 / u (both powers of two)
        const float q = rintf(d.dh[a] * ui) * u;
        const float r = (d.dh[a] - q) + d.dl[a];
        const float w = __int_as_float((eb - 42) << 23);        // u 2^-19
        const float wi = __int_as_float((296 - eb) << 23);      // 1 / w
        Q[a] = make_float2(q, rintf(r * wi) * w);
        U[a] = make_float2(u, ui);
    }
}

// The carry of field-free steps: whole cells out of the high word, and the
// whole quanta the low word has gathered (N r after N steps) into it, which
// leaves the low word in [0, u), so the high word -- which the cell pre-test
// and the trilinear weight read -- stays within u of the position.  Both
// moves are exact.
__device__ __forceinline__ void carry(float cf[3], float2 o[3], const float2 U[3]) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float cc = floorf(o[a].x);
        o[a].x -= cc;
        cf[a] += cc;
        const float qq = floorf(o[a].y * U[a].y) * U[a].x;
        o[a].x += qq;
        o[a].y -= qq;
    }
}

// N whole carry periods (kCarry steps, then the carry) from a carry point,
// in closed form.  In units of w = u 2^-19 the low word is an integer L and a
// period's kCarry r an integer R; a carry moves floor((L + R) / 2^19) quanta u
// into the high word and leaves (L + R) mod 2^19, so after N periods the low
// word is (L0 + N R) mod 2^19 and the quanta moved sum to
// floor((L0 + N R) / 2^19).  In units of u (u = 2^-sh) the high word H gains
// kCarry q / u and the moved quanta each period, and each carry takes the
// whole cells out of it; so after the last carry the cells moved out are
// floor((A - Kp) / 2^sh), with A the high word's total and Kp the last
// period's quanta, and the high word keeps the rest of A.  All of it is exact
// integer arithmetic on exact conversions, so the result has the bits of the
// N periods taken one by one.
__device__ __forceinline__ void carry_periods(float cf[3], float2 o[3], const float2 Q[3], const float2 U[3],
                                              int N) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float u = U[a].x, ui = U[a].y, wi = ui * 0x1p19f;
        const int sh = (__float_as_int(ui) >> 23) - 127;               // ui = 2^sh
        // exact integers below 2^24 in magnitude
        const long long H = __float2int_rz(o[a].x * ui);
        const long long L0 = __float2int_rz(o[a].y * wi);
        const long long Qi = __float2int_rz(Q[a].x * ui);
        const long long R = __float2int_rz((float)kCarry * Q[a].y * wi);
        const long long X = L0 + (long long)N * R;
        const long long Lp = N >= 2 ? ((X - R) & 0x7ffff) : L0;        // the low word before the last period
        const long long A = H + (long long)(kCarry * N) * Qi + (X >> 19);
        const long long C = (A - ((Lp + R) >> 19)) >> sh;               // whole cells moved out
        cf[a] += (float)C;
        o[a].x = (float)(A - (C << sh)) * u;
        o[a].y = (float)(X & 0x7ffff) * (u * 0x1p-19f);
    }
}

// Bring the offset pair onto the drift's grids: hi a multiple of u (its
// finer bits go to lo), lo a multiple of u 2^-19 (rounded, ~1e-13 of a cell,
// once after each stretch in the map).  Idempotent: once on the grids a pair
// stays there (every drift operation is exact), so a call at the start of
// every run changes nothing but the first, and a track's bits do not depend
// on where its runs start.
__device__ __forceinline__ void drift_enter(float2 o[3], const float2 U[3]) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float u = U[a].x, ui = U[a].y;
        const float hq = rintf(o[a].x * ui) * u;
        float lo = o[a].y + (o[a].x - hq);
        const float w = u * 0x1p-19f, wi = ui * 0x1p19f;
        o[a].x = hq;
        o[a].y = rintf(lo * wi) * w;
    }
}

__device__ __forceinline__ void add_quanta(float2 o[3], const float2 Q[3]) {
#pragma unroll
    for (int a = 0; a < 3; ++a) o[a] = __fadd2_rn(o[a], Q[a]);
}

// Whole cells out of the high word (exact: hi is a multiple of u after the
// drift's first steps, and hi - floor(hi) is exact for hi >= 0 anyway), so a
// Boris-family step starts from hi in [0, 1] without normalising it first.
__device__ __forceinline__ void normalise(float cf[3], float2 o[3]) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float cc = floorf(o[a].x);
        o[a].x -= cc;
        cf[a] += cc;
    }
}

// m field-free steps from global step g0.  Every field-free step adds q to
// the high words exactly (drift_quanta), so the k steps up to the first carry
// point, and those after the last, leave hi + k q, which one fused
// multiply-add yields with its single rounding: the same bits as k additions
// (x and y as one packed FFMA2).  The low words take k r the same way, and
// the whole periods in between go in closed form (carry_periods).  The
// carries stay where the global step index puts them.
// (on_grid: the offset pair is on the drift's grids already, the previous
// run having left it there, so drift_enter would change nothing.)
__device__ __forceinline__ void drift_steps(float cf[3], float2 o[3], const float2 Q[3], const float2 U[3],
                                            int64_t g0, int m, bool on_grid) {
    if (!on_grid) drift_enter(o, U);
    const float2 qxy = make_float2(Q[0].x, Q[1].x);
    const float qz = Q[2].x;
    auto run = [&](int k) {
        const float kf = (float)k;
        const float2 hxy = __ffma2_rn(make_float2(kf, kf), qxy, make_float2(o[0].x, o[1].x));
        o[0].x = hxy.x;
        o[1].x = hxy.y;
        o[2].x = fmaf(kf, qz, o[2].x);
#pragma unroll
        for (int a = 0; a < 3; ++a) o[a].y = fmaf(kf, Q[a].y, o[a].y);
    };
    // up to the first carry point (the steps g with (g + 1) % kCarry == 0)
    const int head = (int)((kCarry - ((unsigned)g0 & kCarryMask)) & kCarryMask);
    int j = 0;
    if (head > 0) {
        j = head < m ? head : m;
        run(j);
        if (j == head) carry(cf, o, U);
    }
    const int np = (m - j) / kCarry;
    if (np > 0) {
        carry_periods(cf, o, Q, U, np);
        j += np * kCarry;
    }
    if (j < m) run(m - j);   // the steps after the last carry point (fewer than kCarry)
    normalise(cf, o);
}

// Steps the particle certainly stays outside the cell range of the map (the
// pre-test of family_step), so that they are field-free drift steps: it is
// outside on some axis and must travel `dist` cells at `rate` cells per step
// to come back on that axis.  (cn, fn) is the normalised position and q the
// per-step advance of the high word, which is all the pre-test sees; the
// margin covers a rounding of 2^-24 ((kCarry + 1) |q| + 2) cells per step
// and that of this estimate, so every step counted here is one the pre-test
// would have sent down the drift branch.
__device__ __forceinline__ int quiet_steps(const TrackMixDev& P, const float cn[3], const float fn[3],
                                           const float2 Q[3]) {
    float best = 0.0f;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float dist, rate;
        const float q = Q[a].x;
        if (cn[a] < 0.0f) {
            dist = -cn[a] - fn[a];                          // back in range once cn + fn >= 0
            rate = q;
        } else if (cn[a] > P.cell_max[a]) {
            dist = (cn[a] - (P.cell_max[a] + 1.0f)) + fn[a];   // back once cn + fn < cell_max + 1
            rate = -q;
        } else {
            continue;
        }
        const float k = rate > 0.0f ? dist / (rate + 1.2e-7f * fmaf((float)(kCarry + 1), fabsf(q), 2.0f)) : 2e9f;
        best = fmaxf(best, k);
    }
    best = fmaf(best, 0.99999f, -2.0f);
    return best <= 0.0f ? 0 : (best >= 1e9f ? 1000000000 : (int)best);
}

// One step g of the Boris family with float-valued cell indices (exact
// integers below 2^24).  Returns the number of following steps known to be
// field-free (0 when this step met a field or the particle may come back).
template <int ALG, bool RF, int L>
__device__ __forceinline__ int family_step(MixCtx& c, float cf[3], float2 o[3], float vh[3], float vl[3], Drift& d,
                                           int64_t g) {
    const TrackMixDev& P = *c.P;
    // (cf, hi) is normalised: hi in [0, 1] after steps that may see a field,
    // after field-free runs and steps (normalise), and in the loaded state
    const float cn[3] = {cf[0], cf[1], cf[2]};
    const float fn[3] = {o[0].x, o[1].x, o[2].x};
    // a cell whose 8 corners are inner nodes on every axis (cells 1 .. n-3):
    // the offset in [0, 1] keeps the position strictly inside, so the
    // weights are the offsets, with no face rule to apply; otherwise the
    // cheap pre-test on the cell range (the last node layer included) and
    // the exact bounds rule in gather_mixed
    // (the Boris kernel only: with the relativistic pushers' longer step the
    // second gather path cost more registers than it saved, 6-7 % slower)
    const int cell[3] = {(int)cn[0], (int)cn[1], (int)cn[2]};
    const bool inner = ALG == PPT_ALG_BORIS && ((unsigned)(cell[0] - 1) < P.inner_span[0]) &
                       ((unsigned)(cell[1] - 1) < P.inner_span[1]) & ((unsigned)(cell[2] - 1) < P.inner_span[2]);
    const bool maybe = inner || ((cn[0] >= 0.0f) & (cn[0] <= P.cell_max[0]) & (cn[1] >= 0.0f) &
                                 (cn[1] <= P.cell_max[1]) & (cn[2] >= 0.0f) & (cn[2] <= P.cell_max[2]));
    if (maybe || const_fields<L>(P)) {
        F3 E, B, El;
        const float fln[3] = {o[0].y, o[1].y, o[2].y};
        bool have;
        if (ALG == PPT_ALG_BORIS && inner) {
            field_init<L>(P, E, B, El);
            gather_cell<L>(P, cell[0], cell[1], cell[2], fn[0], fn[1], fn[2], E, B, El);
            c.hits += 1u;
            rf_modulate<RF, L>(c, g, 0.0, E, El);
            have = true;
        } else {
            have = fields_mixed<RF, L>(c, cell, fn, fln, g, 0.0, E, B, El);
        }
        if (have) {
            F3 v = f3(vh[0], vh[1], vh[2]);
            if constexpr (ALG == PPT_ALG_BORIS) {
                // only the velocity components the layout's fields can change;
                // the kick's float32 roundings go to the low word
                constexpr int DM = boris_bits(L);
                vel_add_fast_kc<DM>(vh, vl, boris_dv<L>(v, E, B, P.hqdt), P.wscale,
                                    kick_correction<e_bits(L)>(E, El, P.hqdt));
                if (((unsigned)(g + 1) & 3u) == 0u) vel_renorm<DM>(vh, vl);
                increment<DM>(P, vh, vl, d.dh, d.dl);
            } else if constexpr (ALG == PPT_ALG_BORIS_REL || ALG == PPT_ALG_VAY) {
                // the state is u = gamma v; every component moves with gamma
                float du[3], corr[3];
                if constexpr (ALG == PPT_ALG_BORIS_REL)
                    boris_rel_du<e_bits(L), b_bits(L)>(vh, E, B, P.hqdt, P.wscale, du, corr);
                else
                    vay_du<e_bits(L), b_bits(L)>(vh, E, B, P.hqdt, P.wscale, du, corr);
                vel_add_corr(vh, vl, du, corr);
                if (((unsigned)(g + 1) & 3u) == 0u) vel_renorm<7>(vh, vl);
                increment_u(P, vh, vl, d.dh, d.dl);
            } else {
                vel_add(vh, vl, P.dtf * lorentz_f(v, E, B, P.qm));
                increment(P, vh, vl, d.dh, d.dl);
            }
        }
        // where fields act (or may): the increment (q, r) into the offset pair,
        // nothing rounded away (add_cells_q); lo folds into hi with the
        // velocity's renormalisation, after global steps g with (g + 1) % 4 == 0
        const bool fold = ((unsigned)(g + 1) & 3u) == 0u;
#pragma unroll
        for (int a = 0; a < 3; ++a) add_cells_q(cf[a], o[a].x, o[a].y, d.dh[a], d.dl[a], fold);
        return 0;
    }
    float2 Q[3], U[3];
    drift_quanta(d, Q, U);
    drift_enter(o, U);
    add_quanta(o, Q);
    if (((unsigned)(g + 1) & kCarryMask) == 0u) carry(cf, o, U);
    normalise(cf, o);
    // the next steps' pre-test, decided now from the normalised position
    const float fnext[3] = {o[0].x, o[1].x, o[2].x};
    return quiet_steps(P, cf, fnext, Q);
}

template <int ALG, bool RF, int L>
__device__ __forceinline__ void mixed_step(MixCtx& c, int cell[3], float f[3], float fl[3], float vh[3], float vl[3],
                                           Drift& d, int64_t g) {
    const TrackMixDev& P = *c.P;
    F3 v = f3(vh[0], vh[1], vh[2]);
    if constexpr (ALG == PPT_ALG_VAY_REL) {
        F3 E, B;
        fields_mixed<RF, L>(c, cell, f, fl, g, 0.0, E, B);
        F3 vn = vay_rel_f(v, E, B, P.qm, P.dtf);
        // increment relative to the float32 head keeps the low part's bits
        vel_add(vh, vl, vn - v);
        advance(P, cell, f, fl, vh, vl);
    } else {  // RK4 / RK4_REL (pusher.py:803-892), stage times t, t+h, t+h, t+dt
        constexpr bool REL = ALG == PPT_ALG_RK4_REL;
        const float dt = P.dtf, h = 0.5f * dt;
        F3 E, B;
        int sc[3];
        float sf[3];
        const float sl[3] = {0.0f, 0.0f, 0.0f};   // stage positions: high words only
        fields_mixed<RF, L>(c, cell, f, fl, g, 0.0, E, B);
        F3 k1 = REL ? rk4_rel_deriv_f(v, E, B, P.qm) : lorentz_f(v, E, B, P.qm);
        F3 v2 = v + h * k1;
        offset_point(P, cell, f, h * v, sc, sf);
        fields_mixed<RF, L>(c, sc, sf, sl, g, 0.5 * P.dt, E, B);
        F3 k2 = REL ? rk4_rel_deriv_f(v2, E, B, P.qm) : lorentz_f(v2, E, B, P.qm);
        F3 v3_ = v + h * k2;
        offset_point(P, cell, f, h * v2, sc, sf);
        fields_mixed<RF, L>(c, sc, sf, sl, g, 0.5 * P.dt, E, B);
        F3 k3 = REL ? rk4_rel_deriv_f(v3_, E, B, P.qm) : lorentz_f(v3_, E, B, P.qm);
        F3 v4 = v + dt * k3;
        offset_point(P, cell, f, dt * v3_, sc, sf);
        fields_mixed<RF, L>(c, sc, sf, sl, g, P.dt, E, B);
        F3 k4 = REL ? rk4_rel_deriv_f(v4, E, B, P.qm) : lorentz_f(v4, E, B, P.qm);
        // r_new - r = dt v + dt^2/6 (k1 + k2 + k3); v_new - v = dt/6 (k1 + 2k2 + 2k3 + k4)
        const float s6 = dt * (1.0f / 6.0f);
        F3 dr = (dt * s6) * (k1 + k2 + k3);
        F3 dv = s6 * (k1 + 2.0f * k2 + 2.0f * k3 + k4);
        const float drv[3] = {dr.x, dr.y, dr.z};
        // position: the dt v part in float-float, the stage correction (in
        // cells) added with it into the float-float offset
#pragma unroll
        for (int a = 0; a < 3; ++a)
            advance_axis(cell[a], f[a], fl[a], vh[a], vl[a], P.kh[a], P.kl[a], drv[a] * P.inv_d[a]);
        vel_add(vh, vl, dv);
        if (REL) {
            F3 vn = f3(vh[0], vh[1], vh[2]);
            float vm = sqrtf(dotf(vn, vn));
            if (vm >= 0.9999f * kCf) vel_set(vh, vl, ((0.9999f * kCf) / vm) * vn);
        }
    }
}

// Snapshot row: x = lo + (cell + f + fl) d and v = vh + vl (u / gamma(u)
// for the u state), formed in float64 (output formatting only).
__device__ __forceinline__ void write_mixed_row(const TrackMixDev& P, int64_t rec, int64_t row, const int cell[3],
                                                const float f[3], const float fl[3], const float vh[3],
                                                const float vl[3], bool r_too, bool u_state = false) {
    const int64_t o = (rec * P.n + row) * 3;
    double w[3] = {(double)vh[0] + (double)vl[0], (double)vh[1] + (double)vl[1], (double)vh[2] + (double)vl[2]};
    if (u_state) {
        const double ig = 1.0 / sqrt(1.0 + (w[0] * w[0] + w[1] * w[1] + w[2] * w[2]) / (kClight * kClight));
        w[0] *= ig;
        w[1] *= ig;
        w[2] *= ig;
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (r_too) P.r_hist[o + a] = P.G.lo[a] + ((double)cell[a] + ((double)f[a] + (double)fl[a])) * P.G.d[a];
        P.v_hist[o + a] = w[a];
    }
}

__host__ __device__ constexpr bool alg_u_family(int a) { return a == PPT_ALG_BORIS_REL || a == PPT_ALG_VAY; }

// Half step (+-dt/2 through hq = +-hqdt/2) of the u-state pushers: the
// staggering of the Boris family (the float64 form's half_kick).
template <int ALG, int L>
__device__ __forceinline__ void u_half_kick(float vh[3], float vl[3], F3 E, F3 B, float hq, float ws) {
    float du[3], corr[3];
    if constexpr (ALG == PPT_ALG_BORIS_REL) boris_rel_du<e_bits(L), b_bits(L)>(vh, E, B, hq, ws, du, corr);
    else vay_du<e_bits(L), b_bits(L)>(vh, E, B, hq, ws, du, corr);
    vel_add_corr(vh, vl, du, corr);
    vel_renorm<7>(vh, vl);
}

// float64 position of (cell + offset) on the tracking grid (the snapshot rows' formula)
__device__ __forceinline__ V3 mixed_position(const TrackMixDev& P, const float cf[3], const float2 o[3]) {
    return v3(P.G.lo[0] + ((double)cf[0] + ((double)o[0].x + (double)o[0].y)) * P.G.d[0],
              P.G.lo[1] + ((double)cf[1] + ((double)o[1].x + (double)o[1].y)) * P.G.d[1],
              P.G.lo[2] + ((double)cf[2] + ((double)o[2].x + (double)o[2].y)) * P.G.d[2]);
}

// COLL (Boris only): each step's segment, from the float64 positions before
// and after it, is tested against the electrode surface after the step's
// snapshot, and a particle that hits stops there (pusher.py:966-990).
template <int ALG, bool RF, int L, bool COLL = false>
__device__ __forceinline__ unsigned track_mixed_particle(const TrackMixDev& P, int64_t s, MixCtx& c,
                                                         const CollDev* C = nullptr) {
    {
        const int64_t n = P.n;
        if constexpr (COLL) {
            if (!C->active[P.order ? P.order[s] : s]) return 0;   // stopped in an earlier call
        }
        bool stopped = false;
        unsigned steps_done = (unsigned)P.nsteps;
        int cell[3];
        float f[3], fl[3], vh[3], vl[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            cell[a] = P.ci[a * n + s];
            f[a] = P.fs[a * n + s];
            vh[a] = P.fs[(3 + a) * n + s];
            vl[a] = P.fs[(6 + a) * n + s];
            fl[a] = P.fs[(9 + a) * n + s];
        }
        const int64_t row = P.order ? P.order[s] : s;
        if (RF) {
            c.phase = fma(P.omega, P.t0, P.rf_phase[s]);   // omega t0 + phi_i
            sincos(c.phase, &c.s0, &c.c0);
        }
        if (P.flags & PPT_TRACK_INIT) {
            if constexpr (ALG == PPT_ALG_BORIS) {
                F3 E, B;
                if (fields_mixed<RF, L>(c, cell, f, fl, P.step0, 0.0, E, B))
                    // Boris push with time step -dt/2 (pusher.py:947-958): half of hqdt
                    vel_add_boris<boris_bits(L)>(vh, vl, boris_dv<L>(f3(vh[0], vh[1], vh[2]), E, B, -0.5f * P.hqdt),
                                                 P.wscale);
            } else if constexpr (alg_u_family(ALG)) {
                F3 E, B;
                if (fields_mixed<RF, L>(c, cell, f, fl, P.step0, 0.0, E, B)) u_half_kick<ALG, L>(vh, vl, E, B, -0.5f * P.hqdt, P.wscale);
            }
            if (P.r_hist) write_mixed_row(P, 0, row, cell, f, fl, vh, vl, true, alg_u_family(ALG));
        }
        Drift d;
        if constexpr (alg_u_family(ALG)) increment_u(P, vh, vl, d.dh, d.dl);
        else increment(P, vh, vl, d.dh, d.dl);
        const int nsteps = (int)P.nsteps;
        const int rec_every = P.rec_every > 0x7fffffff ? 0x7fffffff : (int)P.rec_every;
        const int64_t until64 = P.rec_every - 1 - (P.step0 % P.rec_every);
        int until = until64 > 0x7fffffff ? 0x7fffffff : (int)until64;   // beyond this launch anyway
        if constexpr (ALG == PPT_ALG_BORIS || ALG == PPT_ALG_LEAPFROG || alg_u_family(ALG)) {
            float cf[3] = {(float)cell[0], (float)cell[1], (float)cell[2]};
            float2 o[3] = {make_float2(f[0], fl[0]), make_float2(f[1], fl[1]), make_float2(f[2], fl[2])};
            // record-free segments: the inner loop carries only its counter
            int k = 0;
            int quiet = 0;   // upcoming steps known to be field-free (quiet_steps)
            bool on_grid = false;   // the last steps were a field-free run (drift_steps)
            while (k < nsteps) {
                const int64_t to_rec = (int64_t)until + 1;
                const int seg = (int)(to_rec < (int64_t)(nsteps - k) ? to_rec : (int64_t)(nsteps - k));
                const int64_t g0 = P.step0 + k;
                if constexpr (COLL) {
                    // one step at a time, each segment tested (no field-free runs)
                    int i = 0;
                    while (i < seg) {
                        const V3 r0 = mixed_position(P, cf, o);
                        family_step<ALG, RF, L>(c, cf, o, vh, vl, d, g0 + i);
                        ++i;
                        if (segment_hits_surface(C->surf, r0, mixed_position(P, cf, o))) {
                            stopped = true;
                            break;
                        }
                    }
                    k += i;
                    // the reference records the step's position before its collision test
                    if ((int64_t)i == to_rec) {
                        const int64_t rec = (P.step0 + k) / P.rec_every;
                        const int ic[3] = {(int)cf[0], (int)cf[1], (int)cf[2]};
                        const float oh[3] = {o[0].x, o[1].x, o[2].x}, ol[3] = {o[0].y, o[1].y, o[2].y};
                        if (P.r_hist && rec < P.n_rec) write_mixed_row(P, rec, row, ic, oh, ol, vh, vl, true, alg_u_family(ALG));
                        until = rec_every - 1;
                    } else {
                        until -= i;
                    }
                    if (stopped) {
                        steps_done = (unsigned)k;
                        break;
                    }
                    continue;
                }
                for (int i = 0; i < seg;) {
                    if (quiet > 0) {
                        const int m = quiet < seg - i ? quiet : seg - i;
                        float2 Q[3], U[3];
                        drift_quanta(d, Q, U);
                        drift_steps(cf, o, Q, U, g0 + i, m, on_grid);
                        on_grid = true;
                        i += m;
                        quiet -= m;
                    } else {
                        quiet = family_step<ALG, RF, L>(c, cf, o, vh, vl, d, g0 + i);
                        on_grid = false;
                        ++i;
                    }
                }
                k += seg;
                if ((int64_t)seg == to_rec) {
                    const int64_t rec = (P.step0 + k) / P.rec_every;
                    const int ic[3] = {(int)cf[0], (int)cf[1], (int)cf[2]};
                    const float oh[3] = {o[0].x, o[1].x, o[2].x}, ol[3] = {o[0].y, o[1].y, o[2].y};
                    if (P.r_hist && rec < P.n_rec) write_mixed_row(P, rec, row, ic, oh, ol, vh, vl, true, alg_u_family(ALG));
                    until = rec_every - 1;
                } else {
                    until -= seg;
                }
            }
            // the state keeps its (possibly uncarried) offset; exact anyway
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                cell[a] = (int)cf[a];
                f[a] = o[a].x;
                fl[a] = o[a].y;
            }
        } else {
            for (int k = 0; k < nsteps; ++k) {
                mixed_step<ALG, RF, L>(c, cell, f, fl, vh, vl, d, P.step0 + k);
                if (until == 0) {
                    const int64_t rec = (P.step0 + k + 1) / P.rec_every;
                    if (P.r_hist && rec < P.n_rec) write_mixed_row(P, rec, row, cell, f, fl, vh, vl, true);
                    until = rec_every - 1;
                } else {
                    --until;
                }
            }
        }
        if ((P.flags & PPT_TRACK_FINAL) && !stopped) {
            if constexpr (ALG == PPT_ALG_BORIS) {
                F3 E, B;
                int cn[3];
                float fn[3];
#pragma unroll
                for (int a = 0; a < 3; ++a) {   // exact normalisation for the cell lookup
                    const float cc = floorf(f[a]);
                    cn[a] = cell[a] + (int)cc;
                    fn[a] = f[a] - cc;
                }
                if (fields_mixed<RF, L>(c, cn, fn, fl, P.nsteps_total, 0.0, E, B))
                    // Boris push with time step +dt/2 (pusher.py:993-1007)
                    vel_add_boris<boris_bits(L)>(vh, vl, boris_dv<L>(f3(vh[0], vh[1], vh[2]), E, B, 0.5f * P.hqdt),
                                                 P.wscale);
                if (P.v_hist) write_mixed_row(P, P.n_rec - 1, row, cell, f, fl, vh, vl, false);
            } else if constexpr (alg_u_family(ALG)) {
                F3 E, B;
                int cn[3];
                float fn[3];
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    const float cc = floorf(f[a]);
                    cn[a] = cell[a] + (int)cc;
                    fn[a] = f[a] - cc;
                }
                if (fields_mixed<RF, L>(c, cn, fn, fl, P.nsteps_total, 0.0, E, B))
                    u_half_kick<ALG, L>(vh, vl, E, B, 0.5f * P.hqdt, P.wscale);
                if (P.v_hist) write_mixed_row(P, P.n_rec - 1, row, cell, f, fl, vh, vl, false, true);
            }
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            P.ci[a * n + s] = cell[a];
            P.fs[a * n + s] = f[a];
            P.fs[(3 + a) * n + s] = vh[a];
            P.fs[(6 + a) * n + s] = vl[a];
            P.fs[(9 + a) * n + s] = fl[a];
        }
        if (P.status) {
            float sum = f[0] + f[1] + f[2] + vh[0] + vh[1] + vh[2];
            if (!isfinite(sum)) atomicOr(P.status, PPT_STATUS_NONFINITE);
            const int lim = 1 << 24;
            if (abs(cell[0]) >= lim || abs(cell[1]) >= lim || abs(cell[2]) >= lim) atomicOr(P.status, PPT_STATUS_RANGE);
        }
        if constexpr (COLL) {
            if (stopped) C->active[P.order ? P.order[s] : s] = 0;
        }
        return steps_done;
    }
}

template <int ALG, bool RF, int L>
__global__ void __launch_bounds__(128) track_mixed_kernel(const __grid_constant__ TrackMixDev P) {
    const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    unsigned steps_done = 0;
    MixCtx c{&P, 0.0, 0u, 0.0, 0.0, nullptr, 0};
    if constexpr (RF) {
        extern __shared__ double2 rf_tab[];
        if (P.rf_tab_n > 0) {
            build_rf_table(rf_tab, P.step0, P.rf_tab_n, P.wdt);
            c.tab = rf_tab;
            c.tab0 = P.step0;
        }
    }
    if (s < P.n) steps_done = track_mixed_particle<ALG, RF, L>(P, s, c);
    if (P.counters) block_add_counters(P.counters, c.hits, steps_done);
}

// The same with the electrode segment test (Boris).
template <bool RF, int L>
__global__ void __launch_bounds__(128) track_mixed_coll_kernel(const __grid_constant__ TrackMixDev P,
                                                               const __grid_constant__ CollDev C) {
    const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    unsigned steps_done = 0;
    MixCtx c{&P, 0.0, 0u, 0.0, 0.0, nullptr, 0};
    if constexpr (RF) {
        extern __shared__ double2 rf_tab[];
        if (P.rf_tab_n > 0) {
            build_rf_table(rf_tab, P.step0, P.rf_tab_n, P.wdt);
            c.tab = rf_tab;
            c.tab0 = P.step0;
        }
    }
    if (s < P.n) steps_done = track_mixed_particle<PPT_ALG_BORIS, RF, L, true>(P, s, c, &C);
    if (P.counters) block_add_counters(P.counters, c.hits, steps_done);
}

// Serving: the mixed-precision counterpart of track_f64_jobs_kernel.
static_assert(sizeof(TrackMixDev) % 8 == 0, "TrackMixDev is copied as 8-byte words");

template <int ALG, bool RF, int L>
__global__ void __launch_bounds__(kJobBlock) track_mixed_jobs_kernel(const __grid_constant__ JobQueueDev Q) {
    __shared__ __align__(16) TrackMixDev sP;
    __shared__ int s_item, s_job;
    const TrackMixDev* table = static_cast<const TrackMixDev*>(Q.table);
    for (;;) {
        take_item(Q, &s_item, &s_job);
        const int it = s_item;
        if (it >= Q.n_items) return;
        const int cj = s_job;
        const int gjob = Q.job_index[cj];
        {
            const uint64_t* src = reinterpret_cast<const uint64_t*>(table + Q.table_index[cj]);
            uint64_t* dst = reinterpret_cast<uint64_t*>(&sP);
            for (int i = threadIdx.x; i < (int)(sizeof(TrackMixDev) / 8); i += blockDim.x) dst[i] = src[i];
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int64_t s0, k;
            int fl;
            job_window(Q, gjob, sP.nsteps_total, &s0, &k, &fl);
            sP.step0 = s0;
            sP.nsteps = k;
            sP.flags = Q.done[gjob] ? -1 : fl;
        }
        __syncthreads();
        if (sP.flags >= 0) {
            const int64_t s = (int64_t)(it - Q.item_start[cj]) * blockDim.x + threadIdx.x;
            MixCtx c{&sP, 0.0, 0u, 0.0, 0.0, nullptr, 0};
            if constexpr (RF) {
                // this job's step window, when the launch reserved a table
                // that long for it (chunk + 1 entries; a job with a longer
                // window of its own computes the same values directly)
                extern __shared__ double2 rf_tab[];
                const int nt = (int)sP.nsteps + 1;
                if (Q.chunk + 1 <= kRfTable && nt <= Q.chunk + 1) {
                    build_rf_table(rf_tab, sP.step0, nt, sP.wdt);
                    c.tab = rf_tab;
                    c.tab0 = sP.step0;
                }
            }
            unsigned sd = 0;
            if (s < sP.n) sd = track_mixed_particle<ALG, RF, L>(sP, s, c);
            if (sP.counters) block_add_counters(sP.counters, c.hits, sd);
        }
        __syncthreads();
    }
}

// Kernel of (algorithm, RF, layout).  Layouts without E ignore the RF flag:
// their fields have no E to modulate.
template <int ALG, int L>
static cudaError_t launch_mixed_layout(const TrackMixDev* P, const JobQueueDev* Q, bool rf, int grid,
                                       cudaStream_t s) {
    constexpr bool kE = layout_has_e(L);
    if (P) {
        const int block = pick_block(P->n);
        const int g = grid_for(P->n, block);
        const size_t smem = (size_t)P->rf_tab_n * sizeof(double2);
        if (rf && kE) track_mixed_kernel<ALG, kE, L><<<g, block, smem, s>>>(*P);
        else track_mixed_kernel<ALG, false, L><<<g, block, 0, s>>>(*P);
    } else {
        const size_t smem = Q->chunk + 1 <= kRfTable ? (size_t)(Q->chunk + 1) * sizeof(double2) : 0;
        if (rf && kE) track_mixed_jobs_kernel<ALG, kE, L><<<grid, kJobBlock, smem, s>>>(*Q);
        else track_mixed_jobs_kernel<ALG, false, L><<<grid, kJobBlock, 0, s>>>(*Q);
    }
    return cudaGetLastError();
}

template <int ALG>
static cudaError_t launch_mixed_alg(const TrackMixDev* P, const JobQueueDev* Q, int layout, bool rf, int grid,
                                    cudaStream_t s) {
    switch (layout) {
        case kLayFull: return launch_mixed_layout<ALG, kLayFull>(P, Q, rf, grid, s);
        case kLayE: return launch_mixed_layout<ALG, kLayE>(P, Q, rf, grid, s);
        case kLayB: return launch_mixed_layout<ALG, kLayB>(P, Q, rf, grid, s);
        case kLayExEyBz: return launch_mixed_layout<ALG, kLayExEyBz>(P, Q, rf, grid, s);
        case kLayEzBz: return launch_mixed_layout<ALG, kLayEzBz>(P, Q, rf, grid, s);
        default: return launch_mixed_layout<ALG, kLayBz>(P, Q, rf, grid, s);
    }
}

static int launch_mixed(const TrackMixDev* P, const JobQueueDev* Q, int algorithm, int layout, bool rf, int grid,
                        cudaStream_t s, const char* what) {
    cudaError_t e;
    switch (algorithm) {
        case PPT_ALG_LEAPFROG: e = launch_mixed_alg<PPT_ALG_LEAPFROG>(P, Q, layout, rf, grid, s); break;
        case PPT_ALG_BORIS: e = launch_mixed_alg<PPT_ALG_BORIS>(P, Q, layout, rf, grid, s); break;
        case PPT_ALG_RK4: e = launch_mixed_alg<PPT_ALG_RK4>(P, Q, layout, rf, grid, s); break;
        case PPT_ALG_VAY_REL: e = launch_mixed_alg<PPT_ALG_VAY_REL>(P, Q, layout, rf, grid, s); break;
        case PPT_ALG_RK4_REL: e = launch_mixed_alg<PPT_ALG_RK4_REL>(P, Q, layout, rf, grid, s); break;
        case PPT_ALG_BORIS_REL: e = launch_mixed_alg<PPT_ALG_BORIS_REL>(P, Q, layout, rf, grid, s); break;
        case PPT_ALG_VAY: e = launch_mixed_alg<PPT_ALG_VAY>(P, Q, layout, rf, grid, s); break;
        default:
            return fail(PPT_ERR_UNSUPPORTED, "the mixed form covers leapfrog, boris, rk4, vay_rel, rk4_rel, boris_rel "
                                             "and vay; use precision 'fp64'");
    }
    if (e != cudaSuccess) return cuda_fail(e, what);
    return PPT_OK;
}

int launch_mixed_jobs(const JobQueueDev& Q, int algorithm, int layout, bool rf, int grid, cudaStream_t s) {
    return launch_mixed(nullptr, &Q, algorithm, layout, rf, grid, s, "track_mixed_jobs_kernel launch");
}

int launch_track_mixed(const TrackMixDev& P, int algorithm, bool rf, cudaStream_t s) {
    return launch_mixed(&P, nullptr, algorithm, P.map.layout, rf, 0, s, "track_mixed_kernel launch");
}

template <int L>
static cudaError_t launch_coll_layout(const TrackMixDev& P, const CollDev& C, bool rf, cudaStream_t s) {
    constexpr bool kE = layout_has_e(L);
    const int block = pick_block(P.n);
    const int g = grid_for(P.n, block);
    if (rf && kE) track_mixed_coll_kernel<kE, L><<<g, block, (size_t)P.rf_tab_n * sizeof(double2), s>>>(P, C);
    else track_mixed_coll_kernel<false, L><<<g, block, 0, s>>>(P, C);
    return cudaGetLastError();
}

int launch_track_mixed_coll(const TrackMixDev& P, const CollDev& C, bool rf, cudaStream_t s) {
    cudaError_t e;
    switch (P.map.layout) {
        case kLayFull: e = launch_coll_layout<kLayFull>(P, C, rf, s); break;
        case kLayE: e = launch_coll_layout<kLayE>(P, C, rf, s); break;
        case kLayB: e = launch_coll_layout<kLayB>(P, C, rf, s); break;
        case kLayExEyBz: e = launch_coll_layout<kLayExEyBz>(P, C, rf, s); break;
        case kLayEzBz: e = launch_coll_layout<kLayEzBz>(P, C, rf, s); break;
        default: e = launch_coll_layout<kLayBz>(P, C, rf, s); break;
    }
    if (e != cudaSuccess) return cuda_fail(e, "track_mixed_coll_kernel launch");
    return PPT_OK;
}

// host-side construction of the mixed kernel parameters
int make_track_mixed(const FieldsDev& F, const ppt_state* st, const ppt_track_args* a, int64_t n_rec,
                     TrackMixDev* P) {
    int rc = mixed_grid(F, &P->G);
    if (rc) return rc;
    P->map = F.maps[0];
    // an axis the map does not vary along: every cell reads its one layer
    if (axis_is_flat(P->map.ax[0])) P->map.sx = 0;
    if (axis_is_flat(P->map.ax[1])) P->map.sy = 0;
    P->k_elems = axis_is_flat(P->map.ax[2]) ? 0 : layout_width(P->map.layout);
    if (P->k_elems == 0) P->map.idx32 = 0;
    for (int c = 0; c < 3; ++c) {
        P->e_const[c] = (float)F.e_const[c];
        P->b_const[c] = (float)F.b_const[c];
        double k = a->dt / P->G.d[c];
        P->kh[c] = (float)k;
        P->kl[c] = (float)(k - (double)P->kh[c]);
        P->inv_d[c] = (float)P->G.inv_d[c];
        P->cell_max[c] = (float)(P->G.n[c] - 1);
        P->inner_span[c] = P->G.n[c] > 3 ? (uint32_t)(P->G.n[c] - 3) : 0u;
    }
    P->const_nz = F.e_const_nz || F.b_const_nz;
    if (P->const_nz && P->map.layout != kLayFull)
        return fail(PPT_ERR_UNSUPPORTED,
                    "mixed form: fields with constant parts need a map of all six components "
                    "(ppt_fieldmap_create_masked with 0x3F)");
    P->n = st->n;
    P->step0 = a->step0;
    P->nsteps = a->nsteps;
    P->nsteps_total = a->nsteps_total;
    P->rec_every = a->rec_every;
    P->n_rec = n_rec;
    P->flags = a->flags;
    P->dt = a->dt;
    P->t0 = a->t0;
    P->omega = a->rf_omega;
    P->wdt = a->rf_omega * a->dt;
    P->qm = (float)a->q_over_m;
    P->hqdt = (float)(0.5 * a->q_over_m * a->dt);
    P->wscale = 0.0f;
    if (st->algorithm == PPT_ALG_BORIS || alg_u_family(st->algorithm)) {
        // Boris-family increments scaled by (1 + wscale): hqdt (1 + wscale) is
        // q/m dt/2 to float64 accuracy
        const double exact = 0.5 * a->q_over_m * a->dt;
        const double ws = exact / (double)P->hqdt - 1.0;
        P->wscale = (float)ws;
    }
    P->dtf = (float)a->dt;
    P->rf_phase = a->rf_phase;
    // the launch's per-step RF table covers steps step0 .. step0 + nsteps
    // (the closing half step reads the last one)
    P->rf_tab_n = (a->rf_phase && a->nsteps + 1 <= kRfTable) ? (int32_t)(a->nsteps + 1) : 0;
    P->ci = st->i32;
    P->fs = st->f32;
    P->r_hist = a->r_hist;
    P->v_hist = a->v_hist;
    P->order = a->order;
    P->status = a->status;
    P->counters = a->counters;
    return PPT_OK;
}

}  // namespace ppt
