// Plain form: the reference's pushers in float64, fused with the trilinear
// gathers, many steps per launch.
//
// One thread owns one particle for the whole launch.  Its position and
// velocity live in registers across all steps of the call; per step it
// locates its cell, gathers the 8 corner records (one 256-bit load per field
// per corner), interpolates E and B, applies the algorithm's update and
// writes a snapshot row only on record steps.  The reference instead makes 6
// (Boris/Vay) or 24 (RK4) separate interpolation passes per step over
// particle arrays in DRAM, each with its own binary search
// (src/PyPATools/pusher.py:966-980, :699-801, field.py:491-504).
//
// Arithmetic follows the reference's kernels term by term so the results
// agree to rounding: Boris pusher.py:124-165, Vay 'vay_rel' :216-279,
// relativistic gamma :74-96, RK4 :803-892 with derivatives :168-172 and
// :282-298, leapfrog :730-739, Yoshida :184-209 / :332-362 (fields frozen at
// the step start), |v| clamps :275-277 / :886-890.  boris_rel and vay are
// additions (u = gamma v state, see the oracle for their equations).
#pragma once

#include <cmath>

#include "track_params.cuh"

namespace ppt {


__host__ __device__ constexpr bool alg_staggered(int a) {
    return a == PPT_ALG_BORIS || a == PPT_ALG_BORIS_REL || a == PPT_ALG_VAY;
}
__host__ __device__ constexpr bool alg_u_state(int a) { return a == PPT_ALG_BORIS_REL || a == PPT_ALG_VAY; }

// Yoshida (1990) 4th-order coefficients, the float64 values of the
// reference's expressions (pusher.py:176-181), written to round-trip exactly.
constexpr double kYoC1 = 1.3512071919596578;     // 1 / (2 - 2^(1/3))
constexpr double kYoC2 = -1.7024143839193153;    // -2^(1/3) / (2 - 2^(1/3))
constexpr double kYoD1 = 2.7024143839193155;     // 2 C1
constexpr double kYoD2 = -3.0536215758789735;    // -(2^(1/3) + 1) / (2 - 2^(1/3))

// ---------------------------------------------------------------------------
// per-algorithm updates (float64)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double rel_gamma(V3 v) {
    double bsq = dot(v, v) / (kClight * kClight);
    if (bsq >= 0.9999) bsq = 0.9999;
    return 1.0 / sqrt(1.0 - bsq);
}

__device__ __forceinline__ V3 clamp_speed(V3 v) {
    double vm = sqrt(dot(v, v));
    if (vm >= 0.9999 * kClight) v = v * (0.9999 * kClight / vm);
    return v;
}


// (p x q)_I in the reference's form p_J q_K - p_K q_J, without q's components
// outside the mask QM (an exact zero there).  A lone product is rounded on
// its own (__dmul_rn), as the full form rounds it before the caller adds it
// to a vector: left to the compiler, v + p_J q_K would fuse into one FMA and
// round once, which the full form never does.
template <int QM, int I>
__device__ __forceinline__ double cross_md(const double p[3], const double q[3]) {
    constexpr int J = (I + 1) % 3, K = (I + 2) % 3;
    if constexpr (bit(QM, K) && bit(QM, J)) return p[J] * q[K] - p[K] * q[J];
    else if constexpr (bit(QM, K)) return __dmul_rn(p[J], q[K]);
    else if constexpr (bit(QM, J)) return -__dmul_rn(p[K], q[J]);
    else return 0.0;
}

// boris_v for fields whose components outside EM (E) and BM (B) are zero by
// construction (a single map of a pruned record layout, no constant parts):
// the same operations on the components that can be non-zero, none on the
// others (pusher.py:124-165).
template <int EM, int BM>
__device__ __forceinline__ V3 boris_v_m(V3 v, V3 E, V3 B, double dt, double qm) {
    constexpr int CM = cross_bits(BM);
    const double h = 0.5 * qm;
    const double vv[3] = {v.x, v.y, v.z}, e[3] = {E.x, E.y, E.z}, b[3] = {B.x, B.y, B.z};
    double kick[3], vm[3], t[3], s[3], vp[3], out[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        kick[i] = bit(EM, i) ? h * e[i] * dt : 0.0;
        vm[i] = bit(EM, i) ? vv[i] + kick[i] : vv[i];
        t[i] = bit(BM, i) ? h * b[i] * dt : 0.0;
    }
    // t.t: a lone square rounded on its own, as the full form's sum rounds it
    // (left to the compiler, 1 + t_z t_z would fuse into one FMA)
    double tt;
    if constexpr (BM == 0) tt = 0.0;
    else if constexpr (BM == 4) tt = __dmul_rn(t[2], t[2]);
    else if constexpr (BM == 1) tt = __dmul_rn(t[0], t[0]);
    else if constexpr (BM == 2) tt = __dmul_rn(t[1], t[1]);
    else tt = t[0] * t[0] + t[1] * t[1] + t[2] * t[2];
    const double f = 2.0 / (1.0 + tt);
#pragma unroll
    for (int i = 0; i < 3; ++i) s[i] = bit(BM, i) ? t[i] * f : 0.0;
    vp[0] = bit(CM, 0) ? vm[0] + cross_md<BM, 0>(vm, t) : vm[0];
    vp[1] = bit(CM, 1) ? vm[1] + cross_md<BM, 1>(vm, t) : vm[1];
    vp[2] = bit(CM, 2) ? vm[2] + cross_md<BM, 2>(vm, t) : vm[2];
    const double c2[3] = {cross_md<BM, 0>(vp, s), cross_md<BM, 1>(vp, s), cross_md<BM, 2>(vp, s)};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const double vplus = bit(CM, i) ? vm[i] + c2[i] : vm[i];
        out[i] = bit(EM, i) ? vplus + kick[i] : vplus;
    }
    return v3(out[0], out[1], out[2]);
}

// The reference's Boris (pusher.py:124-165): kick = (q/m) E dt / 2,
// v- = v + kick, t = (q/m) B dt / 2, s = 2 t / (1 + t.t), v' = v- + v- x t,
// v+ = v- + v' x s, v_new = v+ + kick -- the masked form with every
// component present, so a map of a pruned record layout computes the same
// bits as one that stores its zero components.
__device__ __forceinline__ V3 boris_v(V3 v, V3 E, V3 B, double dt, double qm) {
    return boris_v_m<7, 7>(v, E, B, dt, qm);
}

__device__ __forceinline__ V3 vay_rel_v(V3 v, V3 E, V3 B, double dt, double qm) {
    double g = rel_gamma(v);
    V3 u = g * v;
    V3 tau = v3(0.5 * qm * B.x * dt, 0.5 * qm * B.y * dt, 0.5 * qm * B.z * dt);
    V3 up = v3(u.x + qm * E.x * dt, u.y + qm * E.y * dt, u.z + qm * E.z * dt);
    double upm = sqrt(dot(up, up));
    double taum = sqrt(dot(tau, tau));
    double udt = dot(up, tau);
    double gis = 1.0 - (upm / kClight) * (upm / kClight);
    if (gis < 1e-10) gis = 1e-10;
    double sigma = gis - taum * taum;
    double q = udt / kClight;
    double gn = sqrt(0.5 * (sigma + sqrt(sigma * sigma + 4.0 * (taum * taum + q * q))));
    double ig = 1.0 / gn;
    V3 t = tau * ig;
    double f = 2.0 / (1.0 + taum * taum * (ig * ig));
    V3 s = t * f;
    V3 us = up + cross(up, t);
    V3 un = up + cross(us, s);
    return clamp_speed(un * ig);
}

__device__ __forceinline__ V3 lorentz(V3 v, V3 E, V3 B, double qm) { return qm * (E + cross(v, B)); }

__device__ __forceinline__ V3 rk4_rel_deriv(V3 v, V3 E, V3 B, double qm) {
    double g = rel_gamma(v);
    V3 F = qm * (E + cross(v, B));
    double vdf = dot(v, F);
    V3 corr = (vdf / (g * kClight * kClight)) * v;
    return F / g - corr;
}

__device__ __forceinline__ double gamma_u(V3 u) { return sqrt(1.0 + dot(u, u) / (kClight * kClight)); }

__device__ __forceinline__ V3 boris_rel_u(V3 u, V3 E, V3 B, double dt, double qm) {
    const double h = 0.5 * qm * dt;
    V3 um = u + h * E;
    double g = gamma_u(um);
    V3 t = (h / g) * B;
    double f = 2.0 / (1.0 + dot(t, t));
    V3 s = t * f;
    V3 up = um + cross(um, t);
    V3 uplus = um + cross(up, s);
    return uplus + h * E;
}

__device__ __forceinline__ V3 vay_u(V3 u, V3 E, V3 B, double dt, double qm) {
    double g_old = gamma_u(u);
    V3 v_old = u / g_old;
    V3 up = u + (qm * dt) * (E + 0.5 * cross(v_old, B));
    V3 tau = (0.5 * qm * dt) * B;
    double tau_sq = dot(tau, tau);
    double ustar = dot(up, tau) / kClight;
    double sigma = 1.0 + dot(up, up) / (kClight * kClight) - tau_sq;
    double gn = sqrt(0.5 * (sigma + sqrt(sigma * sigma + 4.0 * (tau_sq + ustar * ustar))));
    V3 t = tau / gn;
    double s = 1.0 / (1.0 + dot(t, t));
    return s * (up + dot(up, t) * t + cross(up, t));
}

template <int ALG>
__device__ __forceinline__ V3 w_to_v(V3 w) {
    if constexpr (alg_u_state(ALG)) return w / gamma_u(w);
    else return w;
}

template <int ALG>
__device__ __forceinline__ V3 half_kick(V3 w, V3 E, V3 B, double dt, double qm) {
    if constexpr (ALG == PPT_ALG_BORIS) return boris_v(w, E, B, dt, qm);
    else if constexpr (ALG == PPT_ALG_BORIS_REL) return boris_rel_u(w, E, B, dt, qm);
    else return vay_u(w, E, B, dt, qm);
}

struct Ctx {
    const FieldsDev* F;
    double dt, qm, omega, phase, t0;
    unsigned hits;
    int const_nz;
    double c0, s0;            // cos, sin of omega t0 + phase
    const double2* tab;       // (cos, sin) of g omega dt for the launch's steps, or NULL
    int64_t tab0;             // the launch's first step
};

// Per-step RF table length limit (shared memory, 16 B per step): the sorted
// launches of a bunch crossing its map are a few hundred steps; longer
// launches evaluate the same expression directly.
constexpr int kRfTable64 = 512;

// Fill the block's table of (cos, sin) of g omega dt for steps step0 ..
// step0 + n - 1 (all threads of the block call it; n <= kRfTable64).
__device__ __forceinline__ void build_rf_table64(double2* tab, int64_t step0, int n, double wdt) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double sg, cg;
        sincos((double)(step0 + i) * wdt, &sg, &cg);
        tab[i] = make_double2(cg, sg);
    }
    __syncthreads();
}

// E and B of a single uniform-grid map of record layout L with no constant
// parts (E, B zero outside it); returns 1 when r is inside.  The cell search
// is locate_axis's uniform branch, the interpolation tri() per stored
// component, so the values are the run-time dispatch's (eval_fields_f64).
template <int L>
__device__ __forceinline__ int eval_single_f64(const MapDev& m, V3 r, V3& E, V3& B) {
    E = v3(0.0, 0.0, 0.0);
    B = v3(0.0, 0.0, 0.0);
    if (!(axis_contains(m.ax[0], r.x) & axis_contains(m.ax[1], r.y) & axis_contains(m.ax[2], r.z))) return 0;
    Cell c;
    int ijk[3];
    double tt[3];
    const double x[3] = {r.x, r.y, r.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const double u = (x[a] - m.ax[a].lo) * m.ax[a].inv_d;
        ijk[a] = __double2int_rd(u);             // floor: u is in [0, n - 1] here
        tt[a] = u - (double)ijk[a];
    }
    // cells 1 .. n-3 on every axis need none of the clamps below (the cell is
    // in range and u - floor(u) is in [0, 1)); the others take them
    if (!(((unsigned)(ijk[0] - 1) < (unsigned)(m.ax[0].n - 3)) & ((unsigned)(ijk[1] - 1) < (unsigned)(m.ax[1].n - 3)) &
          ((unsigned)(ijk[2] - 1) < (unsigned)(m.ax[2].n - 3)))) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const AxisDev& ax = m.ax[a];
            const double u = (x[a] - ax.lo) * ax.inv_d;
            int cc = ijk[a];
            cc = cc < 0 ? 0 : (cc > ax.n - 2 ? ax.n - 2 : cc);
            const double t = u - (double)cc;
            tt[a] = t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
            ijk[a] = cc;
        }
    }
    c.tx = tt[0];
    c.ty = tt[1];
    c.tz = tt[2];
    c.base = (int64_t)ijk[0] * m.sx + (int64_t)ijk[1] * m.sy + ijk[2];
    if constexpr (L == kLayFull) {
        E = gather_f64s<8>(m, c, 0);
        B = gather_f64s<8>(m, c, 4);
    } else if constexpr (L == kLayE) {
        E = gather_f64s<4>(m, c, 0);
    } else if constexpr (L == kLayB) {
        B = gather_f64s<4>(m, c, 0);
    } else if constexpr (L == kLayExEyBz) {
        const V3 o = gather_f64s<4>(m, c, 0);
        E = v3(o.x, o.y, 0.0);
        B = v3(0.0, 0.0, o.z);
    } else if constexpr (L == kLayEzBz) {
        double o[2];
        gather_slots_f64<2>(m, c, o);
        E = v3(0.0, 0.0, o[0]);
        B = v3(0.0, 0.0, o[1]);
    } else {
        double o[1];
        gather_slots_f64<1>(m, c, o);
        B = v3(0.0, 0.0, o[0]);
    }
    return 1;
}

// Fields at r and field time t0 + g dt + toff; the time and the RF cosine are
// only formed when E is non-zero.  Returns the number of maps containing r.
// L = 0: any fields (maps summed at run time, constant parts); otherwise a
// single map of record layout L (eval_single_f64).
// RF factor cos(omega (t0 + g dt + toff) + phi): at the step's own time
// (toff = 0) as cos(a + b) = cos a cos b - sin a sin b with a = omega t0 + phi
// per particle and b = g omega dt per step, (cos b, sin b) from the launch's
// table or, beyond it, the same float64 expression, so a track's bits do not
// depend on how it is split into launches; at RK4's stage times directly.
template <bool RF, int L>
__device__ __forceinline__ int fields_at(Ctx& c, V3 r, int64_t g, double toff, V3& E, V3& B) {
    int h;
    if constexpr (L == 0) h = eval_fields_f64(*c.F, r, E, B);
    else h = eval_single_f64<L>(c.F->maps[0], r, E, B);
    c.hits += h;
    if (RF) {
        constexpr int EM = L == 0 ? 7 : e_bits(L);
        if ((bit(EM, 0) && E.x != 0.0) || (bit(EM, 1) && E.y != 0.0) || (bit(EM, 2) && E.z != 0.0)) {
            double cf;
            if (toff == 0.0) {
                double cg, sg;
                if (c.tab != nullptr) {
                    const double2 t = c.tab[g - c.tab0];
                    cg = t.x;
                    sg = t.y;
                } else {
                    sincos((double)g * (c.omega * c.dt), &sg, &cg);
                }
                cf = fma(c.c0, cg, -(c.s0 * sg));
            } else {
                const double t = c.t0 + (double)g * c.dt + toff;
                cf = cos(c.omega * t + c.phase);
            }
            if constexpr (bit(EM, 0)) E.x = E.x * cf;
            if constexpr (bit(EM, 1)) E.y = E.y * cf;
            if constexpr (bit(EM, 2)) E.z = E.z * cf;
        }
    }
    return h;
}

// Position advance of one step, r + v dt (pusher.py:395-404).
__device__ __forceinline__ V3 drift(V3 r, V3 v, double dt) {
    return v3(fma(v.x, dt, r.x), fma(v.y, dt, r.y), fma(v.z, dt, r.z));
}

// m field-free steps of one coordinate, x <- fma(v, dt, x) at each, with the
// bits of the step-by-step loop.  The float64 numbers whose magnitude lies
// in one binade [2^E, 2^(E+1)) are the multiples of g = 2^(E-52) there, and x
// is one of them; so when the exact sum x + v dt lies in x's binade it rounds
// to x + D, D being v dt rounded to a multiple of g -- the same D at every
// such step, unless v dt lies exactly halfway between two multiples (then
// round-half-even looks at x's last bit).  Each trip of the loop therefore
// takes the steps whose sums certainly stay inside x's binade as k D in one
// exact fused multiply-add, then one step as it comes (the step out of the
// binade, a halfway case, or a step within four steps of zero).  A
// coordinate crossing zero passes the binades between |v dt| and |x| one
// trip each.
__device__ __forceinline__ double drift_coord(double x, double v, double dt, int m) {
    // a zero advance: the first step settles the sign of a zero x, the others keep x
    if (v == 0.0 || dt == 0.0) return m > 0 ? fma(v, dt, x) : x;
    const double p = v * dt;
    const double ap = fabs(p) * (1.0 + 0x1p-50);   // above |v dt| exactly
    while (m > 0) {
        const double ax = fabs(x);
        // (false for NaN and infinities too)
        if (ax >= 4.0 * ap && ax >= 0x1p-64 && ax < 0x1p1000) {
            const long long eb = __double_as_longlong(ax) >> 52;    // biased exponent of |x|
            const double lo = __longlong_as_double(eb << 52);        // 2^E
            const double D = fma(v, dt, x) - x;   // exact: the sum lies within [x/2, 2x]
            // distance of the sums from the binade's edge ahead, from below
            const double room = ((p > 0.0) == (x > 0.0) ? 2.0 * lo - ax : ax - lo) - ap;
            // not halfway: |v dt - D| != g / 2 = 2^(E-53)
            if (room > 0.0 && fabs(fma(v, dt, -D)) != __longlong_as_double((eb - 53) << 52)) {
                // steps n = 0 .. k-1 with n |D| < room; the quotient's error
                // (a few float32 ulps) is far inside the 1e-4 margin
                int k = m;
                if (D != 0.0) {
                    const float kq = __fdividef((float)room, (float)fabs(D)) * 0.9999f;
                    if (!(kq >= (float)m)) k = kq >= 1.0f ? (int)kq : 1;
                }
                x = fma((double)k, D, x);
                m -= k;
                if (m == 0) break;
            }
        }
        x = fma(v, dt, x);
        --m;
    }
    return x;
}

__device__ __forceinline__ V3 drift_run(V3 r, V3 v, double dt, int m) {
    return v3(drift_coord(r.x, v.x, dt, m), drift_coord(r.y, v.y, dt, m), drift_coord(r.z, v.z, dt, m));
}

__host__ __device__ constexpr bool alg_skips_free(int a) {
    return a == PPT_ALG_LEAPFROG || a == PPT_ALG_BORIS || a == PPT_ALG_BORIS_REL;
}

// Steps a particle moving at v certainly stays outside every map, so that
// they are field-free drift steps (only for fields without constant parts):
// outside the union box of the maps on some axis, it must travel `dist` at
// `rate` per step to come back on that axis.  After j steps the position
// carries at most j * 2^-53 * X of rounding (X bounds |x| on the way), which
// the margin covers.
__device__ __forceinline__ int quiet_steps_f64(const FieldsDev& F, V3 r, V3 v, double dt) {
    if (F.n_maps == 0) return 0;
    const double x[3] = {r.x, r.y, r.z}, u[3] = {v.x * dt, v.y * dt, v.z * dt};
    double best = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        double dist, rate, bound;
        if (x[a] < F.box_lo[a]) {
            dist = F.box_lo[a] - x[a];
            rate = u[a];
            bound = F.box_lo[a];
        } else if (x[a] > F.box_hi[a]) {
            dist = x[a] - F.box_hi[a];
            rate = -u[a];
            bound = F.box_hi[a];
        } else {
            continue;
        }
        const double X = fmax(fabs(x[a]), fabs(bound));
        const double k = rate > 0.0 ? dist / (rate + 2.3e-16 * X) : 2e9;
        best = fmax(best, k);
    }
    best = best * (1.0 - 1e-9) - 2.0;
    return best <= 0.0 ? 0 : (best >= 1e9 ? 1000000000 : (int)best);
}

// One step; returns true for a field-free step of the Boris family (its
// velocity update skipped, see below).
template <int ALG, bool RF, int L>
__device__ __forceinline__ bool step(Ctx& c, V3& r, V3& w, int64_t g) {
    const double dt = c.dt, qm = c.qm;
    if constexpr (ALG == PPT_ALG_RK4 || ALG == PPT_ALG_RK4_REL) {
        constexpr bool REL = ALG == PPT_ALG_RK4_REL;
        V3 E, B;
        const double h = 0.5 * dt;
        fields_at<RF, L>(c, r, g, 0.0, E, B);
        V3 k1v = REL ? rk4_rel_deriv(w, E, B, qm) : lorentz(w, E, B, qm);
        V3 k1r = w;
        V3 r2 = r + h * k1r, v2 = w + h * k1v;
        fields_at<RF, L>(c, r2, g, h, E, B);
        V3 k2v = REL ? rk4_rel_deriv(v2, E, B, qm) : lorentz(v2, E, B, qm);
        V3 r3 = r + h * v2, v3_ = w + h * k2v;
        fields_at<RF, L>(c, r3, g, h, E, B);
        V3 k3v = REL ? rk4_rel_deriv(v3_, E, B, qm) : lorentz(v3_, E, B, qm);
        V3 r4 = r + dt * v3_, v4 = w + dt * k3v;
        fields_at<RF, L>(c, r4, g, dt, E, B);
        V3 k4v = REL ? rk4_rel_deriv(v4, E, B, qm) : lorentz(v4, E, B, qm);
        const double s6 = dt / 6.0;
        r = r + s6 * (k1r + 2.0 * v2 + 2.0 * v3_ + v4);
        w = w + s6 * (k1v + 2.0 * k2v + 2.0 * k3v + k4v);
        if (REL) w = clamp_speed(w);
    } else if constexpr (ALG == PPT_ALG_YOSHIDA || ALG == PPT_ALG_YOSHIDA_REL) {
        constexpr bool REL = ALG == PPT_ALG_YOSHIDA_REL;
        V3 E, B;
        fields_at<RF, L>(c, r, g, 0.0, E, B);
        const double cs[3] = {kYoC1, kYoC2, kYoC1};
        const double ds[3] = {kYoD1, kYoD2, kYoD1};
#pragma unroll
        for (int s = 0; s < 3; ++s) {
            V3 a = REL ? rk4_rel_deriv(w, E, B, qm) : lorentz(w, E, B, qm);
            w = w + (cs[s] * dt) * a;
            r = r + (ds[s] * dt) * w;
        }
        if (REL) w = clamp_speed(w);
    } else {
        V3 E, B;
        // With no map containing r and no constant field, E = B = 0 exactly and
        // the leapfrog, Boris and relativistic Boris updates return w unchanged
        // (every term they add is a signed zero), so they are skipped.
        const bool any = fields_at<RF, L>(c, r, g, 0.0, E, B) != 0 || c.const_nz;
        if constexpr (ALG == PPT_ALG_LEAPFROG) {
            if (any) w = w + lorentz(w, E, B, qm) * dt;
            r = drift(r, w, dt);
        } else if constexpr (ALG == PPT_ALG_BORIS) {
            if (any) {
                if constexpr (L == 0) w = boris_v(w, E, B, dt, qm);
                else w = boris_v_m<e_bits(L), b_bits(L)>(w, E, B, dt, qm);
            }
            r = drift(r, w, dt);
        } else if constexpr (ALG == PPT_ALG_VAY_REL) {
            w = vay_rel_v(w, E, B, dt, qm);
            r = drift(r, w, dt);
        } else if constexpr (ALG == PPT_ALG_BORIS_REL) {
            if (any) w = boris_rel_u(w, E, B, dt, qm);
            r = drift(r, w_to_v<ALG>(w), dt);
        } else {  // PPT_ALG_VAY
            w = vay_u(w, E, B, dt, qm);
            r = drift(r, w_to_v<ALG>(w), dt);
        }
        return alg_skips_free(ALG) && !any;
    }
    return false;
}

__device__ __forceinline__ void write_row(double* hist, int64_t rec, int64_t n, int64_t row, V3 a) {
    double* p = hist + (rec * n + row) * 3;
    p[0] = a.x;
    p[1] = a.y;
    p[2] = a.z;
}

__device__ __forceinline__ Ctx make_ctx(const TrackDev& P) {
    return Ctx{&P.F, P.dt, P.qm, P.omega, 0.0, P.t0, 0u, P.F.e_const_nz | P.F.b_const_nz, 1.0, 0.0, nullptr, 0};
}

// All steps of one call for particle slot s (s < P.n); returns the steps done.
// COLL: each step's segment is tested against the electrode surface after the
// step's snapshot, and a particle that hits stops there (pusher.py:966-990).
template <int ALG, bool RF, bool COLL, int L>
__device__ __forceinline__ unsigned track_f64_particle(const TrackDev& P, int64_t s, Ctx& c) {
    {
        const int64_t n = P.n;
        double* st = P.f64;
        const int64_t row = P.order ? P.order[s] : s;
        if constexpr (COLL) {
            if (!P.active[row]) return 0;   // stopped in an earlier call: nothing moves or records
        }
        V3 r = v3(st[s], st[n + s], st[2 * n + s]);
        V3 w = v3(st[3 * n + s], st[4 * n + s], st[5 * n + s]);
        if constexpr (ALG == PPT_ALG_RK4 || ALG == PPT_ALG_RK4_REL) {
            // the reference's array dt: every stage of this particle's step uses its own
            // dt (pusher.py:815-816), and so does its field time t0 + g dt (the
            // launch's RF table holds the launch's dt: not used then)
            if (P.dt_rows) {
                c.dt = P.dt_rows[row];
                c.tab = nullptr;
            }
        }
        if (RF) {
            c.phase = P.rf_phase[s];
            double sa, ca;
            sincos(fma(c.omega, c.t0, c.phase), &sa, &ca);
            c.c0 = ca;
            c.s0 = sa;
        }
        bool stopped = false;

        if (P.flags & PPT_TRACK_INIT) {
            if constexpr (alg_staggered(ALG)) {
                V3 E, B;
                fields_at<RF, L>(c, r, P.step0, 0.0, E, B);
                w = half_kick<ALG>(w, E, B, -0.5 * P.dt, P.qm);
            }
            if (P.r_hist) {
                write_row(P.r_hist, 0, n, row, r);
                write_row(P.v_hist, 0, n, row, w_to_v<ALG>(w));
            }
        }
        // steps until the next record: record after global step g when (g+1) % rec == 0
        const int nsteps = (int)P.nsteps;
        const int rec_every = P.rec_every > 0x7fffffff ? 0x7fffffff : (int)P.rec_every;
        const int64_t until64 = P.rec_every - 1 - (P.step0 % P.rec_every);
        int until = until64 > 0x7fffffff ? 0x7fffffff : (int)until64;   // beyond this launch anyway
        // record-free segments: the inner loop carries only its counter
        int k = 0;
        int quiet = 0;   // upcoming steps known to be field-free (quiet_steps_f64)
        while (k < nsteps) {
            const int64_t to_rec = (int64_t)until + 1;
            const int seg = (int)(to_rec < (int64_t)(nsteps - k) ? to_rec : (int64_t)(nsteps - k));
            const int64_t g0 = P.step0 + k;
            if constexpr (COLL) {
                // one step at a time, each segment tested (no field-free runs)
                int i = 0;
                while (i < seg) {
                    const V3 r0 = r;
                    step<ALG, RF, L>(c, r, w, g0 + i);
                    ++i;
                    if (segment_hits_surface(P.surf, r0, r)) {
                        stopped = true;
                        break;
                    }
                }
                k += i;
                // the reference records the step's position before its collision test
                if ((int64_t)i == to_rec) {
                    const int64_t rec = (P.step0 + k) / P.rec_every;
                    if (P.r_hist && rec < P.n_rec) {
                        write_row(P.r_hist, rec, n, row, r);
                        write_row(P.v_hist, rec, n, row, w_to_v<ALG>(w));
                    }
                    until = rec_every - 1;
                } else {
                    until -= i;
                }
                if (stopped) break;
                continue;
            }
            if constexpr (alg_skips_free(ALG)) {
                for (int i = 0; i < seg;) {
                    if (quiet > 0) {
                        // a run of field-free steps: the same position advance, no field lookups
                        const int m = quiet < seg - i ? quiet : seg - i;
                        r = drift_run(r, w_to_v<ALG>(w), P.dt, m);
                        i += m;
                        quiet -= m;
                    } else {
                        if (step<ALG, RF, L>(c, r, w, g0 + i)) quiet = quiet_steps_f64(P.F, r, w_to_v<ALG>(w), P.dt);
                        ++i;
                    }
                }
            } else {
                for (int i = 0; i < seg; ++i) step<ALG, RF, L>(c, r, w, g0 + i);
            }
            k += seg;
            if ((int64_t)seg == to_rec) {
                const int64_t rec = (P.step0 + k) / P.rec_every;
                if (P.r_hist && rec < P.n_rec) {
                    write_row(P.r_hist, rec, n, row, r);
                    write_row(P.v_hist, rec, n, row, w_to_v<ALG>(w));
                }
                until = rec_every - 1;
            } else {
                until -= seg;
            }
        }
        if ((P.flags & PPT_TRACK_FINAL) && !stopped) {
            if constexpr (alg_staggered(ALG)) {
                V3 E, B;
                fields_at<RF, L>(c, r, P.nsteps_total, 0.0, E, B);
                w = half_kick<ALG>(w, E, B, 0.5 * P.dt, P.qm);
                if (P.v_hist) write_row(P.v_hist, P.n_rec - 1, n, row, w_to_v<ALG>(w));
            }
        }
        st[s] = r.x;
        st[n + s] = r.y;
        st[2 * n + s] = r.z;
        st[3 * n + s] = w.x;
        st[4 * n + s] = w.y;
        st[5 * n + s] = w.z;
        if (P.status) {
            double sum = r.x + r.y + r.z + w.x + w.y + w.z;
            if (!isfinite(sum)) atomicOr(P.status, PPT_STATUS_NONFINITE);
        }
        if constexpr (COLL) {
            if (stopped) {
                P.active[row] = 0;
                return (unsigned)k;
            }
        }
    }
    return (unsigned)P.nsteps;
}

// Blocks of 128 per SM the launch bounds ask for: the Boris family's kernels
// of a pruned record layout fit 80 registers without spills (6 blocks: the
// RF-gap map crossing 65.0 -> 62.9 ms against 96 registers and 5 blocks);
// the run-time dispatch, the full record and the collision test would spill
// there and keep 5.
__host__ __device__ constexpr int f64_min_blocks(int alg, bool coll, int layout) {
    return !alg_skips_free(alg) ? 1 : (!coll && layout != 0 && layout != kLayFull) ? 6 : 5;
}

// L = 0: any fields; L = a kLay* mask: one uniform-grid map of that record
// layout, no constant parts (fields_at, boris_v_m).
template <int ALG, bool RF, bool COLL, int L>
__global__ void __launch_bounds__(128, f64_min_blocks(ALG, COLL, L)) track_f64_kernel(const __grid_constant__ TrackDev P) {
    const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    unsigned steps_done = 0;
    Ctx c = make_ctx(P);
    if constexpr (RF) {
        extern __shared__ double2 rf_tab64[];
        if (P.rf_tab_n > 0) {
            build_rf_table64(rf_tab64, P.step0, P.rf_tab_n, P.omega * P.dt);
            c.tab = rf_tab64;
            c.tab0 = P.step0;
        }
    }
    if (s < P.n) steps_done = track_f64_particle<ALG, RF, COLL, L>(P, s, c);
    if (P.counters) block_add_counters(P.counters, c.hits, steps_done);
}

// Serving: a persistent block-level work queue over the float64 jobs of one
// (algorithm, RF) class.  Each item is one job's 128-particle block; the job's
// parameter block is staged in shared memory and its step window for this
// tick comes from the device-resident step counters.
static_assert(sizeof(TrackDev) % 8 == 0, "TrackDev is copied as 8-byte words");

template <int ALG, bool RF, int L>
__global__ void __launch_bounds__(kJobBlock) track_f64_jobs_kernel(const __grid_constant__ JobQueueDev Q) {
    __shared__ __align__(16) TrackDev sP;
    __shared__ int s_item, s_job;
    const TrackDev* table = static_cast<const TrackDev*>(Q.table);
    for (;;) {
        take_item(Q, &s_item, &s_job);
        const int it = s_item;
        if (it >= Q.n_items) return;
        const int cj = s_job;
        const int gjob = Q.job_index[cj];
        {
            const uint64_t* src = reinterpret_cast<const uint64_t*>(table + Q.table_index[cj]);
            uint64_t* dst = reinterpret_cast<uint64_t*>(&sP);
            for (int i = threadIdx.x; i < (int)(sizeof(TrackDev) / 8); i += blockDim.x) dst[i] = src[i];
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int64_t s0, k;
            int fl;
            job_window(Q, gjob, sP.nsteps_total, &s0, &k, &fl);
            sP.step0 = s0;
            sP.nsteps = k;
            sP.flags = Q.done[gjob] ? -1 : fl;   // -1: job finished, nothing to do
        }
        __syncthreads();
        if (sP.flags >= 0) {
            const int64_t s = (int64_t)(it - Q.item_start[cj]) * blockDim.x + threadIdx.x;
            Ctx c = make_ctx(sP);
            unsigned sd = 0;
            if (s < sP.n) sd = track_f64_particle<ALG, RF, false, L>(sP, s, c);
            if (sP.counters) block_add_counters(sP.counters, c.hits, sd);
        }
        __syncthreads();
    }
}

}  // namespace ppt
