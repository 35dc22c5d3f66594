/*
 * ppt_oracle.c -- CPU restatement of the reference's batch tracking loop.
 *
 * TEST INFRASTRUCTURE ONLY: used by tests as a checker and by bench.py as
 * the timed CPU baseline (the reference is Python + Numba and cannot travel
 * to the benchmark host).  The product never links or calls it.
 *
 * It keeps the reference's structure so that its timing represents the
 * reference's CPU path: every step evaluates E and B as separate
 * per-component passes over all particles, each point searching its cell by
 * bisection (field.py:491-504, interpolators.py:44-135, :259-267), then a
 * separate push pass and a position pass (pusher.py:699-801, :369-404,
 * :803-892), each pass a parallel loop over particles (OpenMP here, Numba
 * prange in the reference).  Arithmetic follows the same source lines as
 * oracle/pusher_oracle.py.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define CLIGHT 299792458.0

enum { ALG_LEAPFROG = 0, ALG_BORIS = 1, ALG_RK4 = 2, ALG_VAY_REL = 4, ALG_RK4_REL = 5 };

typedef struct {
    int64_t n[3];
    const double* axis[3];
    const double* comp[6];  /* Ex Ey Ez Bx By Bz node values, C order [i][j][k]; NULL = 0 */
} oracle_map;

/* interpolators.py:44-60 */
static int64_t search_cell(const double* g, int64_t n, double x) {
    if (x < g[0]) return 0;
    if (x >= g[n - 1]) return n - 2;
    int64_t left = 0, right = n - 1;
    while (left < right - 1) {
        int64_t mid = (left + right) / 2;
        if (g[mid] <= x) left = mid; else right = mid;
    }
    return left;
}

static double clamp01(double t) { return t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t); }

/* interpolators.py:88-135 */
static double interp3d(const oracle_map* m, const double* v, double x, double y, double z) {
    const double *gx = m->axis[0], *gy = m->axis[1], *gz = m->axis[2];
    const int64_t nx = m->n[0], ny = m->n[1], nz = m->n[2];
    if (x < gx[0] || x > gx[nx - 1] || y < gy[0] || y > gy[ny - 1] || z < gz[0] || z > gz[nz - 1]) return 0.0;
    int64_t i = search_cell(gx, nx, x), j = search_cell(gy, ny, y), k = search_cell(gz, nz, z);
    double tx = clamp01((x - gx[i]) / (gx[i + 1] - gx[i]));
    double ty = clamp01((y - gy[j]) / (gy[j + 1] - gy[j]));
    double tz = clamp01((z - gz[k]) / (gz[k + 1] - gz[k]));
#define V(a, b, c) v[((i + (a)) * ny + (j + (b))) * nz + (k + (c))]
    double c00 = V(0, 0, 0) * (1.0 - tx) + V(1, 0, 0) * tx;
    double c01 = V(0, 0, 1) * (1.0 - tx) + V(1, 0, 1) * tx;
    double c10 = V(0, 1, 0) * (1.0 - tx) + V(1, 1, 0) * tx;
    double c11 = V(0, 1, 1) * (1.0 - tx) + V(1, 1, 1) * tx;
#undef V
    double c0 = c00 * (1.0 - ty) + c10 * ty;
    double c1 = c01 * (1.0 - ty) + c11 * ty;
    return c0 * (1.0 - tz) + c1 * tz;
}

/* one Field evaluation: three per-component passes (field.py:491-504) */
static void eval_field(const oracle_map* m, int which, int64_t n, const double* r, double* out) {
    for (int c = 0; c < 3; ++c) {
        const double* v = m->comp[3 * which + c];
#pragma omp parallel for schedule(static)
        for (int64_t p = 0; p < n; ++p)
            out[3 * p + c] = v ? interp3d(m, v, r[3 * p], r[3 * p + 1], r[3 * p + 2]) : 0.0;
    }
}

static void rf_scale(int64_t n, double* e, double omega, const double* phase, double t) {
    if (!phase) return;
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < n; ++p) {
        double c = cos(omega * t + phase[p]);
        e[3 * p] *= c; e[3 * p + 1] *= c; e[3 * p + 2] *= c;
    }
}

static void fields(const oracle_map* m, int64_t n, const double* r, double t, double omega, const double* phase,
                   double* e, double* b) {
    eval_field(m, 0, n, r, e);
    rf_scale(n, e, omega, phase, t);
    eval_field(m, 1, n, r, b);
}

static void cross(const double* a, const double* b, double* o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

/* pusher.py:124-165 */
static void boris1(const double* v, const double* E, const double* B, double dt, double qm, double* out) {
    double vm[3], t[3], s[3], vp[3], c1[3], c2[3];
    for (int c = 0; c < 3; ++c) { vm[c] = v[c] + 0.5 * qm * E[c] * dt; t[c] = 0.5 * qm * B[c] * dt; }
    double tsq = t[0] * t[0] + t[1] * t[1] + t[2] * t[2];
    for (int c = 0; c < 3; ++c) s[c] = 2.0 * t[c] / (1.0 + tsq);
    cross(vm, t, c1);
    for (int c = 0; c < 3; ++c) vp[c] = vm[c] + c1[c];
    cross(vp, s, c2);
    for (int c = 0; c < 3; ++c) out[c] = vm[c] + c2[c] + 0.5 * qm * E[c] * dt;
}

static double rel_gamma(const double* v) {
    double b2 = (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) / (CLIGHT * CLIGHT);
    if (b2 >= 0.9999) b2 = 0.9999;
    return 1.0 / sqrt(1.0 - b2);
}

static void clamp_speed(double* v) {
    double vm = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (vm >= 0.9999 * CLIGHT) for (int c = 0; c < 3; ++c) v[c] *= 0.9999 * CLIGHT / vm;
}

/* pusher.py:216-279 */
static void vay1(const double* v, const double* E, const double* B, double dt, double qm, double* out) {
    double g = rel_gamma(v), up[3], tau[3], t[3], s[3], us[3], c1[3], c2[3];
    for (int c = 0; c < 3; ++c) { tau[c] = 0.5 * qm * B[c] * dt; up[c] = g * v[c] + qm * E[c] * dt; }
    double upm = sqrt(up[0] * up[0] + up[1] * up[1] + up[2] * up[2]);
    double taum = sqrt(tau[0] * tau[0] + tau[1] * tau[1] + tau[2] * tau[2]);
    double udt = up[0] * tau[0] + up[1] * tau[1] + up[2] * tau[2];
    double gis = 1.0 - (upm / CLIGHT) * (upm / CLIGHT);
    if (gis < 1e-10) gis = 1e-10;
    double sigma = gis - taum * taum;
    double gn = sqrt(0.5 * (sigma + sqrt(sigma * sigma + 4.0 * (taum * taum + (udt / CLIGHT) * (udt / CLIGHT)))));
    for (int c = 0; c < 3; ++c) t[c] = tau[c] / gn;
    for (int c = 0; c < 3; ++c) s[c] = 2.0 * t[c] / (1.0 + taum * taum / (gn * gn));
    cross(up, t, c1);
    for (int c = 0; c < 3; ++c) us[c] = up[c] + c1[c];
    cross(us, s, c2);
    for (int c = 0; c < 3; ++c) out[c] = (up[c] + c2[c]) / gn;
    clamp_speed(out);
}

/* pusher.py:168-172 / :282-298 */
static void deriv(int rel, const double* v, const double* E, const double* B, double qm, double* out) {
    double vb[3], F[3];
    cross(v, B, vb);
    for (int c = 0; c < 3; ++c) F[c] = qm * (E[c] + vb[c]);
    if (!rel) { for (int c = 0; c < 3; ++c) out[c] = F[c]; return; }
    double g = rel_gamma(v);
    double vdf = v[0] * F[0] + v[1] * F[1] + v[2] * F[2];
    for (int c = 0; c < 3; ++c) out[c] = F[c] / g - (vdf / (g * CLIGHT * CLIGHT)) * v[c];
}

/* Pusher.track_batch (pusher.py:894-1012), no electrode assembly. */
int oracle_track(int alg, int64_t n, const double* r0, const double* v0, const oracle_map* m, int64_t nsteps,
                 double dt, double qm, int64_t rec, double omega, const double* phase, double t0, double* r_hist,
                 double* v_hist) {
    if (n <= 0 || rec < 1) return -1;
    if (alg != ALG_LEAPFROG && alg != ALG_BORIS && alg != ALG_RK4 && alg != ALG_VAY_REL && alg != ALG_RK4_REL)
        return -2;
    const int64_t n_rec = nsteps / rec + 1;
    const size_t sz = (size_t)n * 3 * sizeof(double);
    double *r = malloc(sz), *v = malloc(sz), *E = malloc(sz), *B = malloc(sz), *rn = malloc(sz), *vn = malloc(sz);
    double *k[4], *kr = malloc(sz), *vv = malloc(sz);
    for (int q = 0; q < 4; ++q) k[q] = malloc(sz);
    memcpy(r, r0, sz);
    memcpy(v, v0, sz);
    if (alg == ALG_BORIS) {
        fields(m, n, r, t0, omega, phase, E, B);
#pragma omp parallel for schedule(static)
        for (int64_t p = 0; p < n; ++p) boris1(v + 3 * p, E + 3 * p, B + 3 * p, -0.5 * dt, qm, vn + 3 * p);
        memcpy(v, vn, sz);
    }
    if (r_hist) { memcpy(r_hist, r, sz); memcpy(v_hist, v, sz); }
    int64_t ri = 1;
    for (int64_t step = 0; step < nsteps; ++step) {
        const double t = t0 + (double)step * dt;
        if (alg == ALG_RK4 || alg == ALG_RK4_REL) {
            const int rel = alg == ALG_RK4_REL;
            /* pusher.py:803-892 */
            const double cs[4] = {0.0, 0.5 * dt, 0.5 * dt, dt};
            for (int q = 0; q < 4; ++q) {
                if (q == 0) {
                    memcpy(kr, r, sz);
                    memcpy(vv, v, sz);
                } else {
#pragma omp parallel for schedule(static)
                    for (int64_t i = 0; i < 3 * n; ++i) {
                        double prev_v = q == 1 ? v[i] : vv[i];  /* k_{q}_r = v of the previous stage */
                        kr[i] = r[i] + cs[q] * prev_v;
                    }
#pragma omp parallel for schedule(static)
                    for (int64_t i = 0; i < 3 * n; ++i) vv[i] = v[i] + cs[q] * k[q - 1][i];
                }
                fields(m, n, kr, t + cs[q], omega, phase, E, B);
#pragma omp parallel for schedule(static)
                for (int64_t p = 0; p < n; ++p) deriv(rel, vv + 3 * p, E + 3 * p, B + 3 * p, qm, k[q] + 3 * p);
                if (q == 0) memcpy(rn, v, sz);                       /* k1_r */
                else if (q < 3) {
#pragma omp parallel for schedule(static)
                    for (int64_t i = 0; i < 3 * n; ++i) rn[i] += 2.0 * vv[i];
                } else {
#pragma omp parallel for schedule(static)
                    for (int64_t i = 0; i < 3 * n; ++i) rn[i] += vv[i];
                }
            }
#pragma omp parallel for schedule(static)
            for (int64_t p = 0; p < n; ++p) {
                for (int c = 0; c < 3; ++c) {
                    int64_t i = 3 * p + c;
                    r[i] = r[i] + (dt / 6.0) * rn[i];
                    v[i] = v[i] + (dt / 6.0) * (k[0][i] + 2.0 * k[1][i] + 2.0 * k[2][i] + k[3][i]);
                }
                if (rel) clamp_speed(v + 3 * p);
            }
        } else {
            fields(m, n, r, t, omega, phase, E, B);
#pragma omp parallel for schedule(static)
            for (int64_t p = 0; p < n; ++p) {
                if (alg == ALG_BORIS) boris1(v + 3 * p, E + 3 * p, B + 3 * p, dt, qm, vn + 3 * p);
                else if (alg == ALG_VAY_REL) vay1(v + 3 * p, E + 3 * p, B + 3 * p, dt, qm, vn + 3 * p);
                else {
                    double a[3];
                    deriv(0, v + 3 * p, E + 3 * p, B + 3 * p, qm, a);
                    for (int c = 0; c < 3; ++c) vn[3 * p + c] = v[3 * p + c] + a[c] * dt;
                }
            }
            /* position_update_batch, pusher.py:395-404 */
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < 3 * n; ++i) rn[i] = r[i] + vn[i] * dt;
            memcpy(r, rn, sz);
            memcpy(v, vn, sz);
        }
        if ((step + 1) % rec == 0 && ri < n_rec && r_hist) {
            memcpy(r_hist + ri * 3 * n, r, sz);
            memcpy(v_hist + ri * 3 * n, v, sz);
            ++ri;
        }
    }
    if (alg == ALG_BORIS) {
        fields(m, n, r, t0 + (double)nsteps * dt, omega, phase, E, B);
#pragma omp parallel for schedule(static)
        for (int64_t p = 0; p < n; ++p) boris1(v + 3 * p, E + 3 * p, B + 3 * p, 0.5 * dt, qm, vn + 3 * p);
        memcpy(v, vn, sz);
        if (v_hist) memcpy(v_hist + (n_rec - 1) * 3 * n, v, sz);
    }
    free(r); free(v); free(E); free(B); free(rn); free(vn); free(kr); free(vv);
    for (int q = 0; q < 4; ++q) free(k[q]);
    return 0;
}

int oracle_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
