"""CPU oracle for the pusher + trilinear field-interpolation path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product imports this module: only
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
use it, and only as the checker.

It is a vectorised NumPy restatement, in float64, of the reference
(DanielWinklehner/PyPATools) algorithms, each function citing the file:line it
follows.  Parity is pinned by ``tests/test_oracle_golden.py``, which checks
this module against trajectories produced by running the reference itself
(fixtures in ``tests/golden/``, made by ``tests/golden/make_golden.py``).

Beyond the reference, it restates three things the reference lacks, using the
same kernels:
* a time-dependent E field ``E(x) cos(omega t + phi_i)`` evaluated at the
  step's field time (t_n for Boris/Vay/leapfrog/Yoshida, the stage times for
  RK4);
* ``boris_rel``: the relativistic Boris push in u = gamma v space;
* ``vay``: the Vay (2008) push as published.
Those two keep u (not v) as the state between steps, so |u| is conserved to
roundoff in a pure magnetic field.
"""
import numpy as np
from scipy import constants as _const

CLIGHT = _const.speed_of_light

ALGORITHMS = ["leapfrog", "boris", "rk4", "yoshida", "vay_rel", "rk4_rel", "yoshida_rel",
              "boris_rel", "vay"]


# ---------------------------------------------------------------------------
# Trilinear interpolation  (field_src/interpolators.py:44-135)
# ---------------------------------------------------------------------------

def cell_index(axis, q):
    """Cell index of ``q`` on sorted node array ``axis``.

    interpolators.py:44-60 (_searchsorted_numba): 0 below the first node,
    n-2 at or above the last, else the left node of the bracketing cell; then
    clamped to [0, n-2] (interpolators.py:104-106).  ``searchsorted(side=
    'right') - 1`` is the same bracketing rule.
    """
    n = axis.shape[0]
    i = np.searchsorted(axis, q, side="right") - 1
    return np.clip(i, 0, n - 2)


def interp3d(pts, grid, values, fill_value=0.0):
    """One component at (M,3) points.  interpolators.py:88-135, :259-267."""
    gx, gy, gz = grid
    x, y, z = pts[:, 0], pts[:, 1], pts[:, 2]
    out = np.full(pts.shape[0], fill_value, dtype=np.float64)
    inside = ~((x < gx[0]) | (x > gx[-1]) | (y < gy[0]) | (y > gy[-1]) |
               (z < gz[0]) | (z > gz[-1]))
    if not inside.any():
        return out
    x, y, z = x[inside], y[inside], z[inside]
    i = cell_index(gx, x)
    j = cell_index(gy, y)
    k = cell_index(gz, z)
    tx = np.clip((x - gx[i]) / (gx[i + 1] - gx[i]), 0.0, 1.0)
    ty = np.clip((y - gy[j]) / (gy[j + 1] - gy[j]), 0.0, 1.0)
    tz = np.clip((z - gz[k]) / (gz[k + 1] - gz[k]), 0.0, 1.0)
    v = values
    c000 = v[i, j, k]
    c100 = v[i + 1, j, k]
    c010 = v[i, j + 1, k]
    c110 = v[i + 1, j + 1, k]
    c001 = v[i, j, k + 1]
    c101 = v[i + 1, j, k + 1]
    c011 = v[i, j + 1, k + 1]
    c111 = v[i + 1, j + 1, k + 1]
    c00 = c000 * (1.0 - tx) + c100 * tx
    c01 = c001 * (1.0 - tx) + c101 * tx
    c10 = c010 * (1.0 - tx) + c110 * tx
    c11 = c011 * (1.0 - tx) + c111 * tx
    c0 = c00 * (1.0 - ty) + c10 * ty
    c1 = c01 * (1.0 - ty) + c11 * ty
    out[inside] = c0 * (1.0 - tz) + c1 * tz
    return out


def interp1d(x, grid, values, fill_value=0.0):
    """One component at (M,) coordinates.  interpolators.py:192-205, :239-245."""
    (gx,) = grid
    out = np.full(x.shape[0], fill_value, dtype=np.float64)
    inside = ~((x < gx[0]) | (x > gx[-1]))
    x = x[inside]
    i = cell_index(gx, x)
    t = np.clip((x - gx[i]) / (gx[i + 1] - gx[i]), 0.0, 1.0)
    out[inside] = values[i] * (1.0 - t) + values[i + 1] * t
    return out


def interp2d(x, y, grid, values, fill_value=0.0):
    """One component at (M,) x and y.  interpolators.py:208-236, :248-256."""
    gx, gy = grid
    out = np.full(x.shape[0], fill_value, dtype=np.float64)
    inside = ~((x < gx[0]) | (x > gx[-1]) | (y < gy[0]) | (y > gy[-1]))
    x, y = x[inside], y[inside]
    i = cell_index(gx, x)
    j = cell_index(gy, y)
    tx = np.clip((x - gx[i]) / (gx[i + 1] - gx[i]), 0.0, 1.0)
    ty = np.clip((y - gy[j]) / (gy[j + 1] - gy[j]), 0.0, 1.0)
    c0 = values[i, j] * (1.0 - tx) + values[i + 1, j] * tx
    c1 = values[i, j + 1] * (1.0 - tx) + values[i + 1, j + 1] * tx
    out[inside] = c0 * (1.0 - ty) + c1 * ty
    return out


# ---------------------------------------------------------------------------
# Field objects  (field.py:213-244, :441-504, :595-690, :389-407)
# ---------------------------------------------------------------------------

class MapField:
    """1D, 2D or 3D map: per-component interpolation times ``scaling``
    (field.py:457-504).  Components given as None are identically zero.  As
    in the reference, a 1D map (one grid array) is evaluated at the points'
    z and a 2D map at their (x, y), whichever axes the grid was given on."""

    def __init__(self, grid, values, scaling=1.0):
        self.grid = tuple(np.ascontiguousarray(g, dtype=np.float64) for g in grid)
        # NumbaInterpolator stores values as contiguous float64 (interpolators.py:315)
        self.values = {c: (None if values.get(c) is None
                           else np.ascontiguousarray(values[c], dtype=np.float64))
                       for c in "xyz"}
        self.scaling = scaling

    def __call__(self, pts):
        pts = np.atleast_2d(pts)
        cols = []
        for c in "xyz":
            if self.values[c] is None:
                cols.append(self.scaling * np.zeros(pts.shape[0]))
            elif len(self.grid) == 1:
                cols.append(self.scaling * interp1d(pts[:, 2], self.grid, self.values[c]))
            elif len(self.grid) == 2:
                cols.append(self.scaling * interp2d(pts[:, 0], pts[:, 1], self.grid, self.values[c]))
            else:
                cols.append(self.scaling * interp3d(pts, self.grid, self.values[c]))
        return np.column_stack(cols)


class ConstField:
    """0D field (field.py:441-455)."""

    def __init__(self, vec, scaling=1.0):
        self.vec = np.asarray(vec, dtype=np.float64)
        self.scaling = scaling

    def __call__(self, pts):
        m = np.atleast_2d(pts).shape[0]
        return np.column_stack([self.scaling * self.vec[c] * np.ones(m) for c in range(3)])


class ZeroField(ConstField):
    """Field.zero(): zero everywhere (field.py:389-407)."""

    def __init__(self):
        super().__init__([0.0, 0.0, 0.0])


class ScaledOracleField:
    """scale * F + offset (field.py:661-690)."""

    def __init__(self, field, scale=1.0, offset=0.0):
        self.field, self.scale, self.offset = field, scale, offset

    def __call__(self, pts):
        return self.scale * self.field(pts) + self.offset


class CompositeOracleField:
    """sum_i w_i F_i accumulated into a zeroed (M,3) array (field.py:626-655)."""

    def __init__(self, fields, weights):
        self.fields = list(fields)
        self.weights = np.asarray(weights, dtype=np.float64)

    def __call__(self, pts):
        pts = np.atleast_2d(pts)
        total = np.zeros((pts.shape[0], 3))
        for f, w in zip(self.fields, self.weights):
            total += w * f(pts)
        return total


# ---------------------------------------------------------------------------
# Push kernels  (pusher.py:74-423), vectorised over rows
# ---------------------------------------------------------------------------

def _cross(a, b):
    """pusher.py:99-106"""
    return np.stack([a[:, 1] * b[:, 2] - a[:, 2] * b[:, 1],
                     a[:, 2] * b[:, 0] - a[:, 0] * b[:, 2],
                     a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]], axis=1)


def _dot(a, b):
    return a[:, 0] * b[:, 0] + a[:, 1] * b[:, 1] + a[:, 2] * b[:, 2]


def relativistic_gamma(v):
    """pusher.py:74-96: gamma with beta^2 clamped to 0.9999."""
    beta_sq = (v[:, 0] ** 2 + v[:, 1] ** 2 + v[:, 2] ** 2) / CLIGHT ** 2
    beta_sq = np.where(beta_sq >= 0.9999, 0.9999, beta_sq)
    return 1.0 / np.sqrt(1.0 - beta_sq)


def boris_push(v, e, b, dt, qm):
    """Non-relativistic Boris v-update, pusher.py:124-165."""
    v_minus = v + 0.5 * qm * e * dt
    t = 0.5 * qm * b * dt
    t_sq = t[:, 0] ** 2 + t[:, 1] ** 2 + t[:, 2] ** 2
    s = 2.0 * t / (1.0 + t_sq)[:, None]
    v_prime = v_minus + _cross(v_minus, t)
    v_plus = v_minus + _cross(v_prime, s)
    return v_plus + 0.5 * qm * e * dt


def _clamp_speed(v):
    """|v| >= 0.9999 c  ->  rescale to 0.9999 c (pusher.py:275-277, :886-890)."""
    vmag = np.sqrt(v[:, 0] ** 2 + v[:, 1] ** 2 + v[:, 2] ** 2)
    over = vmag >= 0.9999 * CLIGHT
    if np.any(over):
        v = v.copy()
        v[over] *= (0.9999 * CLIGHT / vmag[over])[:, None]
    return v


def vay_rel_push(v, e, b, dt, qm):
    """The reference's 'vay_rel' exactly as written, pusher.py:216-279."""
    gamma_n = relativistic_gamma(v)
    u_n = gamma_n[:, None] * v
    tau = 0.5 * qm * b * dt
    u_prime = u_n + qm * e * dt
    u_prime_mag = np.sqrt(u_prime[:, 0] ** 2 + u_prime[:, 1] ** 2 + u_prime[:, 2] ** 2)
    tau_mag = np.sqrt(tau[:, 0] ** 2 + tau[:, 1] ** 2 + tau[:, 2] ** 2)
    u_dot_tau = _dot(u_prime, tau)
    g_inv_sq = 1.0 - (u_prime_mag / CLIGHT) ** 2
    g_inv_sq = np.where(g_inv_sq < 1e-10, 1e-10, g_inv_sq)
    sigma = g_inv_sq - tau_mag ** 2
    gamma_new = np.sqrt(0.5 * (sigma + np.sqrt(sigma ** 2 + 4.0 * (tau_mag ** 2 + (u_dot_tau / CLIGHT) ** 2))))
    t = tau / gamma_new[:, None]
    s = 2.0 * t / (1.0 + tau_mag ** 2 / gamma_new ** 2)[:, None]
    u_star = u_prime + _cross(u_prime, t)
    u_new = u_prime + _cross(u_star, s)
    return _clamp_speed(u_new / gamma_new[:, None])


def lorentz_accel(v, e, b, qm):
    """q/m (E + v x B): pusher.py:113-121, :168-172, :826-829."""
    return qm * (e + _cross(v, b))


def rk4_rel_deriv(v, e, b, qm):
    """pusher.py:282-298: F/gamma - (v.F) v / (gamma c^2), F = q/m (E + v x B)."""
    gamma = relativistic_gamma(v)
    force = qm * (e + _cross(v, b))
    v_dot_f = _dot(v, force)
    correction = (v_dot_f / (gamma * CLIGHT ** 2))[:, None] * v
    return force / gamma[:, None] - correction


YOSHIDA_C1 = 1.0 / (2.0 - 2.0 ** (1.0 / 3.0))
YOSHIDA_C2 = -2.0 ** (1.0 / 3.0) / (2.0 - 2.0 ** (1.0 / 3.0))
YOSHIDA_C3 = YOSHIDA_C1
YOSHIDA_D1 = 2.0 * YOSHIDA_C1
YOSHIDA_D2 = -(2.0 ** (1.0 / 3.0) + 1.0) / (2.0 - 2.0 ** (1.0 / 3.0))
YOSHIDA_D3 = YOSHIDA_D1


def yoshida_push(r, v, e, b, dt, qm, rel):
    """pusher.py:184-209 (non-rel) and :332-362 (rel); fields frozen at the
    step start (push_batch evaluates them once, pusher.py:726-727)."""
    accel = rk4_rel_deriv if rel else lorentz_accel
    for c, d in ((YOSHIDA_C1, YOSHIDA_D1), (YOSHIDA_C2, YOSHIDA_D2), (YOSHIDA_C3, YOSHIDA_D3)):
        v = v + c * dt * accel(v, e, b, qm)
        r = r + d * dt * v
    if rel:
        v = _clamp_speed(v)
    return r, v


# ---------------------------------------------------------------------------
# Relativistic pushers that the reference lacks (u = gamma v state)
# ---------------------------------------------------------------------------

def gamma_from_u(u):
    return np.sqrt(1.0 + _dot(u, u) / CLIGHT ** 2)


def u_from_v(v):
    """Exact (unclamped) u = gamma v for |v| < c."""
    return v / np.sqrt(1.0 - _dot(v, v) / CLIGHT ** 2)[:, None]


def v_from_u(u):
    return u / gamma_from_u(u)[:, None]


def boris_rel_push_u(u, e, b, dt, qm):
    """Relativistic Boris (Boris 1970; Birdsall & Langdon 15-4) in u space."""
    u_minus = u + 0.5 * qm * dt * e
    g = gamma_from_u(u_minus)
    t = (0.5 * qm * dt) * b / g[:, None]
    t_sq = _dot(t, t)
    s = 2.0 * t / (1.0 + t_sq)[:, None]
    u_prime = u_minus + _cross(u_minus, t)
    u_plus = u_minus + _cross(u_prime, s)
    return u_plus + 0.5 * qm * dt * e


def vay_push_u(u, e, b, dt, qm):
    """Vay, Phys. Plasmas 15, 056701 (2008), eqs. (9)-(11), in u space."""
    g_old = gamma_from_u(u)
    v_old = u / g_old[:, None]
    u_prime = u + qm * dt * (e + 0.5 * _cross(v_old, b))
    tau = (0.5 * qm * dt) * b
    tau_sq = _dot(tau, tau)
    u_star = _dot(u_prime, tau) / CLIGHT
    sigma = 1.0 + _dot(u_prime, u_prime) / CLIGHT ** 2 - tau_sq
    g_new = np.sqrt(0.5 * (sigma + np.sqrt(sigma ** 2 + 4.0 * (tau_sq + u_star ** 2))))
    t = tau / g_new[:, None]
    s = 1.0 / (1.0 + _dot(t, t))
    return s[:, None] * (u_prime + _dot(u_prime, t)[:, None] * t + _cross(u_prime, t))


# ---------------------------------------------------------------------------
# Step and track drivers  (pusher.py:699-1012)
# ---------------------------------------------------------------------------

class _Fields:
    """Field evaluation with the optional RF factor on E."""

    def __init__(self, efield, bfield, rf=None):
        self.efield, self.bfield = efield, bfield
        self.rf = rf  # (omega, phase (M,)) or None

    def subset(self, rows):
        """The same fields for the particles ``rows`` (their RF phases)."""
        if self.rf is None:
            return self
        return _Fields(self.efield, self.bfield, (self.rf[0], self.rf[1][rows]))

    def __call__(self, r, t):
        e = self.efield(r)
        if self.rf is not None:
            omega, phase = self.rf
            e = e * np.cos(omega * t + phase)[:, None]
        return e, self.bfield(r)


def rk4_step(r, v, fields, t, dt, qm, rel):
    """pusher.py:803-892 with stage field times t, t+dt/2, t+dt/2, t+dt.
    ``dt`` may hold one value per particle: the reference broadcasts such an
    array over each particle's three components (pusher.py:815-816)."""
    deriv = rk4_rel_deriv if rel else lorentz_accel
    ts = dt
    if np.ndim(dt) == 1:
        dt = np.asarray(dt, dtype=np.float64)[:, None]
    e1, b1 = fields(r, t)
    k1_v = deriv(v, e1, b1, qm)
    k1_r = v.copy()
    r2 = r + 0.5 * dt * k1_r
    v2 = v + 0.5 * dt * k1_v
    e2, b2 = fields(r2, t + 0.5 * ts)
    k2_v = deriv(v2, e2, b2, qm)
    k2_r = v2.copy()
    r3 = r + 0.5 * dt * k2_r
    v3 = v + 0.5 * dt * k2_v
    e3, b3 = fields(r3, t + 0.5 * ts)
    k3_v = deriv(v3, e3, b3, qm)
    k3_r = v3.copy()
    r4 = r + dt * k3_r
    v4 = v + dt * k3_v
    e4, b4 = fields(r4, t + ts)
    k4_v = deriv(v4, e4, b4, qm)
    k4_r = v4.copy()
    r_new = r + (dt / 6.0) * (k1_r + 2.0 * k2_r + 2.0 * k3_r + k4_r)
    v_new = v + (dt / 6.0) * (k1_v + 2.0 * k2_v + 2.0 * k3_v + k4_v)
    if rel:
        v_new = _clamp_speed(v_new)
    return r_new, v_new


def push_step(alg, r, w, fields, t, dt, qm):
    """One push_batch step (pusher.py:699-801).  ``w`` is v, or u for the
    u-state algorithms."""
    if alg in ("rk4", "rk4_rel"):
        return rk4_step(r, w, fields, t, dt, qm, alg == "rk4_rel")
    e, b = fields(r, t)
    if alg == "leapfrog":
        w_new = w + lorentz_accel(w, e, b, qm) * dt
        return r + w_new * dt, w_new
    if alg == "boris":
        w_new = boris_push(w, e, b, dt, qm)
        return r + w_new * dt, w_new
    if alg == "vay_rel":
        w_new = vay_rel_push(w, e, b, dt, qm)
        return r + w_new * dt, w_new
    if alg in ("yoshida", "yoshida_rel"):
        return yoshida_push(r, w, e, b, dt, qm, alg == "yoshida_rel")
    if alg == "boris_rel":
        w_new = boris_rel_push_u(w, e, b, dt, qm)
        return r + v_from_u(w_new) * dt, w_new
    if alg == "vay":
        w_new = vay_push_u(w, e, b, dt, qm)
        return r + v_from_u(w_new) * dt, w_new
    raise ValueError(f"unknown algorithm {alg!r}")


U_STATE = ("boris_rel", "vay")
STAGGERED = ("boris", "boris_rel", "vay")


def _half_kick(alg, w, e, b, dt, qm):
    if alg == "boris":
        return boris_push(w, e, b, dt, qm)
    if alg == "boris_rel":
        return boris_rel_push_u(w, e, b, dt, qm)
    return vay_push_u(w, e, b, dt, qm)


# ---------------------------------------------------------------------------
# Electrode surfaces  (pusher.py:966-990; the segment test the external
# py_electrodes package provides, restated as Moller-Trumbore)
# ---------------------------------------------------------------------------

def segments_hit(p0, p1, vertices, triangles, chunk=4096):
    """hit[i]: does the segment p0[i] -> p1[i] meet a triangle?  Moller-Trumbore
    (J. Graphics Tools 2(1), 1997) with the segment parameter 0 <= t <= 1 and
    triangle edges included; every product and sum rounded separately, in the
    order of the device code, so the decisions are the same bit for bit."""
    p0 = np.asarray(p0, dtype=np.float64).reshape(-1, 3)
    p1 = np.asarray(p1, dtype=np.float64).reshape(-1, 3)
    v = np.asarray(vertices, dtype=np.float64)
    t = np.asarray(triangles, dtype=np.int64)
    v0 = v[t[:, 0]]
    e1 = v[t[:, 1]] - v0
    e2 = v[t[:, 2]] - v0
    hit = np.zeros(p0.shape[0], dtype=bool)

    def cross(a, b):
        return np.stack([a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1],
                         a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                         a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]], axis=-1)

    def dot(a, b):
        return a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1] + a[..., 2] * b[..., 2]

    for s in range(0, p0.shape[0], chunk):
        a = p0[s:s + chunk, None, :]
        d = (p1[s:s + chunk] - p0[s:s + chunk])[:, None, :]
        pv = cross(d, e2[None])
        det = dot(e1[None], pv)
        with np.errstate(divide="ignore", invalid="ignore"):
            inv = 1.0 / det
            tv = a - v0[None]
            u = dot(tv, pv) * inv
            qv = cross(tv, e1[None])
            w = dot(d, qv) * inv
            tt = dot(e2[None], qv) * inv
            ok = (det != 0.0) & (u >= 0.0) & (u <= 1.0) & (w >= 0.0) & (u + w <= 1.0) & (tt >= 0.0) & (tt <= 1.0)
        hit[s:s + chunk] = ok.any(axis=1)
    return hit


def track_batch(alg, qm, r0, v0, efield, bfield, nsteps, dt, rec_every_n_steps=1,
                rf=None, t0=0.0, surface=None):
    """pusher.py:894-1012.  Returns (r_hist, v_hist, active) with the
    reference's shapes.

    ``rf=(omega, phase)`` multiplies E by cos(omega t + phase_i).  Field time
    of step n is t0 + n dt; the Boris-family initial half step uses t0 and the
    final one t0 + nsteps dt.  ``surface=(vertices, triangles)``: after each
    step (and its record) the active particles whose step segment meets the
    surface are deactivated; they are pushed and recorded no more, and the
    closing half step skips them (pusher.py:966-1007).
    """
    if surface is not None:
        return _track_batch_surface(alg, qm, r0, v0, efield, bfield, nsteps, dt, rec_every_n_steps, rf, t0,
                                    surface)
    m = r0.shape[0]
    n_rec = nsteps // rec_every_n_steps + 1
    r_hist = np.full((n_rec, m, 3), np.nan)
    v_hist = np.full((n_rec, m, 3), np.nan)
    active = np.ones(m, dtype=bool)
    fields = _Fields(efield, bfield, rf)
    r = np.array(r0, dtype=np.float64, copy=True)
    w = np.array(v0, dtype=np.float64, copy=True)
    if alg in U_STATE:
        w = u_from_v(w)
    as_v = v_from_u if alg in U_STATE else (lambda x: x)
    if alg in STAGGERED:
        e, b = fields(r, t0)
        w = _half_kick(alg, w, e, b, -0.5 * dt, qm)
    r_hist[0] = r
    v_hist[0] = as_v(w)
    rec = 1
    for step in range(nsteps):
        r, w = push_step(alg, r, w, fields, t0 + step * dt, dt, qm)
        if (step + 1) % rec_every_n_steps == 0 and rec < n_rec:
            r_hist[rec] = r
            v_hist[rec] = as_v(w)
            rec += 1
    if alg in STAGGERED:
        e, b = fields(r, t0 + nsteps * dt)
        w = _half_kick(alg, w, e, b, 0.5 * dt, qm)
        v_hist[-1] = as_v(w)
    return r_hist, v_hist, active


def _track_batch_surface(alg, qm, r0, v0, efield, bfield, nsteps, dt, rec_every_n_steps, rf, t0, surface):
    vertices, triangles = surface
    m = r0.shape[0]
    n_rec = nsteps // rec_every_n_steps + 1
    r_hist = np.full((n_rec, m, 3), np.nan)
    v_hist = np.full((n_rec, m, 3), np.nan)
    active = np.ones(m, dtype=bool)
    fields = _Fields(efield, bfield, rf)
    r = np.array(r0, dtype=np.float64, copy=True)
    w = np.array(v0, dtype=np.float64, copy=True)
    if alg in U_STATE:
        w = u_from_v(w)
    as_v = v_from_u if alg in U_STATE else (lambda x: x)
    if alg in STAGGERED:
        e, b = fields(r, t0)
        w = _half_kick(alg, w, e, b, -0.5 * dt, qm)
    r_hist[0] = r
    v_hist[0] = as_v(w)
    rec = 1
    for step in range(nsteps):
        rows = np.nonzero(active)[0]
        if rows.size == 0:
            break
        r_old = r[rows].copy()
        r[rows], w[rows] = push_step(alg, r[rows], w[rows], fields.subset(rows), t0 + step * dt, dt, qm)
        if (step + 1) % rec_every_n_steps == 0 and rec < n_rec:
            r_hist[rec][rows] = r[rows]
            v_hist[rec][rows] = as_v(w[rows])
            rec += 1
        active[rows[segments_hit(r_old, r[rows], vertices, triangles)]] = False
    rows = np.nonzero(active)[0]
    if alg in STAGGERED and rows.size:
        e, b = fields.subset(rows)(r[rows], t0 + nsteps * dt)
        w[rows] = _half_kick(alg, w[rows], e, b, 0.5 * dt, qm)
        v_hist[-1][rows] = as_v(w[rows])
    return r_hist, v_hist, active


def track_single(alg, qm, r0, v0, efield, bfield, nsteps, dt, rec_every_n_steps=1):
    """Pusher.track (pusher.py:620-693): one particle, zero-initialised
    (n_rec, 3) histories.  Same per-step arithmetic as the batch path."""
    rh, vh, _ = track_batch(alg, qm, np.asarray(r0, float).reshape(1, 3),
                            np.asarray(v0, float).reshape(1, 3), efield, bfield,
                            nsteps, dt, rec_every_n_steps)
    return rh[:, 0, :], vh[:, 0, :]


# ---------------------------------------------------------------------------
# Boundary conversions and bunch moments  (particles.py:44-117, :693-788)
# ---------------------------------------------------------------------------

def momenta_from_velocities(v):
    """Per-component v -> beta*gamma (particles.py:94-117; relativistic)."""
    v_sq = v ** 2
    v_sq = np.where(v_sq >= CLIGHT ** 2, 0.99999 * CLIGHT ** 2, v_sq)
    return v / np.sqrt(CLIGHT ** 2 - v_sq)


def velocities_from_momenta(p):
    """Per-component beta*gamma -> v (particles.py:71-91; relativistic)."""
    return CLIGHT * p / np.sqrt(p ** 2 + 1.0)


def kinetic_energies(p, mass_mev):
    """particles.py:44-68 with Z_ENERGY False, RELATIVISTIC True."""
    pr = np.sqrt(p[:, 0] ** 2 + p[:, 1] ** 2 + p[:, 2] ** 2)
    return np.sqrt((pr * mass_mev) ** 2 + mass_mev ** 2) - mass_mev


def bunch_moments(x, p, mass_mev):
    """The ParticleDistribution statistics (particles.py:693-719, :761-788,
    :600-605, :701-705) for positions x (N,3) [m] and momenta p (N,3)
    [beta*gamma].  Returns a dict of float64 values."""
    v = velocities_from_momenta(p)
    vz_safe = np.where(np.abs(v[:, 2]) < 1e-10, 1e-10, v[:, 2])
    xp = v / vz_safe[:, None]
    centroid = np.mean(x, axis=0)
    x_std = np.std(x, axis=0)
    xp_std = np.std(xp, axis=0)
    xp_mean = np.mean(xp, axis=0)
    xxp = np.mean((x[:, 0] - centroid[0]) * (xp[:, 0] - xp_mean[0]))
    yyp = np.mean((x[:, 1] - centroid[1]) * (xp[:, 1] - xp_mean[1]))
    xyp = np.mean((x[:, 0] - centroid[0]) * (xp[:, 1] - xp_mean[1]))
    yxp = np.mean((x[:, 1] - centroid[1]) * (xp[:, 0] - xp_mean[0]))
    mean_p = np.mean(np.linalg.norm(p, axis=1))
    e_raw = np.array([
        (x_std[0] * xp_std[0]) ** 2 - xxp ** 2,
        (x_std[1] * xp_std[1]) ** 2 - yyp ** 2,
        (x_std[0] * xp_std[1]) ** 2 - xyp ** 2,
        (x_std[1] * xp_std[0]) ** 2 - yxp ** 2])
    with np.errstate(invalid="ignore"):
        emit = np.sqrt(e_raw)
    ek = kinetic_energies(p, mass_mev)
    return {
        "centroid": centroid, "mean_momentum": np.mean(p, axis=0),
        "x_std": x_std, "xp_std": xp_std, "xp_mean": xp_mean,
        "xxp": xxp, "yyp": yyp, "xyp": xyp, "yxp": yxp,
        "mean_p": mean_p, "emittance": emit, "emittance_n": emit * mean_p,
        "ekin_mean": np.mean(ek), "ekin_std": np.std(ek),
    }
