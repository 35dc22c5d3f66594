"""Physics known-answer tests and invariances of the GPU path (the reference
has no tests for its pushers; these are the analytic checks the path must
satisfy): |v| or |u| conservation in a pure magnetic field, gyro-radius,
E x B drift, trilinear exactness on linear fields, and bitwise invariance of
each particle's result under chunking and cell re-sorting."""
import numpy as np
import pytest

from pypatools_b200 import PusherGPU, Field, IonSpecies, workloads
from pypatools_b200.constants import CLIGHT
from tests.helpers import gpu_fields

pytestmark = pytest.mark.gpu


def _uniform_b(bz, half=10.0, nodes=5):
    g = np.linspace(-half, half, nodes)
    shape = (nodes,) * 3
    return Field.from_arrays({"x": g, "y": g, "z": g},
                             {"x": np.zeros(shape), "y": np.zeros(shape), "z": np.full(shape, bz)})


def _beam(n, speed, seed=1):
    rng = np.random.default_rng(seed)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    return rng.uniform(-0.01, 0.01, (n, 3)), d * speed


def test_boris_speed_conserved_in_pure_b(cuda):
    ion = IonSpecies("proton")
    r0, v0 = _beam(512, 1.0e7)
    _, vh, _ = PusherGPU(ion, "boris").track_batch(r0, v0, Field.zero(3), _uniform_b(1.0), 5000, 1e-11, 5000)
    s0 = np.linalg.norm(vh[0], axis=1)
    s1 = np.linalg.norm(vh[-1], axis=1)
    assert np.max(np.abs(s1 / s0 - 1.0)) < 5e-14


@pytest.mark.parametrize("alg", ["boris_rel", "vay"])
def test_u_conserved_in_pure_b_relativistic(cuda, alg):
    ion = IonSpecies("electron")
    r0, v0 = _beam(512, 0.998 * CLIGHT)
    g0 = 1.0 / np.sqrt(1.0 - 0.998 ** 2)
    _, vh, _ = PusherGPU(ion, alg).track_batch(r0, v0, Field.zero(3), _uniform_b(0.05), 10000, 1e-12, 10000)
    # gamma from |v| of the snapshots; |u| = gamma |v| must stay put
    v = np.linalg.norm(vh[-1], axis=1)
    u = v / np.sqrt(1.0 - (v / CLIGHT) ** 2)
    u0 = g0 * 0.998 * CLIGHT
    assert np.max(np.abs(u / u0 - 1.0)) < 1e-9   # conversion v <-> u in the check costs ~gamma^2 eps


def test_gyro_radius_uniform_b(cuda):
    ion = IonSpecies("proton")
    v_perp = 2.0e6
    bz = 0.5
    n_steps = 4000                     # period 1.31e-7 s = 1310 steps of 1e-10 s: three orbits
    r0 = np.zeros((1, 3))
    v0 = np.array([[v_perp, 0.0, 0.0]])
    rh, _, _ = PusherGPU(ion, "boris").track_batch(r0, v0, Field.zero(3), _uniform_b(bz), n_steps, 1e-10, 1)
    radius = v_perp / (abs(ion.q_over_m) * bz)
    xy = rh[:, 0, :2]
    center = 0.5 * (xy.max(axis=0) + xy.min(axis=0))
    rr = np.linalg.norm(xy - center, axis=1)
    assert abs(rr.mean() / radius - 1.0) < 1e-4


def test_e_cross_b_drift(cuda):
    ion = IonSpecies("proton")
    e0, b0 = 1.0e5, 1.0
    e = Field(dim=0, field={"x": e0, "y": 0.0, "z": 0.0})
    b = Field(dim=0, field={"x": 0.0, "y": 0.0, "z": b0})
    period = 2 * np.pi / (ion.q_over_m * b0)
    dt = period / 400
    steps = 400 * 20
    rh, _, _ = PusherGPU(ion, "boris").track_batch(np.zeros((1, 3)), np.zeros((1, 3)), e, b, steps, dt, 400)
    drift = (rh[-1, 0] - rh[0, 0]) / (steps * dt)
    # E x B / B^2 = (Ex x Bz)/B^2 = -Ex/Bz y-hat
    assert abs(drift[1] / (-e0 / b0) - 1.0) < 1e-3
    assert abs(drift[0]) < 1e-3 * e0 / b0


def test_trilinear_exact_on_linear_field(cuda):
    g = np.linspace(-1.0, 2.0, 7)
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    f = Field.from_arrays({"x": g, "y": g, "z": g}, {"x": 1 + 2 * X - Y + 0.5 * Z, "y": X * 0 + 3.0, "z": -Z})
    rng = np.random.default_rng(3)
    pts = rng.uniform(-1.0, 2.0, (1000, 3))
    out = f(pts)
    np.testing.assert_allclose(out[:, 0], 1 + 2 * pts[:, 0] - pts[:, 1] + 0.5 * pts[:, 2], rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(out[:, 2], -pts[:, 2], rtol=1e-13, atol=1e-13)
    outside = f(np.array([[2.5, 0.0, 0.0], [0.0, -1.0 - 1e-12, 0.0]]))
    np.testing.assert_array_equal(outside, 0.0)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("nsteps", [300, 1100])
def test_chunking_and_sorting_are_bitwise_invariant(cuda, precision, nsteps):
    # 1100 steps: the protons leave the map after about 360, so the field-free
    # runs (and, in the mixed form, their whole-cell carries) are split by the
    # launch boundaries differently in each schedule
    wl = workloads.quad_solenoid_protons(n=3000, nsteps=nsteps)
    e, b = gpu_fields(wl)
    base = PusherGPU(wl.species, "boris", precision=precision).track_batch(wl.r0, wl.v0, e, b, nsteps, wl.dt, 50)
    chunked = PusherGPU(wl.species, "boris", precision=precision, steps_per_launch=7).track_batch(
        wl.r0, wl.v0, e, b, nsteps, wl.dt, 50)
    sorted_ = PusherGPU(wl.species, "boris", precision=precision, sort_every=40).track_batch(
        wl.r0, wl.v0, e, b, nsteps, wl.dt, 50)
    for other in (chunked, sorted_):
        np.testing.assert_array_equal(base[0], other[0])
        np.testing.assert_array_equal(base[1], other[1])
    if nsteps > 400:
        assert np.all(np.abs(base[0][-1, :, 2]) > 0.05)   # every proton ended outside the map


def test_nonfinite_input_warns(cuda):
    wl = workloads.quad_solenoid_protons(n=4)
    e, b = gpu_fields(wl)
    r0 = wl.r0.copy()
    r0[1, 0] = np.nan
    with pytest.warns(RuntimeWarning, match="non-finite"):
        rh, _, _ = PusherGPU(wl.species, "boris").track_batch(r0, wl.v0, e, b, 5, wl.dt)
    assert np.isnan(rh[-1, 1, 0]) and np.isfinite(rh[-1, 0]).all()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_row_order_restored_after_the_bunch_leaves(cuda, precision):
    """The launch schedule sorts the RF-gap bunch by cell while it crosses the
    map, then puts it back in row order (ppt_restore_order) once a launch met
    no map: the histories, the final state and the RF phases are those of the
    unsorted run, bit for bit."""
    import torch
    from pypatools_b200.device_fields import DeviceFields
    from pypatools_b200.pusher import DeviceTracker
    dev = torch.device("cuda", 0)
    n, nsteps = 4096, 2500
    wl = workloads.rf_gap_protons(n=n, nsteps=nsteps, nodes=64, rec_every=100)
    g = {"x": wl.grid[0], "y": wl.grid[1], "z": wl.grid[2]}
    df = DeviceFields(Field.from_arrays(g, wl.e_values), Field.from_arrays(g, wl.b_values), precision, dev)
    r0 = torch.from_numpy(wl.r0).to(dev)
    v0 = torch.from_numpy(wl.v0).to(dev)
    out = {}
    for sort_every in (0, 100):
        tr = DeviceTracker("boris", wl.species.q_over_m, df, n, nsteps, wl.dt, wl.rec_every, precision,
                           rf_omega=2 * np.pi * wl.rf_frequency, rf_phase=torch.from_numpy(wl.rf_phase),
                           counters=True, device=dev)
        tr.load(r0, v0)
        tr.run(nsteps, 100, sort_every=sort_every, long_chunk=200)
        r = torch.empty_like(r0)
        v = torch.empty_like(v0)
        tr.store(r, v)
        torch.cuda.synchronize()
        out[sort_every] = (tr.r_hist.cpu(), tr.v_hist.cpu(), r.cpu(), v.cpu(), tr.rf_phase.cpu(), tr)
    base, srt = out[0], out[100]
    tr = srt[5]
    assert tr.row_order and torch.equal(tr.order.cpu(), torch.arange(n))
    for a, b in zip(base[:5], srt[:5]):
        assert torch.equal(a, b)
    assert bool(torch.all(base[0][-1, :, 2] > wl.grid[2][-1]))     # every proton left through the far face
    # a second job on the same tracker starts from row order again
    tr.step = 0
    tr.load(r0, v0)
    assert tr.order is None and not tr.row_order


def _fma_exact(a, b, c):
    """a * b + c rounded once (float64), as the device's fma."""
    from fractions import Fraction
    s = Fraction(a) * Fraction(b) + Fraction(c)
    if s == 0:
        # an exact zero sum is -0 only when both addends are -0
        return -0.0 if (np.signbit(a) != np.signbit(b)) and np.signbit(c) else 0.0
    return float(s)


def test_f64_field_free_runs_are_stepwise_fma(cuda):
    """Outside the maps the float64 kernel takes a run of field-free steps a
    binade at a time (k D in one fused multiply-add, see drift_coord); the
    positions must be those of x <- fma(v, dt, x) at every step, bit for bit:
    coordinates crossing zero (many binades), z through powers of two, zero
    velocity components, and steps exactly halfway between two float64
    neighbours (round-half-even alternates)."""
    rng = np.random.default_rng(5)
    dt = 2.0 ** -33                      # v dt exact for the halfway cases below
    nsteps, rec = 2000, 500
    rows = []
    for i in range(40):                  # transverse coordinates crossing zero
        vx, vy = rng.choice([-1, 1], 2) * 10 ** rng.uniform(2, 5, 2)
        kx, ky = rng.uniform(0, 1500, 2)
        rows.append(([-vx * dt * kx, -vy * dt * ky, rng.uniform(0.06, 0.4)], [vx, vy, 10 ** rng.uniform(6, 7.3)]))
    for z in (0.0625, 0.125, 0.25, 0.5, 1.0):   # z starting on a power of two
        rows.append(([1e-3, -2e-3, z], [3e3, -1e4, 1.2e7]))
    rows.append(([0.0, -0.0, 0.07], [0.0, 0.0, 1e7]))          # zero velocity components
    rows.append(([0.75, -0.75, 0.08], [1 + 2.0 ** -21, -(1 + 2.0 ** -21), 1e7]))   # halfway, both signs
    rows.append(([0.3, 1e-9, 0.09], [(2 ** 18 + 0.5) * 2.0 ** -21, 5.0, 2e6]))     # halfway in [0.25, 0.5)
    r0 = np.array([r for r, _ in rows], dtype=np.float64)
    v0 = np.array([v for _, v in rows], dtype=np.float64)
    rh, vh, _ = PusherGPU(IonSpecies("proton"), "boris").track_batch(r0, v0, Field.zero(3), _uniform_b(1.0, half=0.05),
                                                                   nsteps, dt, rec)
    assert np.array_equal(vh[0], v0)     # outside the map: no kick
    for p in range(len(rows)):
        for a in range(3):
            x = float(r0[p, a])
            for s in range(1, nsteps + 1):
                x = _fma_exact(float(v0[p, a]), dt, x)
                if s % rec == 0:
                    got = float(rh[s // rec, p, a])
                    assert got == x and np.signbit(got) == np.signbit(x), (p, a, s, got, x)
