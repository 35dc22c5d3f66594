"""Electrode collision termination (pusher.py:966-1007): after each step and
its snapshot, the active particles whose step segment meets an electrode stop.

The reference takes the surfaces from the external py_electrodes package
(``PyElectrodeAssembly.segment_intersects_surface``), which is not installed
here, so parity with it is unpinned; the oracle restates the reference's
tracking logic around the call (tests pin that against the reference's
collision-free fixtures) and restates the segment test as Moller-Trumbore.
The GPU path must match the oracle: hit decisions bit for bit (the device test
rounds every operation like NumPy), trajectories to the 1e-10 bar, the NaN
pattern of stopped particles and the active mask exactly."""
import ctypes

import numpy as np
import pytest

from oracle import pusher_oracle as orc
from pypatools_b200 import _lib, workloads
from pypatools_b200.electrodes import ElectrodeSurface
from tests.helpers import oracle_fields, gpu_fields, half_width

TOL = 1e-10


def _beamline():
    """An aperture plate (hole radius 5 mm) at z = 3 cm inside a 12 mm beam pipe."""
    return ElectrodeSurface.aperture_plate(0.03, 0.005, 0.02, n_phi=48, n_r=3) + \
        ElectrodeSurface.tube(0.012, -0.05, 0.06, n_phi=48, n_z=22)


def _square():
    v = np.array([[-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0]], dtype=float)
    return v, np.array([[0, 1, 2], [0, 2, 3]])


def _probe_segments(rng, m=20000):
    """Random short and long segments around the beam line, plus designed
    edge cases: ending on the plate's plane, starting on it, lying in it."""
    p0 = np.column_stack([rng.uniform(-0.025, 0.025, m), rng.uniform(-0.025, 0.025, m),
                          rng.uniform(-0.06, 0.07, m)])
    step = rng.normal(0, 1, (m, 3)) * np.where(rng.uniform(size=(m, 1)) < 0.5, 1e-3, 2e-2)
    p1 = p0 + step
    extra0 = np.array([[0.01, 0.0, 0.02], [0.01, 0.0, 0.03], [0.01, 0.0, 0.03], [0.0, 0.0, 0.0],
                       [0.012, 0.0, 0.0]])
    extra1 = np.array([[0.01, 0.0, 0.03], [0.01, 0.0, 0.04], [0.015, 0.0, 0.03], [0.0, 0.0, 0.06],
                       [0.013, 0.0, 0.0]])
    return np.concatenate([p0, extra0]), np.concatenate([p1, extra1])


# ---------------------------------------------------------------------------
# CPU
# ---------------------------------------------------------------------------

def test_oracle_segment_test_known_cases():
    v, t = _square()
    p0 = np.array([[0, 0, -1], [0, 0, -1], [0, 0, 1], [0.5, 0.5, -1], [2, 0, -1], [0, 0, 0], [-1, -1, -1]],
                  dtype=float)
    p1 = np.array([[0, 0, 1], [0, 0, -0.1], [0, 0, 0], [0.5, 0.5, 1], [2, 0, 1], [1, 0, 0], [-1, -1, 1]],
                  dtype=float)
    # through; short of the plane; ending on it; through the shared edge;
    # beside it; lying in it (parallel: no hit); through a corner
    expect = [True, False, True, True, False, False, True]
    np.testing.assert_array_equal(orc.segments_hit(p0, p1, v, t), expect)


def test_oracle_surface_far_away_changes_nothing():
    wl = workloads.quad_solenoid_protons(n=64, nsteps=200, rec_every=50)
    e, b = oracle_fields(wl)
    far = ElectrodeSurface.aperture_plate(5.0, 0.1, 0.2)
    ref = orc.track_batch("boris", wl.species.q_over_m, wl.r0, wl.v0, e, b, 200, wl.dt, 50)
    got = orc.track_batch("boris", wl.species.q_over_m, wl.r0, wl.v0, e, b, 200, wl.dt, 50,
                          surface=(far.vertices, far.triangles))
    for a, c in zip(ref, got):
        np.testing.assert_array_equal(a, c)


def test_oracle_stopped_particles_freeze():
    wl = workloads.quad_solenoid_protons(n=256, nsteps=600, rec_every=50)
    e, b = oracle_fields(wl)
    s = _beamline()
    rh, vh, act = orc.track_batch("boris", wl.species.q_over_m, wl.r0, wl.v0, e, b, 600, wl.dt, 50,
                                  surface=(s.vertices, s.triangles))
    assert 0 < act.sum() < act.size
    # every stopped particle has NaN rows after its last record, including the
    # closing half step's v row; the active ones have none
    assert np.isnan(rh[-1][~act]).all() and not np.isnan(rh[-1][act]).any()
    assert np.isnan(vh[-1][~act]).all()


def test_surface_argument_checks_without_gpu():
    lib = _lib.load()
    h = ctypes.c_void_p()
    v = np.zeros((2, 3))
    t = np.zeros((1, 3), dtype=np.int64)
    assert lib.ppt_surface_create(2, v.ctypes.data, 1, t.ctypes.data, h) == -1
    v = np.zeros((3, 3))
    t = np.array([[0, 1, 3]], dtype=np.int64)
    assert lib.ppt_surface_create(3, v.ctypes.data, 1, t.ctypes.data, h) == -1
    assert b"out of range" in lib.ppt_last_error()
    with pytest.raises(ValueError):
        ElectrodeSurface(np.zeros((3, 3)), np.array([[0, 1, 5]]))
    with pytest.raises(NotImplementedError):
        ElectrodeSurface.from_assembly(object())


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------

@pytest.mark.gpu
def test_gpu_segment_test_matches_oracle_bitwise(cuda):
    s = _beamline()
    p0, p1 = _probe_segments(np.random.default_rng(3))
    got = s.segment_intersects_surface(p0, p1)["hit_mask"]
    ref = orc.segments_hit(p0, p1, s.vertices, s.triangles)
    np.testing.assert_array_equal(got, ref)
    assert 100 < ref.sum() < ref.size - 100
    v, t = _square()
    sq = ElectrodeSurface(v, t)
    p0 = np.array([[0, 0, -1], [0, 0, 1], [0.5, 0.5, -1], [0, 0, 0], [-1, -1, -1]], dtype=float)
    p1 = np.array([[0, 0, 1], [0, 0, 0], [0.5, 0.5, 1], [1, 0, 0], [-1, -1, 1]], dtype=float)
    np.testing.assert_array_equal(sq.segment_intersects_surface(p0, p1)["hit_mask"],
                                  [True, True, True, False, True])
    info = s.info()
    assert info["bytes"] > 0 and all(c >= 1 for c in info["cells"])


def _compare(got, ref, hw):
    rh, vh, act = got
    ro, vo, ao = ref
    np.testing.assert_array_equal(act, ao)
    np.testing.assert_array_equal(np.isnan(rh), np.isnan(ro))
    np.testing.assert_array_equal(np.isnan(vh), np.isnan(vo))
    ok = ~np.isnan(ro[..., 0])
    num = np.linalg.norm(rh[ok] - ro[ok], axis=1)
    assert float(np.max(num / np.maximum(np.linalg.norm(ro[ok], axis=1), hw))) < TOL
    ok = ~np.isnan(vo[..., 0])
    num = np.linalg.norm(vh[ok] - vo[ok], axis=1)
    assert float(np.max(num / np.linalg.norm(vo[ok], axis=1))) < TOL


@pytest.mark.gpu
@pytest.mark.parametrize("alg", ["boris", "rk4_rel", "vay_rel", "leapfrog"])
def test_gpu_track_with_surface_matches_oracle(cuda, alg):
    from pypatools_b200 import PusherGPU
    wl = workloads.quad_solenoid_protons(n=192, nsteps=400, rec_every=50)
    e, b = gpu_fields(wl)
    oe, ob = oracle_fields(wl)
    s = _beamline()
    got = PusherGPU(wl.species, alg, electrode_assembly=s).track_batch(wl.r0, wl.v0, e, b, 400, wl.dt, 50)
    ref = orc.track_batch(alg, wl.species.q_over_m, wl.r0, wl.v0, oe, ob, 400, wl.dt, 50,
                          surface=(s.vertices, s.triangles))
    assert 0 < ref[2].sum() < ref[2].size
    _compare(got, ref, half_width(wl))


@pytest.mark.gpu
def test_gpu_surface_chunking_and_sorting_bitwise_invariant(cuda):
    from pypatools_b200 import PusherGPU
    wl = workloads.quad_solenoid_protons(n=3000, nsteps=500, rec_every=50)
    e, b = gpu_fields(wl)
    s = _beamline()
    base = PusherGPU(wl.species, "boris", electrode_assembly=s).track_batch(wl.r0, wl.v0, e, b, 500, wl.dt, 50)
    for kw in ({"steps_per_launch": 7}, {"sort_every": 40}):
        other = PusherGPU(wl.species, "boris", electrode_assembly=s, **kw).track_batch(wl.r0, wl.v0, e, b, 500,
                                                                                        wl.dt, 50)
        for a, c in zip(base, other):
            np.testing.assert_array_equal(a, c)


@pytest.mark.gpu
def test_gpu_surface_api_edges(cuda):
    from pypatools_b200 import PusherGPU
    wl = workloads.quad_solenoid_protons(n=16, nsteps=300, rec_every=100)
    e, b = gpu_fields(wl)
    s = _beamline()
    with pytest.raises(NotImplementedError):
        PusherGPU(wl.species, "rk4", electrode_assembly=s, precision="mixed")
    p = PusherGPU(wl.species, "boris", electrode_assembly=s)
    # the single-particle track makes no collision test in the reference
    rh, _ = p.track(wl.r0[0], wl.v0[0], e, b, 300, wl.dt, 100)
    assert not np.isnan(rh).any()
    # snapshots on the device keep the NaN rows of stopped particles too
    p.snapshot = "device"
    rh_d, vh_d, act = p.track_batch(wl.r0, wl.v0, e, b, 300, wl.dt, 100)
    p.snapshot = "host"
    rh_h, vh_h, act_h = p.track_batch(wl.r0, wl.v0, e, b, 300, wl.dt, 100)
    np.testing.assert_array_equal(rh_d.cpu().numpy(), rh_h)
    np.testing.assert_array_equal(act, act_h)
    # as the reference, change_algorithm drops the electrode assembly
    p.change_algorithm("rk4")
    assert p.surface is None


@pytest.mark.gpu
def test_gpu_mixed_boris_with_surface_vs_float64(cuda):
    # the mixed form tests its float64 positions (cell + float32 offset), so
    # grazing hits may differ from the float64 form's; the stops agree for all
    # but a few particles and the others' tracks agree to the mixed form's bar
    from pypatools_b200 import PusherGPU
    wl = workloads.quad_solenoid_protons(n=4000, nsteps=600, rec_every=50)
    e, b = gpu_fields(wl)
    s = _beamline()
    out = {}
    for prec in ("fp64", "mixed"):
        out[prec] = PusherGPU(wl.species, "boris", electrode_assembly=s, precision=prec).track_batch(
            wl.r0, wl.v0, e, b, 600, wl.dt, 50)
    (r64, v64, a64), (rmx, vmx, amx) = out["fp64"], out["mixed"]
    assert 0 < a64.sum() < a64.size
    differ = a64 != amx
    assert differ.sum() <= 0.005 * a64.size, int(differ.sum())
    same = ~differ
    np.testing.assert_array_equal(np.isnan(rmx[:, same]), np.isnan(r64[:, same]))
    ok = ~np.isnan(r64[:, same, 0])
    num = np.linalg.norm(rmx[:, same][ok] - r64[:, same][ok], axis=1)
    assert float(np.max(num / np.maximum(np.linalg.norm(r64[:, same][ok], axis=1), half_width(wl)))) < 1e-5
    # chunking does not change the mixed form's stops
    chunked = PusherGPU(wl.species, "boris", electrode_assembly=s, precision="mixed",
                        steps_per_launch=7).track_batch(wl.r0, wl.v0, e, b, 600, wl.dt, 50)
    for a, c in zip(out["mixed"], chunked):
        np.testing.assert_array_equal(a, c)


def _mesh_grid(vertices, n_tri):
    """The cell grid the library lays over a mesh (surface.cu, grid_for_mesh):
    origin and cell size per axis."""
    lo_in, hi_in = vertices.min(axis=0), vertices.max(axis=0)
    big = float(np.max(hi_in - lo_in))
    pad = max(big * 1e-9, 1e-30)
    lo = lo_in - pad
    ext = (hi_in + pad) - lo
    side = np.cbrt(np.prod(ext) / max(1.0, 2.0 * n_tri))
    dims = np.clip(np.ceil(ext / side), 1, 256)
    return lo, ext / dims, dims.astype(int)


@pytest.mark.gpu
def test_gpu_triangles_on_cell_faces_match_oracle_bitwise(cuda):
    """The mesh is binned into cells; the segment test works on v0 and the
    rounded edge vectors, whose hits can lie an ulp outside the vertices' box.
    Triangles with vertices exactly on cell faces (tilted, so the test's
    arithmetic rounds) and short segments starting or ending on those faces
    and a few ulps around them: the GPU's decisions must equal the oracle's,
    which tests every triangle."""
    rng = np.random.default_rng(17)
    # a frame of 8 points fixes the mesh box, then 400 tilted triangles inside it
    frame = np.array([[x, y, z] for x in (0.0, 1.0) for y in (0.0, 1.0) for z in (0.0, 1.0)])
    n_tri = 402
    lo, h, dims = _mesh_grid(frame, n_tri)
    faces = [lo[a] + h[a] * np.arange(1, dims[a]) for a in range(3)]
    tris, verts = [], [frame]
    base = len(frame)
    for t in range(n_tri - 2):
        a = t % 3
        f = rng.choice(faces[a])
        v = rng.uniform(0.05, 0.95, (3, 3))
        v[:, a] = f + rng.normal(0, 0.3, 3) * h[a]
        v[rng.integers(0, 3), a] = f                            # one vertex exactly on the face
        verts.append(v)
        tris.append([base, base + 1, base + 2])
        base += 3
    tris.append([0, 1, 3])
    tris.append([4, 5, 7])
    vertices = np.concatenate(verts)
    triangles = np.array(tris, dtype=np.int64)
    s = ElectrodeSurface(vertices, triangles)
    assert tuple(s.info()["cells"]) == tuple(dims)
    m = 60000
    a = rng.integers(0, 3, m)
    p0 = rng.uniform(0.05, 0.95, (m, 3))
    f = np.array([rng.choice(faces[k]) for k in a])
    ulps = rng.integers(-3, 4, m).astype(float)
    p0[np.arange(m), a] = f + ulps * np.spacing(f)
    step = rng.normal(0, 1, (m, 3)) * 0.3 * h[None, :]
    back = rng.uniform(size=m) < 0.5                           # half of them end on the face instead
    p1 = p0 + step
    p0[back], p1[back] = p1[back].copy(), p0[back].copy()
    got = s.segment_intersects_surface(p0, p1)["hit_mask"]
    ref = orc.segments_hit(p0, p1, vertices, triangles)
    np.testing.assert_array_equal(got, ref)
    assert ref.sum() > 1000
