"""1D and 2D fields: a 1D field varies along z only, a 2D field along x and y
(the reference's Field._get_field_1d / _get_field_2d, field.py:457-489).

The fixture tests/golden/fields12_golden.npz comes from the reference itself
(tests/golden/make_golden_fields12.py): field values at probe points (faces,
nodes, one ulp outside, far along the constant axes) and Pusher.track_batch
trajectories through a 2D sector field (protons on a ring) and through a 1D
Ez / Bz gap.  The oracle is pinned to it; the float64 GPU form is held to the
1e-10 parity bar, the mixed form to its error bar against the oracle."""
import ctypes

import numpy as np
import pytest

from oracle import pusher_oracle as orc
from pypatools_b200 import _lib
from pypatools_b200.species import IonSpecies
from tests.conftest import REPO
from tests.helpers import rel_pos_err, rel_vel_err

G = np.load(REPO / "tests" / "golden" / "fields12_golden.npz")
ION = IonSpecies("proton")
TOL = 1e-10


def _ring():
    return (G["ring2d/gx"], G["ring2d/gy"]), G["ring2d/bz"]


def _gap():
    return G["gap1d/gz"], G["gap1d/ez"], G["gap1d/bz"]


def _oracle_ring():
    grid, bz = _ring()
    return orc.ZeroField(), orc.MapField(grid, {"x": None, "y": None, "z": bz})


def _oracle_gap():
    gz, ez, bz = _gap()
    return (orc.MapField((gz,), {"x": None, "y": None, "z": ez}),
            orc.MapField((gz,), {"x": None, "y": None, "z": bz}))


def _gpu_ring():
    from pypatools_b200 import Field
    (gx, gy), bz = _ring()
    zero = np.zeros_like(bz)
    return Field.zero(3), Field.from_arrays({"x": gx, "y": gy}, {"x": zero, "y": zero, "z": bz})


def _gpu_gap():
    from pypatools_b200 import Field
    gz, ez, bz = _gap()
    z = np.zeros_like(gz)
    return (Field.from_arrays({"z": gz}, {"x": z, "y": z, "z": ez}),
            Field.from_arrays({"z": gz}, {"x": z, "y": z, "z": bz}))


# ---------------------------------------------------------------------------
# CPU: the oracle against the reference, the host decomposition, the ABI checks
# ---------------------------------------------------------------------------

def test_oracle_field_values_match_reference():
    f2 = orc.MapField((G["f2/gx"], G["f2/gy"]), {c: G[f"f2/values_{c}"] for c in "xyz"})
    np.testing.assert_allclose(f2(G["f2/probe"]), G["f2/out"], rtol=0, atol=1e-15)
    f1 = orc.MapField((G["f1/gz"],), {c: G[f"f1/values_{c}"] for c in "xyz"})
    np.testing.assert_allclose(f1(G["f1/probe"]), G["f1/out"], rtol=0, atol=1e-15 * np.abs(G["f1/out"]).max())
    # the constant axes have no bounds: points far along them still see the field
    assert np.any(G["f2/out"][-1] != 0.0) and np.any(G["f1/out"][-1] != 0.0)


def test_reference_numba_1d_batch_failure_recorded():
    # the reference's default (Numba) interpolator rejects M > 1 points in a 1D
    # field (interpolators.py:357-364 reads the M z values as one M-dim point);
    # the fixture's 1D cases use its scipy backend, and this package evaluates
    # batches as that backend does
    assert int(G["f1/numba_batch_raises"]) == 1


@pytest.mark.parametrize("alg", ["boris", "vay_rel", "rk4_rel"])
def test_oracle_ring_2d_matches_reference(alg):
    e, b = _oracle_ring()
    rh, vh, _ = orc.track_batch(alg, ION.q_over_m, G["ring2d/r0"], G["ring2d/v0"], e, b, 2000, 1e-10, 500)
    assert rel_pos_err(rh, G[f"ring2d/{alg}/r_hist"], 0.3) < 1e-12
    assert rel_vel_err(vh, G[f"ring2d/{alg}/v_hist"]) < 1e-12


@pytest.mark.parametrize("alg", ["boris", "rk4_rel"])
def test_oracle_gap_1d_matches_reference(alg):
    e, b = _oracle_gap()
    rh, vh, _ = orc.track_batch(alg, ION.q_over_m, G["gap1d/r0"], G["gap1d/v0"], e, b, 3000, 1e-11, 750)
    assert rel_pos_err(rh, G[f"gap1d/{alg}/r_hist"], 0.2) < 1e-12
    assert rel_vel_err(vh, G[f"gap1d/{alg}/v_hist"]) < 1e-12


def test_decompose_maps_1d_to_z_and_2d_to_xy():
    from pypatools_b200.device_fields import decompose
    e, b = _gpu_gap()
    (t,) = decompose(e).terms
    assert [g.shape[0] for g in t.grid] == [1, 1, 201]
    _, b2 = _gpu_ring()
    (t,) = decompose(2.0 * b2).terms
    assert [g.shape[0] for g in t.grid] == [121, 121, 1] and t.scale == 2.0
    # the node arrays keep their shape: flattened in C order they are [i][j][k]
    assert t.comps["z"].shape == (121, 121)


def test_grid_argument_checks_without_gpu():
    lib = _lib.load()
    desc = _lib.GridDesc()
    h = ctypes.c_void_p()
    for d in range(3):
        desc.n[d] = 1
    assert lib.ppt_fieldmap_create_masked(desc, 0x20, _lib.DTYPE_F64, h) == -1
    assert b"at least 2 nodes" in lib.ppt_last_error()
    desc.n[0] = 0
    assert lib.ppt_fieldmap_create_masked(desc, 0x20, _lib.DTYPE_F64, h) == -1
    assert b"at least 1 node" in lib.ppt_last_error()


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------

@pytest.mark.gpu
def test_gpu_field_values_match_reference(cuda):
    from pypatools_b200 import Field
    f2 = Field.from_arrays({"x": G["f2/gx"], "y": G["f2/gy"], "z": np.array([0.0])},
                           {c: G[f"f2/values_{c}"] for c in "xyz"})
    assert f2.dim == 2
    np.testing.assert_allclose(f2(G["f2/probe"]), G["f2/out"], rtol=0, atol=1e-15)
    f1 = Field.from_arrays({"z": G["f1/gz"]}, {c: G[f"f1/values_{c}"] for c in "xyz"})
    assert f1.dim == 1
    np.testing.assert_allclose(f1(G["f1/probe"]), G["f1/out"], rtol=0,
                               atol=1e-15 * np.abs(G["f1/out"]).max())
    # the standalone interpolators: a 1D one takes (M, 1) coordinates, a 2D one (M, 2)
    z = G["f1/probe"][:, 2:3]
    np.testing.assert_allclose(f1._field["z"](z), G["f1/out"][:, 2], rtol=0,
                               atol=1e-15 * np.abs(G["f1/out"]).max())
    np.testing.assert_allclose(f2._field["z"](G["f2/probe"][:, :2]), G["f2/out"][:, 2], rtol=0, atol=1e-15)
    # float32 records (the mixed form's maps, uniform grids) through the same
    # evaluation kernel, against the oracle on float32-rounded node values
    import torch
    from pypatools_b200.device_fields import DeviceFields
    _, b2 = _gpu_ring()
    (gx, gy), bz = _ring()
    df = DeviceFields(None, b2, "mixed", torch.device("cuda", 0))
    assert df.layouts == [0x20]
    probe = G["f2/probe"]
    pts = torch.from_numpy(probe).cuda()
    out = torch.empty_like(pts)
    _lib.check(_lib.load().ppt_field_eval(df.fields, pts.shape[0], pts.data_ptr(), None, out.data_ptr(),
                                          _lib.stream_handle()))
    ref = orc.MapField((gx, gy), {"x": None, "y": None, "z": bz.astype(np.float32)})(probe)
    np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=0, atol=1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("alg", ["boris", "vay_rel", "rk4_rel"])
def test_gpu_ring_2d_fp64_matches_reference(cuda, alg):
    from pypatools_b200 import PusherGPU
    e, b = _gpu_ring()
    rh, vh, act = PusherGPU(ION, alg).track_batch(G["ring2d/r0"], G["ring2d/v0"], e, b, 2000, 1e-10, 500)
    assert rel_pos_err(rh, G[f"ring2d/{alg}/r_hist"], 0.3) < TOL
    assert rel_vel_err(vh, G[f"ring2d/{alg}/v_hist"]) < TOL
    assert act.all()


@pytest.mark.gpu
@pytest.mark.parametrize("alg", ["boris", "rk4_rel"])
def test_gpu_gap_1d_fp64_matches_reference(cuda, alg):
    from pypatools_b200 import PusherGPU
    e, b = _gpu_gap()
    rh, vh, _ = PusherGPU(ION, alg).track_batch(G["gap1d/r0"], G["gap1d/v0"], e, b, 3000, 1e-11, 750)
    assert rel_pos_err(rh, G[f"gap1d/{alg}/r_hist"], 0.2) < TOL
    assert rel_vel_err(vh, G[f"gap1d/{alg}/v_hist"]) < TOL


@pytest.mark.gpu
@pytest.mark.parametrize("alg,bound", [("boris", 2e-6), ("rk4_rel", 5e-6)])
def test_gpu_ring_2d_mixed_vs_oracle(cuda, alg, bound):
    # three turns (2000 steps of 0.01 rad): the float32 rotation's phase drift
    # (~1e-9 rad per step) sets the error, as on the sector ring
    from pypatools_b200 import PusherGPU
    e, b = _gpu_ring()
    rh, vh, _ = PusherGPU(ION, alg, precision="mixed").track_batch(G["ring2d/r0"], G["ring2d/v0"], e, b,
                                                                    2000, 1e-10, 500)
    err_r = rel_pos_err(rh, G[f"ring2d/{alg}/r_hist"], 0.3)
    err_v = rel_vel_err(vh, G[f"ring2d/{alg}/v_hist"])
    print(f"mixed {alg} 2D ring: pos {err_r:.2e} vel {err_v:.2e}")
    assert err_r < bound and err_v < bound


@pytest.mark.gpu
@pytest.mark.parametrize("alg", ["boris", "rk4_rel"])
def test_gpu_gap_1d_mixed_vs_oracle(cuda, alg):
    # E and B on the same 1D grid share one map ({Ez Bz} records, x and y constant)
    from pypatools_b200 import PusherGPU
    from pypatools_b200.device_fields import DeviceFields
    import torch
    e, b = _gpu_gap()
    df = DeviceFields(e, b, "mixed", torch.device("cuda", 0))
    assert df.layouts == [0x24]
    rh, vh, _ = PusherGPU(ION, alg, precision="mixed").track_batch(G["gap1d/r0"], G["gap1d/v0"], e, b,
                                                                    3000, 1e-11, 750)
    err_r = rel_pos_err(rh, G[f"gap1d/{alg}/r_hist"], 0.2)
    err_v = rel_vel_err(vh, G[f"gap1d/{alg}/v_hist"])
    print(f"mixed {alg} 1D gap: pos {err_r:.2e} vel {err_v:.2e}")
    assert err_r < 1e-6 and err_v < 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gpu_2d_chunking_and_sorting_bitwise_invariant(cuda, precision):
    from pypatools_b200 import PusherGPU
    e, b = _gpu_ring()
    r0, v0 = G["ring2d/r0"], G["ring2d/v0"]
    base = PusherGPU(ION, "boris", precision=precision).track_batch(r0, v0, e, b, 600, 1e-10, 50)
    chunked = PusherGPU(ION, "boris", precision=precision, steps_per_launch=7).track_batch(r0, v0, e, b, 600,
                                                                                          1e-10, 50)
    sorted_ = PusherGPU(ION, "boris", precision=precision, sort_every=40).track_batch(r0, v0, e, b, 600, 1e-10, 50)
    for other in (chunked, sorted_):
        np.testing.assert_array_equal(base[0], other[0])
        np.testing.assert_array_equal(base[1], other[1])


@pytest.mark.gpu
def test_gpu_1d_e_with_2d_b_two_maps_fp64(cuda):
    # a 1D E map and a 2D B map on different grids: two device maps, float64 form
    from pypatools_b200 import PusherGPU
    e1, _ = _gpu_gap()
    _, b2 = _gpu_ring()
    oe, _ = _oracle_gap()
    _, ob = _oracle_ring()
    r0 = G["ring2d/r0"].copy()
    r0[:, 2] = np.linspace(-0.15, 0.15, r0.shape[0])
    rh, vh, _ = PusherGPU(ION, "boris").track_batch(r0, G["ring2d/v0"], 0.01 * e1, b2, 800, 1e-10, 200)
    ro, vo, _ = orc.track_batch("boris", ION.q_over_m, r0, G["ring2d/v0"], orc.ScaledOracleField(oe, 0.01), ob,
                                800, 1e-10, 200)
    assert rel_pos_err(rh, ro, 0.3) < TOL
    assert rel_vel_err(vh, vo) < TOL
