"""Maps that store only the components that are not identically zero.

A component that is zero in every term contributes exact zeros to the
interpolation, so in the float64 form a map without it must give the same
bits as a map that stores it: compared bitwise against maps of the full
E / B / E+B records, for every compiled layout.  The mixed form's Boris
kernels of a pruned layout also leave the zero components' products out of
the rotation (the full-record kernels evaluate them, and the compiler fuses
the remaining products differently), so there the two agree to float32
rounding: within 1e-6 relative."""
import ctypes

import numpy as np
import pytest

from pypatools_b200 import Field, _lib, workloads
from pypatools_b200.device_fields import DeviceFields
from pypatools_b200.pusher import DeviceTracker, MIXED_ALGORITHMS

from tests.helpers import gpu_fields

pytestmark = pytest.mark.gpu


def _rf_gap():
    wl = workloads.rf_gap_protons(n=2000, nsteps=600, nodes=48, rec_every=100)
    return wl, 2 * np.pi * wl.rf_frequency, wl.rf_phase


def _cases():
    out = []
    wl = workloads.quad_solenoid_protons(n=2000, nsteps=400, rec_every=100)
    out.append(("quad_solenoid", wl, 0x38, None, None))
    wl = workloads.radial_e_solenoid_electrons(n=2000, nsteps=400, nodes=33, rec_every=100)
    out.append(("radial_e_solenoid", wl, 0x23, None, None))
    wl, omega, phase = _rf_gap()
    out.append(("rf_gap", wl, 0x24, omega, phase))
    wl = workloads.sector_ring_protons(n=2000, nsteps=400, nodes=40, rec_every=100)
    out.append(("sector_ring", wl, 0x20, None, None))
    return out


def _track(wl, efield, bfield, precision, prune, alg="boris", omega=None, phase=None):
    import torch
    dev = torch.device("cuda", 0)
    df = DeviceFields(efield, bfield, precision, dev, prune=prune)
    tr = DeviceTracker(alg, wl.species.q_over_m, df, wl.n, wl.nsteps, wl.dt, wl.rec_every, precision,
                       rf_omega=omega or 0.0, rf_phase=None if phase is None else torch.from_numpy(phase),
                       device=dev)
    tr.load(torch.from_numpy(wl.r0).to(dev), torch.from_numpy(wl.v0).to(dev))
    tr.run(wl.nsteps, 64)
    return df, tr.r_hist.cpu().numpy(), tr.v_hist.cpu().numpy()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case", range(4))
def test_pruned_maps_are_bitwise_equal_to_full_maps(cuda, precision, case):
    name, wl, layout, omega, phase = _cases()[case]
    e, b = gpu_fields(wl)
    algs = ["boris", "rk4_rel", "vay_rel"] if precision == "mixed" else ["boris", "rk4_rel", "boris_rel"]
    for alg in algs:
        df, rh, vh = _track(wl, e, b, precision, True, alg, omega, phase)
        assert df.layouts == [layout], (name, df.layouts)
        full, rh0, vh0 = _track(wl, e, b, precision, False, alg, omega, phase)
        assert full.layouts[0] in (0x07, 0x38, 0x3F) and full.map_bytes >= df.map_bytes
        if precision == "fp64":
            np.testing.assert_array_equal(rh, rh0, err_msg=f"{name} {alg} r")
            np.testing.assert_array_equal(vh, vh0, err_msg=f"{name} {alg} v")
        else:
            assert np.array_equal(np.isnan(rh), np.isnan(rh0)), (name, alg)
            fin = ~np.isnan(rh0[..., 0])
            dr = np.linalg.norm(rh - rh0, axis=-1)[fin] / np.maximum(np.linalg.norm(rh0, axis=-1)[fin], 0.05)
            dv = np.linalg.norm(vh - vh0, axis=-1)[fin] / np.linalg.norm(vh0, axis=-1)[fin]
            assert dr.max() <= 1e-6 and dv.max() <= 1e-6, (name, alg, dr.max(), dv.max())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_six_component_layout_and_constant_parts(cuda, precision):
    # Ex and By only -> no smaller layout holds both; a constant Bz on top
    # forces the six-component layout in the mixed form as well
    from pypatools_b200.field import CompositeField
    wl = workloads.quad_solenoid_protons(n=1500, nsteps=300, rec_every=100)
    g = {"x": wl.grid[0], "y": wl.grid[1], "z": wl.grid[2]}
    gx, gy, gz = np.meshgrid(*wl.grid, indexing="ij")
    zero = np.zeros_like(gx)
    e = Field.from_arrays(g, {"x": 2e5 * gy, "y": zero, "z": zero})
    b = Field.from_arrays(g, {"x": zero, "y": 0.3 + 2.0 * gx, "z": zero})
    df, rh, vh = _track(wl, e, b, precision, True)
    assert df.layouts == [0x3F]
    bconst = CompositeField([b, Field(dim=0, field={"x": 0.0, "y": 0.0, "z": 0.5})], [1.0, 1.0])
    df, rh, vh = _track(wl, e, bconst, precision, True)
    assert df.layouts == [0x3F]
    _, rh0, vh0 = _track(wl, e, bconst, precision, False)
    np.testing.assert_array_equal(rh, rh0)
    np.testing.assert_array_equal(vh, vh0)


def test_point_evaluation_with_pruned_maps(cuda):
    # the 'cuda' interpolator backend reads the same records
    import torch
    wl, _, _ = _rf_gap()
    e, b = gpu_fields(wl)
    pts = np.random.default_rng(1).uniform(-0.12, 0.12, (5000, 3))
    for precision in ("fp64", "mixed"):
        outs = []
        for prune in (True, False):
            df = DeviceFields(e, b, precision, torch.device("cuda", 0), prune=prune)
            lib = _lib.load()
            d_pts = torch.from_numpy(pts).cuda()
            d_e = torch.empty_like(d_pts)
            d_b = torch.empty_like(d_pts)
            _lib.check(lib.ppt_field_eval(df.fields, len(pts), d_pts.data_ptr(), d_e.data_ptr(), d_b.data_ptr(),
                                          _lib.stream_handle()))
            outs.append((d_e.cpu().numpy(), d_b.cpu().numpy()))
        np.testing.assert_array_equal(outs[0][0], outs[1][0])
        np.testing.assert_array_equal(outs[0][1], outs[1][1])
        assert np.all(outs[0][0][:, :2] == 0.0) and np.any(outs[0][0][:, 2] != 0.0)


def test_add_rejects_components_the_layout_does_not_store(cuda):
    import torch
    lib = _lib.load()
    g = _lib.GridDesc()
    axes = [np.linspace(0.0, 1.0, 4) for _ in range(3)]
    for d in range(3):
        g.n[d] = 4
        g.axis[d] = axes[d].ctypes.data
    h = ctypes.c_void_p()
    _lib.check(lib.ppt_fieldmap_create_masked(g, 0x20, _lib.DTYPE_F32, h))
    try:
        src = torch.ones(64, dtype=torch.float32, device="cuda")
        ptrs = (ctypes.c_void_p * 6)()
        scales = (ctypes.c_double * 6)(*([1.0] * 6))
        ptrs[5] = src.data_ptr()                  # Bz: stored
        _lib.check(lib.ppt_fieldmap_add(h, ptrs, scales, _lib.DTYPE_F32, _lib.stream_handle()))
        ptrs[2] = src.data_ptr()                  # Ez: not stored by the Bz layout
        assert lib.ppt_fieldmap_add(h, ptrs, scales, _lib.DTYPE_F32, _lib.stream_handle()) == -1
        assert b"Ez" in lib.ppt_last_error()
        nbytes, flags = ctypes.c_int64(), ctypes.c_int()
        _lib.check(lib.ppt_fieldmap_info(h, nbytes, flags))
        assert nbytes.value == 64 * 4 and (flags.value >> 8) == 0x20
    finally:
        torch.cuda.synchronize()
        lib.ppt_fieldmap_destroy(h)


def test_mixed_algorithms_cover_every_layout(cuda):
    # every (algorithm, layout) kernel of the mixed form runs and stays finite
    for name, wl, layout, omega, phase in _cases():
        e, b = gpu_fields(wl)
        for alg in MIXED_ALGORITHMS:
            df, rh, vh = _track(wl, e, b, "mixed", True, alg, omega, phase)
            assert np.all(np.isfinite(rh)) and np.all(np.isfinite(vh)), (name, alg)
