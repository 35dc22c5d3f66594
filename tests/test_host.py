"""Host-side checks that need no GPU: the C-ABI library loads and exports
every symbol include/ppt.h declares, argument errors come back as status
codes with messages, and the Python layer mirrors the reference's API."""
import ctypes
import re
import warnings

import numpy as np
import pytest

from pypatools_b200 import _lib
from pypatools_b200.device_fields import decompose
from pypatools_b200.field import Field, ScaledField, CompositeField, FieldMap, get_interpolator
from pypatools_b200.pusher import PusherGPU, REFERENCE_ALGORITHMS
from pypatools_b200.species import IonSpecies
from tests.conftest import REPO


def header_symbols():
    text = (REPO / "include" / "ppt.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:int|int64_t|const char\*)\s+(ppt_\w+)\s*\(", text, re.M)))


def test_library_exports_every_header_symbol():
    lib = _lib.load()
    syms = header_symbols()
    assert len(syms) >= 14
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) == set(_lib.SIGNATURES)
    assert lib.ppt_abi_version() == _lib.ABI_VERSION == 4


def test_struct_layouts_match_header():
    # natural C alignment of the ABI structs
    assert ctypes.sizeof(_lib.GridDesc) == 48
    assert ctypes.sizeof(_lib.Fields) == 4 * 8 + 8 + 48
    assert ctypes.sizeof(_lib.State) == 40
    assert ctypes.sizeof(_lib.TrackArgs) == 4 * 8 + 8 + 4 * 8 + 9 * 8
    assert ctypes.sizeof(_lib.JobDesc) == 40 + ctypes.sizeof(_lib.Fields) + 10 * 8 + 2 * 8


def test_capi_argument_errors_without_gpu():
    lib = _lib.load()
    # non-increasing axis is rejected before any CUDA call
    desc = _lib.GridDesc()
    axes = [np.array([0.0, 1.0, 1.0]), np.array([0.0, 1.0]), np.array([0.0, 1.0])]
    for d in range(3):
        desc.n[d] = axes[d].shape[0]
        desc.axis[d] = axes[d].ctypes.data
    h = ctypes.c_void_p()
    rc = lib.ppt_fieldmap_create(desc, 1, 0, _lib.DTYPE_F64, h)
    assert rc == -1 and b"strictly increasing" in lib.ppt_last_error()
    rc = lib.ppt_fieldmap_create(desc, 0, 0, _lib.DTYPE_F64, h)
    assert rc == -1
    assert lib.ppt_track(None, None, None, None) == -1
    st = _lib.State(_lib.PREC_F64, 99, 10, None, None, None)
    assert lib.ppt_track(st, _lib.Fields(), _lib.TrackArgs(), None) == -1
    assert b"algorithm" in lib.ppt_last_error()
    st = _lib.State(_lib.PREC_F64, 1, 0, None, None, None)
    a = _lib.TrackArgs()
    a.rec_every = 0
    assert lib.ppt_track(st, _lib.Fields(), a, None) == -1
    assert lib.ppt_moments(0, None, None, 1.0, None, None, None) == -1
    assert lib.ppt_cell_sort_scratch_bytes(-1) == -1
    assert lib.ppt_cell_sort_scratch_bytes(1000) > 1000 * 64
    assert lib.ppt_moments_scratch_bytes(10) > 0
    # empty state: nothing to do, no CUDA call
    st = _lib.State(_lib.PREC_F64, 1, 0, None, None, None)
    a.rec_every = 1
    assert lib.ppt_track(st, _lib.Fields(), a, None) == 0
    # back to row order: a state is needed, then order and scratch
    assert lib.ppt_restore_order(None, None, None, None, None) == -1
    assert lib.ppt_restore_order(st, None, None, None, None) == 0          # n = 0
    st10 = _lib.State(_lib.PREC_F64, 1, 10, 256, None, None)               # never dereferenced here
    assert lib.ppt_restore_order(st10, None, None, None, None) == -1
    assert b"order and scratch" in lib.ppt_last_error()
    # a job's own step window must be in [0, 2^31)
    job = _lib.JobDesc()
    job.state = st10
    job.nsteps_total = 100
    job.rec_every = 10
    job.dt = 1e-11
    job.q_over_m = 1.0
    job.tick_steps = -1
    h = ctypes.c_void_p()
    assert lib.ppt_jobs_create((_lib.JobDesc * 1)(job), 1, 256, h, None) == -1
    assert b"tick_steps" in lib.ppt_last_error() and not h.value


def test_map_layout_choice_without_gpu():
    # smallest compiled layout containing the stored components
    lib = _lib.load()
    bz, ez, ex, ey, bx, by = 0x20, 0x04, 0x01, 0x02, 0x08, 0x10
    assert lib.ppt_fieldmap_layout(bz) == bz                      # sector magnet: Bz only
    assert lib.ppt_fieldmap_layout(ez | bz) == ez | bz            # RF gap + solenoid
    assert lib.ppt_fieldmap_layout(ez) == ez | bz
    assert lib.ppt_fieldmap_layout(ex | ey | bz) == ex | ey | bz  # radial E + solenoid
    assert lib.ppt_fieldmap_layout(bx | by | bz) == bx | by | bz  # quadrupole + solenoid
    assert lib.ppt_fieldmap_layout(by) == bx | by | bz
    assert lib.ppt_fieldmap_layout(ex) == ex | ey | ez
    assert lib.ppt_fieldmap_layout(ex | by) == 0x3F
    assert lib.ppt_fieldmap_layout(ez | bx) == 0x3F
    assert lib.ppt_fieldmap_layout(0) == -1
    assert lib.ppt_fieldmap_layout(0x40) == -1
    out = ctypes.c_void_p()
    assert lib.ppt_fieldmap_create_masked(None, 0x20, _lib.DTYPE_F32, out) == -1
    g = _lib.GridDesc()
    assert lib.ppt_fieldmap_create_masked(g, 0, _lib.DTYPE_F32, out) == -1
    assert b"comp_mask" in lib.ppt_last_error()


def test_check_raises_with_message():
    lib = _lib.load()
    with pytest.raises(_lib.PptError, match="PPT_ERR_ARG"):
        _lib.check(lib.ppt_moments(0, None, None, 1.0, None, None, None))


class _FakeNumbaInterp:
    """Looks like the reference's NumbaInterpolator to the adaptor."""

    def __init__(self, grid, values):
        self._grid = grid
        self._values = values
        self.fill_value = 0.0
        self.method = "linear"


class _FakeRefField:
    def __init__(self, dim, field, scaling=1.0):
        self._dim, self._field, self._scaling = dim, field, scaling


def test_decompose_reference_duck_types():
    g = (np.linspace(0, 1, 3),) * 3
    v = np.arange(27.0).reshape(3, 3, 3)
    f3 = _FakeRefField(3, {c: _FakeNumbaInterp(g, v) for c in "xyz"}, scaling=2.0)
    t = decompose(f3)
    assert len(t.terms) == 1 and t.terms[0].scale == 2.0 and not t.const.any()
    from pypatools_b200.device_fields import check_term_sizes
    check_term_sizes(t.terms[0])
    f0 = _FakeRefField(0, {"x": 1.0, "y": 2.0, "z": 3.0}, scaling=0.5)
    np.testing.assert_array_equal(decompose(f0).const, [0.5, 1.0, 1.5])

    class _Scaled:
        def __init__(self, field, scale, offset):
            self.field, self.scale, self.offset = field, scale, offset

    class _Comp:
        def __init__(self, fields, weights):
            self.fields, self.weights = fields, weights

    s = decompose(_Scaled(f3, 3.0, 0.25))
    assert s.terms[0].scale == 6.0
    np.testing.assert_array_equal(s.const, [0.25] * 3)
    c = decompose(_Comp([f3, f0], [0.5, -2.0]))
    assert c.terms[0].scale == 1.0
    np.testing.assert_array_equal(c.const, [-1.0, -2.0, -3.0])
    with pytest.raises(NotImplementedError):
        decompose(lambda pts: pts)


def test_decompose_package_fields_and_zero():
    g = {"x": np.linspace(0, 1, 4), "y": np.linspace(0, 1, 4), "z": np.linspace(0, 1, 5)}
    vals = {c: np.ones((4, 4, 5)) for c in "xyz"}
    f = Field.from_arrays(g, vals)
    assert f.dim == 3 and len(decompose(f).terms) == 1
    assert decompose(Field.zero(3)).terms == []
    assert len(decompose(2.0 * f + f).terms) == 2
    assert isinstance(f - f, CompositeField) and isinstance(f * 2.0, ScaledField)
    fm = FieldMap(bfield=f)
    assert decompose(fm.efield).terms == []
    with pytest.raises(NotImplementedError):
        get_interpolator((g["x"], g["y"], g["z"]), vals["x"], backend="numba")


def test_pusher_constructor_mirrors_reference():
    ion = IonSpecies("proton")
    with pytest.raises(ValueError, match=r"Unknown algorithm 'nope'. Must be one of"):
        PusherGPU(ion, "nope")
    p = PusherGPU(ion, "RK4_REL")
    assert p.algorithm == "rk4_rel" and p.relativistic
    assert PusherGPU.ALGORITHMS == REFERENCE_ALGORITHMS

    class _Hot:
        name = "x"
        q_over_m = 1.0
        energy_mev = 1.0

    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        assert PusherGPU(_Hot(), "leapfrog").algorithm == "vay_rel"
        assert any("Leapfrog is non-relativistic" in str(x.message) for x in w)
    with pytest.raises(NotImplementedError):
        PusherGPU(ion, "boris", electrode_assembly=object())
    p.change_algorithm("boris")
    assert p.algorithm == "boris" and "PusherGPU(ion=proton" in repr(p)


def test_array_dt_only_where_the_reference_takes_one():
    """An (M,) dt array goes to the float64 rk4 / rk4_rel only (the
    reference's batch RK4 step, pusher.py:815-816); it is checked on the host
    before anything is uploaded."""
    ion = IonSpecies("proton")
    r = np.zeros((4, 3))
    dts = np.full(4, 1e-11)
    with pytest.raises(TypeError, match="dt must be a scalar"):
        PusherGPU(ion, "boris").track_batch(r, r, None, None, 3, dts)
    with pytest.raises(TypeError, match="dt must be a scalar"):
        PusherGPU(ion, "rk4", precision="mixed").push_batch(r, r, None, None, dts)
    with pytest.raises(ValueError, match=r"shape \(4,\)"):
        PusherGPU(ion, "rk4").track_batch(r, r, None, None, 3, np.full(5, 1e-11))
    assert PusherGPU(ion, "rk4_rel")._time_step(dts, 4)[1] is not None
    assert PusherGPU(ion, "rk4_rel")._time_step(np.float64(1e-11), 4) == (1e-11, None)


def test_state_rows_are_checked_before_a_launch():
    # the state load / store kernels address n rows of 24 B: the tracker
    # refuses anything else on the host
    import torch
    from pypatools_b200.pusher import check_rows
    dev = torch.device("cpu")
    r = torch.zeros((4, 3), dtype=torch.float64)
    assert check_rows(r, 4, dev, "r") is r
    with pytest.raises(TypeError):
        check_rows(np.zeros((4, 3)), 4, dev, "r")
    with pytest.raises(ValueError, match=r"\(4, 3\) float64"):
        check_rows(r[:3], 4, dev, "r")
    with pytest.raises(ValueError, match=r"\(4, 3\) float64"):
        check_rows(r.float(), 4, dev, "r")
    with pytest.raises(ValueError, match="strided"):
        check_rows(torch.zeros((3, 4), dtype=torch.float64).t(), 4, dev, "r")
    with pytest.raises(ValueError, match="contiguous on cuda:0"):
        check_rows(r, 4, torch.device("cuda", 0), "r")


def test_map_terms_hold_one_value_per_node():
    # the map add kernel reads one value per grid node from each component
    from pypatools_b200.device_fields import check_term_sizes, _MapTerm
    g3 = {"x": np.linspace(0, 1, 4), "y": np.linspace(0, 1, 3), "z": np.linspace(0, 1, 5)}
    f3 = Field.from_arrays(g3, {c: np.ones((4, 3, 5)) for c in "xyz"})
    z = np.linspace(0, 1, 7)
    f1 = Field.from_arrays({"z": z}, {c: np.ones(7) for c in "xyz"})
    f2 = Field.from_arrays({"x": z, "y": z[:4]}, {c: np.ones((7, 4)) for c in "xyz"})
    for f in (f3, f1, f2, 2.0 * f3 + f3):
        for t in decompose(f).terms:
            check_term_sizes(t)
    t = decompose(f3).terms[0]
    bad = _MapTerm(t.grid, {"x": np.ones(59), "y": None, "z": t.comps["z"]}, 1.0)
    with pytest.raises(ValueError, match="59 node values, its grid 4 x 3 x 5 = 60 nodes"):
        check_term_sizes(bad)


def test_tracking_job_arguments_checked_at_submission():
    from pypatools_b200.serving import TrackingJob
    r = np.zeros((5, 3))
    j = TrackingJob(0, 1.0, "boris", r, r, None, None, 100, 1e-11, rec_every=10)
    assert j.n == 5 and j.n_rec == 11
    with pytest.raises(ValueError, match=r"\(M, 3\)"):
        TrackingJob(0, 1.0, "boris", r, np.zeros((4, 3)), None, None, 100, 1e-11)
    with pytest.raises(ValueError, match=r"\(M, 3\)"):
        TrackingJob(0, 1.0, "boris", np.zeros(15), np.zeros(15), None, None, 100, 1e-11)
    with pytest.raises(ValueError, match="rec_every"):
        TrackingJob(0, 1.0, "boris", r, r, None, None, 100, 1e-11, rec_every=0)


def test_host_result_pool_recycles_released_mappings():
    """track_batch's numpy results sit on pooled mappings: one goes back to
    the pool only when the array and every view of it are gone, is handed out
    again for the same size, and the pool keeps no more than its limit."""
    import gc
    from pypatools_b200.pusher import HostResultPool, host_array
    import pypatools_b200.pusher as pusher_mod
    saved = pusher_mod.HOST_POOL
    size = 3 * (1 << 22) * 3 * 8                        # 288 MiB
    pool = pusher_mod.HOST_POOL = HostResultPool(2 * size)
    try:
        shape = (3, 1 << 22, 3)
        a = host_array(shape)
        assert a.shape == shape and a.dtype == np.float64 and a.flags.writeable
        addr = a.ctypes.data
        a[:] = 1.0
        view = a[1]
        del a
        gc.collect()
        assert pool.free_bytes == 0                     # the view still holds it
        del view
        gc.collect()
        assert pool.free_bytes == size
        b = host_array(shape)
        assert b.ctypes.data == addr and pool.free_bytes == 0
        c = host_array(shape)
        assert c.ctypes.data != addr
        d = host_array(shape)
        del b, c, d
        gc.collect()
        assert pool.free_bytes == 2 * size              # the third was over the limit: unmapped
        small = host_array((10, 3))                     # below 64 MiB: plain numpy
        assert small.base is None
        pool.clear()
        assert pool.free_bytes == 0
    finally:
        pusher_mod.HOST_POOL = saved
