"""Field-map loaders (field_src/field_loaders.py) and Field.from_file
(field.py:284-343) against the reference run on the same files.

tests/golden/loaders_golden.npz holds the reference loaders' results on the
seeded files of tests/golden/loader_files.py (make_golden_loaders.py).  Text
parsing must agree bit for bit; the cylindrical maps' resampling runs on the
GPU with its own bilinear arithmetic, so it agrees to rounding (1e-12 of the
largest field value)."""
import sys
import types

import numpy as np
import pytest

from pypatools_b200 import loaders
from tests.conftest import REPO

sys.path.insert(0, str(REPO / "tests" / "golden"))
from loader_files import write_cases  # noqa: E402

G = np.load(REPO / "tests" / "golden" / "loaders_golden.npz")
PARSED = ("opera3d", "opera2d", "opera_e", "opera_ext", "comsol3d", "comsol2d", "opal_cyl")
RESAMPLED = ("opal", "opal_cut", "aima", "aima_mirror")
LOADER = {"opera": loaders.load_opera_table, "comsol": loaders.load_comsol, "opal": loaders.load_opal_midplane,
          "aima": loaders.load_aima_agora}


@pytest.fixture(scope="module")
def cases(tmp_path_factory):
    return write_cases(str(tmp_path_factory.mktemp("maps")))


def _load(cases, name):
    path, kwargs = cases[name]
    kind = next(k for k in LOADER if name.startswith(k))
    return LOADER[kind](path, **kwargs)


def _check_meta(name, data):
    assert data["dim"] == int(G[f"{name}/dim"])
    assert data["field_type"] == str(G[f"{name}/field_type"])
    for k, v in data["metadata"].get("n_points", {}).items():
        assert int(v) == int(G[f"{name}/n_points/{k}"])


@pytest.mark.parametrize("name", PARSED)
def test_parsed_maps_match_reference_bitwise(cases, name):
    data = _load(cases, name)
    _check_meta(name, data)
    for part in ("grid", "values"):
        keys = sorted(k.split("/")[2] for k in G.files if k.startswith(f"{name}/{part}/"))
        assert sorted(data[part]) == keys
        for k in keys:
            np.testing.assert_array_equal(np.asarray(data[part][k]), G[f"{name}/{part}/{k}"], err_msg=f"{part} {k}")


def test_loader_errors_match_reference(tmp_path):
    bad = tmp_path / "mixed.table"
    bad.write_text("2 1 1\n1 X [cm]\n2 BX [T]\n3 EX [V/m]\n0\n0 1 2\n1 1 2\n")
    with pytest.raises(RuntimeError) as exc:
        loaders.load_opera_table(str(bad))
    assert f"{type(exc.value).__name__}: {exc.value}" == str(G["errors/opera_mixed"])
    with pytest.raises(FileNotFoundError):
        loaders.load_comsol(str(tmp_path / "missing.comsol"))
    with pytest.raises(ValueError, match="extension"):
        (tmp_path / "m.txt").write_text("1\n")
        loaders.load_opal_midplane(str(tmp_path / "m.txt"))
    with pytest.raises(ValueError, match="extents_dims"):
        loaders.load_opera_table(str(bad), extents=[(0, 1)] * 3)


def test_blank_lines_are_skipped(tmp_path):
    # trailing whitespace lines break the reference's OPERA and OPAL readers;
    # here they are skipped
    p = tmp_path / "t.table"
    p.write_text("2 2 1\n1 X [cm]\n2 Y [cm]\n3 BZ [T]\n0\n0 0 1\n0 1 2\n1 0 3\n1 1 4\n   \n\n")
    d = loaders.load_opera_table(str(p))
    np.testing.assert_array_equal(d["values"]["z"][:, :, 0], [[1, 2], [3, 4]])
    np.testing.assert_array_equal(d["grid"]["x"], [0.0, 0.01])
    q = tmp_path / "m.dat"
    q.write_text("0.0\n10.0\n0.0\n90.0\n4\n2\n1 2 3 4\n5 6 7 8\n  \n")
    d = loaders.load_opal_midplane(str(q), cartesian_grid=False)
    np.testing.assert_allclose(d["values"]["z"], 0.1 * np.arange(1, 9).reshape(2, 4))


def test_from_file_dims_and_reference_failures(cases):
    from pypatools_b200 import Field
    for name in ("opera3d", "opera2d", "opera_e", "comsol3d", "comsol2d"):
        path, _ = cases[name]
        if f"{name}/from_file_error" in G.files:
            # e.g. a 2D OPERA table: (nx, ny, 1) values on a 2-axis grid are
            # rejected by the interpolator, as in the reference
            with pytest.raises(ValueError):
                Field.from_file(path)
        else:
            assert Field.from_file(path).dim == int(G[f"{name}/from_file_dim"])
    with pytest.raises(ValueError, match="Unknown file extension"):
        Field.from_file(__file__)


def test_pickle_round_trip(cases, tmp_path):
    from pypatools_b200 import Field
    f = Field.from_file(cases["comsol3d"][0], label="solenoid", scaling=2.0)
    p = tmp_path / "f.pickle"
    f.save_pickle(str(p))
    g = Field.from_file(str(p))
    assert g.label == "solenoid" and g.scaling == 2.0 and g.dim == 3
    np.testing.assert_array_equal(g._field["z"]._values, f._field["z"]._values)


def test_h5part_layout_with_a_stand_in_h5py(tmp_path, monkeypatch):
    # h5py is not installed here: a stand-in module serves the file's groups
    nz, ny, nx = 2, 3, 4
    comps = [np.arange(nz * ny * nx, dtype=float).reshape(nz, ny, nx) * (k + 1) for k in range(3)]

    class Group(dict):
        def __init__(self, items, attrs=None):
            super().__init__(items)
            self.attrs = attrs or {}

    hfield = Group({"0": comps[0], "1": comps[1], "2": comps[2]},
                   {"__Spacing__": np.array([0.1, 0.2, 0.3]), "__Origin__": np.array([-1.0, 0.0, 1.0])})
    tree = Group({"Step#0": Group({"Block": Group({"Hfield": hfield})})})

    class File:
        def __init__(self, name, mode):
            self.tree = tree

        def __getitem__(self, k):
            return self.tree[k]

        def close(self):
            pass

    fake = types.ModuleType("h5py")
    fake.File = File
    monkeypatch.setitem(sys.modules, "h5py", fake)
    path = tmp_path / "f.h5part"
    path.write_bytes(b"")
    d = loaders.load_h5part(str(path))
    np.testing.assert_array_equal(d["values"]["y"], np.transpose(comps[1], (2, 1, 0)))
    np.testing.assert_allclose(d["grid"]["z"], [1.0, 1.3])
    assert d["metadata"]["shape"] == (nx, ny, nz) and d["metadata"]["has_efield"] is False


def test_resample_oracle_matches_reference_bitwise():
    # the oracle's RegularGridInterpolator resampling reproduces the reference's
    # OPAL midplane map exactly (same nodes: the file's r0 = 10 mm, dr = 10 mm,
    # 20 radii; theta0 = 0, dtheta = 2.5 deg, 144 angles)
    from oracle import loader_oracle
    r = np.linspace(10.0, 200.0, 20)
    th = np.linspace(0.0, 357.5, 144)
    bz_cyl = G["opal_cyl/values/z"]
    x, y = G["opal/grid/x"], G["opal/grid/y"]
    _, _, bz = loader_oracle.polar_to_cartesian(r, th, (None, None, bz_cyl), x, y, r_scale=1000.0)
    np.testing.assert_array_equal(bz, G["opal/values/z"])


def test_polar_argument_checks_without_gpu():
    import ctypes
    from pypatools_b200 import _lib
    lib = _lib.load()
    g = _lib.PolarGrid(1, 4, 16, 16)
    nul = (ctypes.c_void_p * 3)()
    assert lib.ppt_polar_to_cartesian(g, nul, 2, 16, 2, 16, 1.0, nul, None) == -1
    assert b"2 nodes" in lib.ppt_last_error()


@pytest.mark.gpu
def test_gpu_polar_resample_vs_oracle_all_components(cuda):
    from oracle import loader_oracle
    rng = np.random.default_rng(4)
    r = np.linspace(0.5, 30.0, 100)
    th = np.linspace(0.0, 359.0, 360)
    comps = [rng.normal(0, 1, (100, 360)) for _ in range(3)]
    x = np.linspace(-31.0, 31.0, 301)
    y = np.linspace(-25.0, 31.0, 257)
    got = loaders.polar_to_cartesian(r, th, comps, x, y)
    ref = loader_oracle.polar_to_cartesian(r, th, comps, x, y)
    for g, o in zip(got, ref):
        np.testing.assert_allclose(g, o, rtol=0, atol=1e-12 * np.abs(o).max())


@pytest.mark.gpu
@pytest.mark.parametrize("name", RESAMPLED)
def test_gpu_resampled_maps_match_reference(cuda, cases, name):
    data = _load(cases, name)
    _check_meta(name, data)
    for k in ("x", "y", "z"):
        np.testing.assert_array_equal(data["grid"][k], G[f"{name}/grid/{k}"])
        ref = G[f"{name}/values/{k}"]
        scale = max(np.abs(ref).max(), 1e-300)
        np.testing.assert_allclose(data["values"][k], ref, rtol=0, atol=1e-12 * scale, err_msg=k)


@pytest.mark.gpu
def test_gpu_from_file_midplane_evaluates(cuda, cases):
    from oracle import pusher_oracle as orc
    from pypatools_b200 import Field
    f = Field.from_file(cases["opal"][0])
    assert f.dim == 2
    gx, gy = G["opal/grid/x"], G["opal/grid/y"]
    pts = np.random.default_rng(2).uniform(-0.2, 0.2, (2000, 3))
    ref = orc.MapField((gx, gy), {"x": None, "y": None, "z": G["opal/values/z"]})(pts)
    np.testing.assert_allclose(f(pts), ref, rtol=0, atol=1e-12 * np.abs(ref).max())


def test_aima_directory_checks(tmp_path):
    # field_loaders.py's AIMA reader: files not named <...>Z<z>-<br|bf|bz>.map
    # are skipped; none left, or components on different z sets, is an error
    # (raised before any resampling)
    d = tmp_path / "aima"
    d.mkdir()
    for junk in ("notes.map", "fieldZabc-br.map", "fieldZ010-bx.map", "field-Z.map"):
        (d / junk).write_text("x\n")
    with pytest.raises(ValueError, match="No valid .map files"):
        loaders.load_aima_agora(str(d))
    for name in ("fieldZ000-br.map", "fieldZ000-bf.map", "fieldZ000-bz.map", "fieldZ010-br.map"):
        (d / name).write_text("x\n")
    with pytest.raises(ValueError, match="same z positions"):
        loaders.load_aima_agora(str(d))
    with pytest.raises(FileNotFoundError):
        loaders.load_aima_agora(str(tmp_path / "missing"))


def test_polar_resample_argument_checks_without_gpu():
    # the resampling kernel reads nr x nt values per component: shapes are
    # checked on the host first
    r, th, x = np.linspace(0, 1, 4), np.linspace(0, 350, 36), np.linspace(-1, 1, 5)
    with pytest.raises(ValueError, match=r"shape \(36, 4\) on a \(4, 36\)"):
        loaders.polar_to_cartesian(r, th, (None, None, np.zeros((36, 4))), x, x)
    with pytest.raises(ValueError, match="1D"):
        loaders.polar_to_cartesian(r[None], th, (None, None, None), x, x)
    with pytest.raises(ValueError, match="three entries"):
        loaders.polar_to_cartesian(r, th, (None, np.zeros((4, 36))), x, x)
