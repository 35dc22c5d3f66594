"""Space-charge solve: deposition, Poisson solve and E = -grad phi
(PyAMGPoissonSolver, src/PyPATools/poisson_amg.py), with and without
conductor cells.

The oracle's operator, cell classification, Shortley-Weller rows and field
step are pinned bit for bit to the reference's own code (tests/golden/
poisson_golden.npz, made by make_golden_poisson.py; the classification runs
on ray results served to it, since its electrode package is not installed).
The GPU ray casting matches the oracle's bit for bit; the GPU solves are held
to the exact solution of the operator (sparse direct solve) at 1e-8 relative
when solved to a 1e-12 residual; the field step to the reference bit for bit."""
import ctypes

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import space_charge_oracle as sco
from pypatools_b200 import _lib
from tests.conftest import REPO

G = np.load(REPO / "tests" / "golden" / "poisson_golden.npz")
CASES = ("box", "flat")


def _mesh(extent, cells):
    m = _lib.MeshDesc()
    for a in range(3):
        m.extent[a] = extent[a]
        m.cells[a] = int(cells[a])
    return m


@pytest.mark.parametrize("name", CASES)
def test_oracle_operator_matches_reference_bitwise(name):
    cells = tuple(int(c) for c in G[f"{name}/cells"])
    m = int(np.prod(cells))
    ref = sp.csr_matrix((G[f"{name}/A_val"], (G[f"{name}/A_row"], G[f"{name}/A_col"])), shape=(m, m))
    ours = sco.assemble_matrix(G[f"{name}/extent"], cells)
    assert (ours != ref).nnz == 0
    np.testing.assert_array_equal(ours.toarray(), ref.toarray())


@pytest.mark.parametrize("name", CASES)
def test_oracle_field_matches_reference_bitwise(name):
    ex, ey, ez = sco.field_from_potential(G[f"{name}/phi"], G[f"{name}/extent"])
    for got, key in ((ex, "ex"), (ey, "ey"), (ez, "ez")):
        np.testing.assert_array_equal(got, G[f"{name}/{key}"])


def test_poisson_argument_checks_without_gpu():
    lib = _lib.load()
    assert lib.ppt_poisson_scratch_bytes(None) == -1
    mesh = _mesh((0.1, 0.1, 0.1), (4, 4, 4))
    m, nb = 64, 1
    assert lib.ppt_poisson_scratch_bytes(mesh) == (3 * m + 2 * nb + 7) * 8
    it, res = ctypes.c_int64(), ctypes.c_double()
    assert lib.ppt_poisson_solve(mesh, None, None, None, 1e-6, 10, it, res, None) == -1
    bad = _mesh((0.1, -1.0, 0.1), (4, 4, 4))
    assert lib.ppt_field_from_potential(bad, ctypes.c_void_p(16), None, None, None, None) == -1
    assert b"positive" in lib.ppt_last_error()


def test_device_solve_input_checks_without_gpu():
    # the deposit kernel reads (M, 3) float64 rows: anything else is refused
    # on the host before a launch
    import torch
    from pypatools_b200.space_charge import check_device_inputs
    dev = torch.device("cpu")
    p, q = torch.zeros((5, 3), dtype=torch.float64), torch.zeros(5, dtype=torch.float64)
    a, b = check_device_inputs(p, q, dev)
    assert a.is_contiguous() and b.shape == (5,)
    a, _ = check_device_inputs(torch.zeros((3, 5), dtype=torch.float64).t(), q, dev)   # made contiguous
    assert a.is_contiguous() and a.shape == (5, 3)
    with pytest.raises(TypeError, match="torch tensors"):
        check_device_inputs(np.zeros((5, 3)), q, dev)
    with pytest.raises(TypeError, match="float64"):
        check_device_inputs(p.float(), q, dev)
    with pytest.raises(ValueError, match=r"\(M, 3\)"):
        check_device_inputs(torch.zeros((5, 2), dtype=torch.float64), q, dev)
    with pytest.raises(ValueError, match=r"\(M, 3\)"):
        check_device_inputs(p, torch.zeros(4, dtype=torch.float64), dev)
    with pytest.raises(ValueError, match="must be on"):
        check_device_inputs(p, q, torch.device("cuda", 0))
    check_device_inputs(torch.zeros((0, 3), dtype=torch.float64), torch.zeros(0, dtype=torch.float64), dev)


def _cond():
    cells = tuple(int(c) for c in G["cond/cells"])
    h = [G["cond/extent"][a] / cells[a] for a in range(3)]
    return G["cond/extent"], cells, h


def test_oracle_conductor_classification_and_rows_match_reference():
    extent, cells, h = _cond()
    kind = sco.classify_cells(G["cond/dist"], G["cond/hits"], h)
    np.testing.assert_array_equal(kind, G["cond/cell_type"])
    a, keep = sco.assemble_reduced(extent, cells, kind, G["cond/dist"])
    np.testing.assert_array_equal(keep, G["cond/keep"])
    ref = sp.csr_matrix((G["cond/A_val"], (G["cond/A_row"], G["cond/A_col"])), shape=a.shape)
    np.testing.assert_array_equal(a.toarray(), ref.toarray())


def test_product_rows_match_oracle():
    # the solver's (m, 7) coefficient rows are the reference's reduced matrix
    # on the non-conductor cells and the identity on the conductor ones
    from pypatools_b200.space_charge import classify_cells, operator_coefficients
    extent, cells, h = _cond()
    kind = classify_cells(G["cond/dist"], G["cond/hits"], h)
    np.testing.assert_array_equal(kind, G["cond/cell_type"])
    coef = operator_coefficients(cells, h, kind, G["cond/dist"])
    m = coef.shape[0]
    strides = (cells[1] * cells[2], cells[2], 1)
    rows, cols, vals = [], [], []
    for c in range(m):
        rows.append(c); cols.append(c); vals.append(coef[c, 0])
        for a in range(3):
            for k, sgn in ((1 + 2 * a, 1), (2 + 2 * a, -1)):
                if coef[c, k] != 0.0:
                    rows.append(c); cols.append(c + sgn * strides[a]); vals.append(coef[c, k])
    full = sp.csr_matrix((vals, (rows, cols)), shape=(m, m)).toarray()
    keep = G["cond/keep"]
    ref = sp.csr_matrix((G["cond/A_val"], (G["cond/A_row"], G["cond/A_col"])), shape=(keep.size, keep.size))
    np.testing.assert_array_equal(full[np.ix_(keep, keep)], ref.toarray())
    cond = np.setdiff1d(np.arange(m), keep)
    np.testing.assert_array_equal(full[cond], np.eye(m)[cond])
    assert not full[np.ix_(keep, cond)].any()


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_gpu_field_from_potential_matches_reference_bitwise(cuda, name):
    torch = cuda
    phi = torch.from_numpy(G[f"{name}/phi"]).cuda()
    e = torch.empty((3,) + tuple(phi.shape), dtype=torch.float64, device="cuda")
    _lib.check(_lib.load().ppt_field_from_potential(_mesh(G[f"{name}/extent"], phi.shape), phi.data_ptr(),
                                                    e[0].data_ptr(), e[1].data_ptr(), e[2].data_ptr(),
                                                    _lib.stream_handle()))
    e = e.cpu().numpy()
    for k, key in enumerate(("ex", "ey", "ez")):
        np.testing.assert_array_equal(e[k], G[f"{name}/{key}"])


@pytest.mark.gpu
def test_gpu_poisson_solve_vs_direct_solve(cuda):
    torch = cuda
    extent, cells = (0.1, 0.08, 0.16), (24, 20, 28)
    rng = np.random.default_rng(7)
    b = rng.normal(0, 1.0, cells)
    exact = sco.spsolve(sco.assemble_matrix(extent, cells).tocsc(), b.ravel()).reshape(cells)
    lib = _lib.load()
    mesh = _mesh(extent, cells)
    scratch = torch.empty(lib.ppt_poisson_scratch_bytes(mesh), dtype=torch.uint8, device="cuda")
    d_b = torch.from_numpy(b).cuda()
    outs = []
    for _ in range(2):
        phi = torch.zeros(cells, dtype=torch.float64, device="cuda")
        it, res = ctypes.c_int64(), ctypes.c_double()
        _lib.check(lib.ppt_poisson_solve(mesh, d_b.data_ptr(), phi.data_ptr(), scratch.data_ptr(), 1e-12, 5000,
                                         it, res, _lib.stream_handle()))
        assert 0 < it.value < 5000 and res.value <= 1e-12
        outs.append(phi.cpu().numpy())
    np.testing.assert_array_equal(outs[0], outs[1])            # deterministic
    err = np.abs(outs[0] - exact).max() / np.abs(exact).max()
    assert err < 1e-8, err
    # the residual the solver reports is the true one
    a = sco.assemble_matrix(extent, cells)
    true_res = np.linalg.norm(a @ outs[0].ravel() - b.ravel()) / np.linalg.norm(b)
    assert true_res < 1e-11


@pytest.mark.gpu
def test_gpu_space_charge_solve_vs_oracle(cuda):
    from pypatools_b200.space_charge import PoissonSolverConfig, SpaceChargeSolver
    rng = np.random.default_rng(8)
    extent, cells = (0.04, 0.04, 0.1), (16, 16, 32)
    n = 50_000
    p = np.column_stack([rng.normal(0, 3e-3, n), rng.normal(0, 3e-3, n), rng.normal(0, 1e-2, n)])
    q = np.full(n, 1.602176634e-19 * 1e4)
    solver = SpaceChargeSolver(PoissonSolverConfig(extent, cells, solver_tol=1e-12))
    phi, field = solver.solve(p, q)
    ref = sco.solve(p, q, extent, cells)
    scale = np.abs(ref[0]).max()
    np.testing.assert_allclose(phi, ref[0], rtol=0, atol=1e-8 * scale)
    e = solver.e.cpu().numpy()
    for k in range(3):
        np.testing.assert_allclose(e[k], ref[k + 1], rtol=0, atol=1e-8 * np.abs(ref[k + 1]).max())
    # the returned Field interpolates the field on the cell centres
    assert field.dim == 3 and solver.turn_count == 1
    pts = np.column_stack([rng.uniform(-0.015, 0.015, 500), rng.uniform(-0.015, 0.015, 500),
                           rng.uniform(-0.04, 0.04, 500)])
    from oracle import pusher_oracle as orc
    oe = orc.MapField(solver.cell_centres(), {"x": ref[1], "y": ref[2], "z": ref[3]})(pts)
    np.testing.assert_allclose(field(pts), oe, rtol=0, atol=1e-8 * np.abs(oe).max())
    # no charge: zero potential, no iterations
    phi0, _ = solver.solve(np.zeros((0, 3)), np.zeros(0))
    assert not np.any(phi0) and solver.last_iterations == 0
    with pytest.raises(NotImplementedError):
        SpaceChargeSolver(PoissonSolverConfig(extent, cells), electrode_assembly=object())


def _electrode_case():
    from pypatools_b200.electrodes import ElectrodeSurface
    # closed solids: a thick beam pipe (wall 12-16 mm) and a 4 mm thick
    # aperture plate (hole 5 mm) at z = 0
    return ElectrodeSurface.annular_cylinder(0.012, 0.016, -0.05, 0.05, n_phi=40, n_z=10) + \
        ElectrodeSurface.annular_cylinder(0.005, 0.012, -0.002, 0.002, n_phi=40, n_z=1)


@pytest.mark.gpu
def test_gpu_axis_rays_match_oracle_bitwise(cuda):
    torch = cuda
    s = _electrode_case()
    rng = np.random.default_rng(12)
    pts = np.column_stack([rng.uniform(-0.02, 0.02, 3000), rng.uniform(-0.02, 0.02, 3000),
                           rng.uniform(-0.06, 0.06, 3000)])
    pts = np.concatenate([pts, [[0.0, 0.0, 0.0], [0.015, 0.0, 0.01], [0.0, 0.0, 0.07]]])
    d_p = torch.from_numpy(pts).cuda()
    dist = torch.empty((pts.shape[0], 6), dtype=torch.float64, device="cuda")
    hits = torch.empty((pts.shape[0], 6), dtype=torch.int32, device="cuda")
    _lib.check(_lib.load().ppt_surface_axis_rays(s.handle("cuda"), pts.shape[0], d_p.data_ptr(), dist.data_ptr(),
                                                 hits.data_ptr(), _lib.stream_handle()))
    ref_d, ref_h = sco.axis_ray_hits(pts, s.vertices, s.triangles)
    np.testing.assert_array_equal(hits.cpu().numpy(), ref_h)
    np.testing.assert_array_equal(dist.cpu().numpy(), ref_d)
    assert (ref_h % 2 == 1).any() and (ref_h == 0).any()


@pytest.mark.gpu
def test_gpu_space_charge_with_conductors_vs_oracle(cuda):
    from pypatools_b200.space_charge import PoissonSolverConfig, SpaceChargeSolver, CONDUCTOR
    s = _electrode_case()
    extent, cells = (0.04, 0.04, 0.1), (16, 16, 40)
    rng = np.random.default_rng(13)
    n = 20000
    p = np.column_stack([rng.normal(0, 2e-3, n), rng.normal(0, 2e-3, n), rng.normal(0.02, 8e-3, n)])
    q = np.full(n, 1.602176634e-19 * 1e5)
    solver = SpaceChargeSolver(PoissonSolverConfig(extent, cells, solver_tol=1e-12, max_iterations=20000),
                               electrode_assembly=s)
    kind = solver.cell_type
    assert (kind == CONDUCTOR).sum() > 100 and (kind == 1).sum() > 100
    # the pipe's inside is vacuum, its wall and the plate are conductor
    assert kind.reshape(cells)[8, 8, 30] == 0 and kind.reshape(cells)[2, 8, 30] == CONDUCTOR
    assert kind.reshape(cells)[1, 8, 30] == 1           # just outside the wall
    assert kind.reshape(cells)[3, 8, 20] == CONDUCTOR
    # the cell types come from the same rays as the oracle's
    gx, gy, gz = solver.cell_centres()
    xx, yy, zz = np.meshgrid(gx, gy, gz, indexing="ij")
    ref_d, ref_h = sco.axis_ray_hits(np.column_stack([xx.ravel(), yy.ravel(), zz.ravel()]), s.vertices,
                                     s.triangles)
    h = (solver.hx, solver.hy, solver.hz)
    np.testing.assert_array_equal(kind, sco.classify_cells(ref_d, ref_h, h))
    phi, _ = solver.solve(p, q)
    assert solver.last_residual <= 1e-12
    a, keep = sco.assemble_reduced(extent, cells, kind, ref_d)
    rho = sco.bin_particles_cic(p, q, extent, cells).reshape(-1)
    x = np.zeros(kind.size)
    x[keep] = sco.spsolve(a.tocsc(), (rho / sco.EPS0)[keep])
    x = x.reshape(cells)
    np.testing.assert_allclose(phi, x, rtol=0, atol=1e-8 * np.abs(x).max())
    assert not phi.reshape(-1)[kind == CONDUCTOR].any()


@pytest.mark.gpu
def test_gpu_space_charge_field_feeds_the_pusher_on_the_device(cuda):
    # a space-charge step then a push: the field left on the device and the
    # host field of the reference's API give the same map, hence the same bits
    torch = cuda
    from pypatools_b200 import PusherGPU, IonSpecies, CompositeField, Field
    from pypatools_b200.space_charge import PoissonSolverConfig, SpaceChargeSolver
    rng = np.random.default_rng(21)
    extent, cells = (0.02, 0.02, 0.06), (16, 16, 48)
    n = 4000
    p = np.column_stack([rng.normal(0, 1.5e-3, n), rng.normal(0, 1.5e-3, n), rng.normal(0, 5e-3, n)])
    v = np.column_stack([rng.normal(0, 1e4, n), rng.normal(0, 1e4, n), np.full(n, 1.0e6)])
    q = np.full(n, 1.602176634e-19 * 1e6)
    solver = SpaceChargeSolver(PoissonSolverConfig(extent, cells, solver_tol=1e-10))
    phi_h, _ = solver.solve(p, q)
    phi_d, e_dev = solver.solve_field_device(torch.from_numpy(p).cuda(), torch.from_numpy(q).cuda())
    assert phi_d.is_cuda and e_dev._field["z"]._values.is_cuda
    # two solves differ only by the deposition's float64 atomics order
    np.testing.assert_allclose(phi_d.cpu().numpy(), phi_h, rtol=0, atol=1e-12 * np.abs(phi_h).max())
    # the same node values through the host (numpy) and the device (tensor) paths
    e_host = Field.from_arrays(dict(zip("xyz", solver.cell_centres())),
                               {c: e_dev._field[c]._values.cpu().numpy() for c in "xyz"})
    b = Field(dim=0, field={"x": 0.0, "y": 0.0, "z": 0.5})
    ion = IonSpecies("proton")
    out = []
    for e in (e_host, e_dev):
        rh, vh, _ = PusherGPU(ion, "boris").track_batch(p, v, CompositeField([e], [1.0]), b, 300, 1e-10, 100)
        out.append((rh, vh))
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])
    assert np.abs(out[0][1][-1] - out[0][1][0]).max() > 0.0      # the space-charge kick is there
    # the device field's node values changed in place count as a new field
    pusher = PusherGPU(ion, "boris")
    comp = CompositeField([e_dev], [1.0])
    rh1, _, _ = pusher.track_batch(p, v, comp, b, 300, 1e-10, 100)
    np.testing.assert_array_equal(rh1, out[1][0])
    e_dev._field["z"]._values.mul_(2.0)
    rh2, _, _ = pusher.track_batch(p, v, comp, b, 300, 1e-10, 100)
    assert not np.array_equal(rh2, rh1)
