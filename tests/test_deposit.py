"""Cloud-in-cell charge deposition (ppt_deposit_cic) against the reference.

The oracle is pinned bit for bit to the reference's own deposition kernel run
on the fixtures in tests/golden/cic_golden.npz; the GPU kernel accumulates with
float64 atomics (and whole-warp sums for warps in one cell), so it agrees with
the sequential sum to rounding: rtol 1e-12 of the largest |rho|."""
import ctypes

import numpy as np
import pytest

from oracle.deposit_oracle import bin_particles_cic as oracle_cic
from pypatools_b200 import _lib
from tests.conftest import REPO

GOLDEN = np.load(REPO / "tests" / "golden" / "cic_golden.npz")
CASES = ("inside", "edges", "anisotropic")


def _case(name):
    return (GOLDEN[f"{name}_particles"], GOLDEN[f"{name}_charges"], GOLDEN[f"{name}_extent"],
            GOLDEN[f"{name}_cells"], GOLDEN[f"{name}_rho"])


def _close(rho, ref):
    scale = max(np.abs(ref).max(), 1e-300)
    np.testing.assert_allclose(rho, ref, rtol=0, atol=1e-12 * scale)


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_fixture(name):
    p, q, ext, cells, rho = _case(name)
    np.testing.assert_array_equal(oracle_cic(p, q, ext, cells), rho)


def test_deposit_argument_errors_without_gpu():
    lib = _lib.load()
    mesh = _lib.MeshDesc()
    assert lib.ppt_deposit_cic(0, None, None, None, None, None) == -1
    for a in range(3):
        mesh.extent[a] = 1.0
        mesh.cells[a] = 4
    assert lib.ppt_deposit_cic(-1, None, None, mesh, ctypes.c_void_p(16), None) == -1
    assert lib.ppt_deposit_cic(5, None, None, mesh, ctypes.c_void_p(16), None) == -1
    mesh.cells[1] = 1
    assert lib.ppt_deposit_cic(0, None, None, mesh, ctypes.c_void_p(16), None) == -1
    assert b"2 nodes" in lib.ppt_last_error()


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_gpu_deposit_matches_reference_fixture(cuda, name):
    from pypatools_b200 import bin_particles_cic
    p, q, ext, cells, rho = _case(name)
    _close(bin_particles_cic(p, q, ext, cells), rho)


@pytest.mark.gpu
def test_gpu_deposit_sorted_bunch_and_conservation(cuda):
    # a dense, cell-sorted bunch: most warps lie in one cell and take the
    # whole-warp sum; charge is conserved exactly up to rounding
    import torch
    from pypatools_b200 import bin_particles_cic
    rng = np.random.default_rng(5)
    n = 400_000
    ext, cells = (0.04, 0.04, 0.2), (24, 24, 96)
    p = np.column_stack([rng.normal(0, 2e-3, n), rng.normal(0, 2e-3, n), rng.uniform(-0.09, 0.09, n)])
    h = np.array(ext) / np.array(cells)
    key = np.floor((p + np.array(ext) / 2) / h).astype(np.int64)
    p = p[np.lexsort((key[:, 2], key[:, 1], key[:, 0]))]
    q = rng.uniform(0.9, 1.1, n) * 1.6e-19
    ref = oracle_cic(p, q, ext, cells)
    for _ in range(2):                       # two calls in a row: rho is overwritten, not accumulated
        rho = bin_particles_cic(p, q, ext, cells)
        _close(rho, ref)
    np.testing.assert_allclose(rho.sum() * h.prod(), q.sum(), rtol=1e-12)
    # device tensors in, device tensor out
    d = bin_particles_cic(torch.from_numpy(p).cuda(), torch.from_numpy(q).cuda(), ext, cells)
    assert d.is_cuda
    _close(d.cpu().numpy(), ref)


@pytest.mark.gpu
def test_gpu_deposit_nan_and_empty(cuda):
    from pypatools_b200 import bin_particles_cic
    ext, cells = (0.1, 0.1, 0.1), (8, 8, 8)
    p = np.array([[0.0, 0.0, 0.0], [np.nan, 0.0, 0.0], [0.01, -0.02, 0.03]])
    q = np.array([1.0, 5.0, 2.0])
    rho = bin_particles_cic(p, q, ext, cells)
    _close(rho, oracle_cic(p[[0, 2]], q[[0, 2]], ext, cells))
    empty = bin_particles_cic(np.zeros((0, 3)), np.zeros(0), ext, cells)
    assert empty.shape == (512,) and not np.any(empty)
