"""Generate the CIC deposition fixture (cic_golden.npz) by running the reference.

The reference deposits particle charge onto its Poisson mesh with
``PyAMGPoissonSolver._bin_particles_cic_cpu`` (src/PyPATools/poisson_amg.py:849-878),
which calls the Numba kernel ``_cic_deposit_numba`` (:880-911).  That kernel does
not compile under Numba 0.65 (``np.clip`` on integer scalars, :889-891, has no
nopython implementation), and it adds to ``rho`` from a ``prange`` loop without
atomics (concurrent updates of a node could be lost); so the fixture runs the
kernel's own Python source (the Numba dispatcher's ``py_func``) as plain,
sequential Python.  The solver's constructor builds
the whole mesh and needs ``pyamg`` and ``py_electrodes`` (not installed), so
the method is called on an instance whose grid attributes are set directly
(the ones ``__init__`` sets at :178-185: extents, cell counts, spacings L/n).
The module also cannot be imported without cupy (see ``main``).

    PYPATOOLS_REFERENCE_SRC=<checkout>/src python tests/golden/make_golden_cic.py
"""
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

from make_golden import load_reference  # noqa: E402


def cases():
    """(name, particles (M,3), charges (M,), domain_extent, mesh_cells)."""
    out = []
    rng = np.random.default_rng(11)
    ext, cells = (0.2, 0.15, 0.1), (16, 12, 10)
    p = rng.uniform(-0.5, 0.5, (20000, 3)) * np.array(ext) * 0.95
    out.append(("inside", p, rng.uniform(0.5, 1.5, 20000) * 1e-15, ext, cells))
    # partly outside (clamped onto the boundary nodes), nodes and last node exactly
    h = np.array(ext) / np.array(cells)
    p = rng.uniform(-0.7, 0.7, (5000, 3)) * np.array(ext)
    nodes = np.array([[-ext[0] / 2 + i * h[0], -ext[1] / 2 + j * h[1], -ext[2] / 2 + k * h[2]]
                      for i, j, k in [(0, 0, 0), (cells[0] - 1, cells[1] - 1, cells[2] - 1), (3, 5, 7),
                                      (cells[0] - 1, 0, 4), (2, cells[1] - 1, cells[2] - 1)]])
    p = np.concatenate([p, nodes])
    out.append(("edges", p, rng.normal(0.0, 1e-15, len(p)), ext, cells))
    ext, cells = (1.0, 0.5, 2.0), (7, 5, 9)
    p = rng.normal(0.0, 0.2, (3000, 3)) * np.array(ext)
    out.append(("anisotropic", p, np.full(3000, 1.6e-19), ext, cells))
    return out


def main():
    # pyamg is not installed; cupy neither, and poisson_amg.py evaluates a
    # `-> cp.ndarray` annotation at class definition (:801), which fails when
    # its cupy import fails, so inert stand-ins are registered for both
    sys.modules.setdefault("pyamg", types.ModuleType("pyamg"))
    cupy = types.ModuleType("cupy")
    cupy.ndarray = type("ndarray", (), {})
    sys.modules.setdefault("cupy", cupy)
    for name in ("cupyx", "cupyx.scipy", "cupyx.scipy.sparse"):
        sys.modules.setdefault(name, types.ModuleType(name))
    sys.modules["cupyx"].scipy = sys.modules["cupyx.scipy"]
    sys.modules["cupyx.scipy"].sparse = sys.modules["cupyx.scipy.sparse"]
    load_reference()
    from PyPATools import poisson_amg
    arrays = {}
    for name, p, q, ext, cells in cases():
        solver = object.__new__(poisson_amg.PyAMGPoissonSolver)
        solver.Lx, solver.Ly, solver.Lz = ext
        solver.nx, solver.ny, solver.nz = cells
        solver.hx, solver.hy, solver.hz = (ext[0] / cells[0], ext[1] / cells[1], ext[2] / cells[2])
        solver.n_dofs = cells[0] * cells[1] * cells[2]
        solver._cic_deposit_numba = poisson_amg.PyAMGPoissonSolver._cic_deposit_numba.py_func
        rho = solver._bin_particles_cic_cpu(np.ascontiguousarray(p, dtype=np.float64),
                                            np.ascontiguousarray(q, dtype=np.float64))
        arrays[f"{name}_particles"] = p
        arrays[f"{name}_charges"] = q
        arrays[f"{name}_extent"] = np.array(ext, dtype=np.float64)
        arrays[f"{name}_cells"] = np.array(cells, dtype=np.int64)
        arrays[f"{name}_rho"] = np.asarray(rho, dtype=np.float64)
        print(name, len(q), "particles, rho sum", float(np.sum(rho)), "nodes", rho.size)
    np.savez_compressed(HERE / "cic_golden.npz", **arrays)


if __name__ == "__main__":
    main()
