"""Generate the space-charge fixture (poisson_golden.npz) by running the reference.

PyAMGPoissonSolver (src/PyPATools/poisson_amg.py) cannot be constructed here:
its constructor classifies cells through the external py_electrodes package
and builds a pyamg hierarchy, neither installed.  So its matrix assembly
(``_assemble_system_matrix``, :293-443) is run on an instance whose mesh
attributes are set directly (those __init__ sets at :178-185) with every cell
interior and no boundary distances, i.e. a domain without conductors, and its
field step ``compute_field_from_potential_numba`` (:98-130) on a seeded
potential.  For conductor cells, its classification (``_classify_cells``,
:241-291) runs on seeded ray results served by a stand-in electrode assembly,
followed by the assembly with Shortley-Weller rows.  The module needs inert stand-ins for cupy and pyamg to import
(see make_golden_cic.py).

    PYPATOOLS_REFERENCE_SRC=<checkout>/src python tests/golden/make_golden_poisson.py
"""
import contextlib
import io
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

from make_golden import load_reference  # noqa: E402


def import_solver_module():
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
    return poisson_amg


def main():
    pa = import_solver_module()
    out = {}
    for name, extent, cells in (("box", (0.1, 0.08, 0.12), (6, 5, 7)), ("flat", (0.3, 0.05, 0.05), (9, 3, 4))):
        s = object.__new__(pa.PyAMGPoissonSolver)
        s.Lx, s.Ly, s.Lz = extent
        s.nx, s.ny, s.nz = cells
        s.hx, s.hy, s.hz = (extent[0] / cells[0], extent[1] / cells[1], extent[2] / cells[2])
        s.n_dofs = cells[0] * cells[1] * cells[2]
        s.cell_type = np.full(s.n_dofs, pa.CellType.INTERIOR, dtype=np.int32)
        s.boundary_distances = np.zeros((s.n_dofs, 6))
        with contextlib.redirect_stdout(io.StringIO()):
            s._assemble_system_matrix()
        a = s.A.tocoo()
        out[f"{name}/extent"] = np.array(extent)
        out[f"{name}/cells"] = np.array(cells)
        out[f"{name}/A_row"], out[f"{name}/A_col"], out[f"{name}/A_val"] = a.row, a.col, a.data
        phi = np.random.default_rng(len(name)).normal(0, 1e3, cells)
        ex, ey, ez = pa.compute_field_from_potential_numba(phi, s.hx, s.hy, s.hz)
        out[f"{name}/phi"] = phi
        out[f"{name}/ex"], out[f"{name}/ey"], out[f"{name}/ez"] = ex, ey, ez
        print(name, "nnz", a.nnz)
    # conductor cells: the reference's classification (:241-291) on ray
    # results served by a stand-in electrode assembly, then its assembly with
    # the Shortley-Weller rows
    rng = np.random.default_rng(17)
    extent, cells = (0.08, 0.07, 0.09), (8, 7, 9)
    m = int(np.prod(cells))
    h = np.array([extent[a] / cells[a] for a in range(3)])
    hits = np.zeros((m, 6), dtype=np.int64)
    dist = np.full((m, 6), np.inf)
    ijk = np.stack(np.meshgrid(*[np.arange(c) for c in cells], indexing="ij"), -1).reshape(-1, 3)
    blob = (np.abs(ijk - np.array([3, 3, 4])) <= np.array([1, 1, 2])).all(axis=1)
    hits[blob] = rng.integers(0, 2, (blob.sum(), 6)) * 2 + 1      # odd: inside the blob
    near = ~blob & (np.abs(ijk - np.array([3, 3, 4])) <= np.array([2, 2, 3])).all(axis=1)
    hits[near] = 2
    dist[near] = rng.uniform(0.05, 1.6, (near.sum(), 6)) * np.repeat(h, 2)
    dist[rng.uniform(size=m) < 0.05, 0] = 1e-9                       # a crossing almost on the centre

    class Electrodes:
        def compute_axis_aligned_surface_intersections(self, mesh_nodes, axes="all", use_gpu=False):
            return dist.copy(), hits.copy()

    s = object.__new__(pa.PyAMGPoissonSolver)
    s.Lx, s.Ly, s.Lz = extent
    s.nx, s.ny, s.nz = cells
    s.hx, s.hy, s.hz = h
    s.n_dofs = m
    s.use_gpu = False
    s.electrodes = Electrodes()
    s.mesh_nodes = np.zeros((m, 3))
    with contextlib.redirect_stdout(io.StringIO()):
        s._classify_cells()
        s._assemble_system_matrix()
    a = s.A.tocoo()
    out.update({"cond/extent": np.array(extent), "cond/cells": np.array(cells), "cond/dist": dist,
                "cond/hits": hits, "cond/cell_type": np.asarray(s.cell_type), "cond/keep": s.keep_indices,
                "cond/A_row": a.row, "cond/A_col": a.col, "cond/A_val": a.data})
    print("cond", "conductor", int((s.cell_type == 2).sum()), "boundary", int((s.cell_type == 1).sum()), "nnz", a.nnz)
    dest = HERE / "poisson_golden.npz"
    np.savez_compressed(dest, **out)
    print("wrote", dest, dest.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
