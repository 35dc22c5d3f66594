"""CPU oracle for the cloud-in-cell charge deposition.

TEST INFRASTRUCTURE ONLY.  Nothing in the product imports this module: only
``tests/`` and ``bench.py``'s CPU-baseline leg use it, as the checker.

A vectorised NumPy restatement, in float64, of the reference's
``PyAMGPoissonSolver._bin_particles_cic_cpu`` and ``_cic_deposit_numba``
(src/PyPATools/poisson_amg.py:849-911), with the mesh of its ``__init__``
(:178-185: ``h = extent / cells``, ``cells`` nodes per axis from
``-extent / 2``).  The corner contributions are accumulated particle by
particle, corners in the reference's loop order, so the sum is the
reference's sequential one.  Pinned by ``tests/test_deposit.py`` against
``tests/golden/cic_golden.npz`` (made by running the reference's own kernel
source, ``tests/golden/make_golden_cic.py``).
"""
import numpy as np


def bin_particles_cic(particles, charges, domain_extent, mesh_cells):
    """rho (cells[0]*cells[1]*cells[2],) float64, [i][j][k] with k fastest."""
    p = np.asarray(particles, dtype=np.float64).reshape(-1, 3)
    q = np.asarray(charges, dtype=np.float64).reshape(-1)
    ext = [float(e) for e in domain_extent]
    n = [int(c) for c in mesh_cells]
    h = [ext[a] / n[a] for a in range(3)]
    rho = np.zeros(n[0] * n[1] * n[2], dtype=np.float64)
    if len(q) == 0:
        return rho / (h[0] * h[1] * h[2])
    g = [np.clip((p[:, a] + ext[a] / 2) / h[a], 0, n[a] - 1) for a in range(3)]   # :861-867
    i = [np.floor(g[a]).astype(np.int64) for a in range(3)]                          # :886-888
    f = [g[a] - i[a] for a in range(3)]                                              # :890-892 order: f first
    i = [np.clip(i[a], 0, n[a] - 2) for a in range(3)]                               # then the clip
    idx = np.empty((len(q), 8), dtype=np.int64)
    val = np.empty((len(q), 8), dtype=np.float64)
    c = 0
    for di in (0, 1):
        for dj in (0, 1):
            for dk in (0, 1):
                jx, jy, jz = (i[0] + di) % n[0], (i[1] + dj) % n[1], (i[2] + dk) % n[2]
                idx[:, c] = jx * (n[1] * n[2]) + jy * n[2] + jz
                w = ((1.0 - f[0]) if di == 0 else f[0]) * ((1.0 - f[1]) if dj == 0 else f[1]) * \
                    ((1.0 - f[2]) if dk == 0 else f[2])
                val[:, c] = q * w
                c += 1
    np.add.at(rho, idx.reshape(-1), val.reshape(-1))
    return rho / (h[0] * h[1] * h[2])
