"""CPU restatement of the reference's space-charge solve without conductor
cells (src/PyPATools/poisson_amg.py): the 7-point operator as its matrix
assembly builds it (:293-443, every cell interior), rhs = rho / eps0
(:913-921), a direct sparse solve, and E = -grad phi by central differences
on the interior (compute_field_from_potential_numba, :98-130).

TEST INFRASTRUCTURE ONLY: used by tests/ and by bench.py's CPU baseline of the
space-charge leg, as the checker; nothing in the product imports it.
"""
import numpy as np
import scipy.sparse as sp
from scipy import constants
from scipy.sparse.linalg import spsolve, cg

from oracle.deposit_oracle import bin_particles_cic

EPS0 = constants.epsilon_0


def assemble_matrix(extent, cells):
    """CSR matrix of the operator, rows and columns in [i][j][k] order (k
    fastest): per axis 2 / (h h) on the diagonal (summed x, y, z from 0) and
    -2 / (h (h + h)) for each neighbour inside the box."""
    n = [int(c) for c in cells]
    h = [float(e) / c for e, c in zip(extent, n)]
    m = n[0] * n[1] * n[2]
    idx = np.arange(m).reshape(n)
    diag = 0.0
    for a in range(3):
        diag += 2.0 / (h[a] * h[a])
    rows, cols, vals = [idx.ravel()], [idx.ravel()], [np.full(m, diag)]
    for a in range(3):
        off = -2.0 / (h[a] * (h[a] + h[a]))
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[a], hi[a] = slice(0, n[a] - 1), slice(1, n[a])
        a_lo, a_hi = idx[tuple(lo)].ravel(), idx[tuple(hi)].ravel()
        rows += [a_lo, a_hi]
        cols += [a_hi, a_lo]
        vals += [np.full(a_lo.size, off), np.full(a_hi.size, off)]
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(m, m))


def field_from_potential(phi, extent):
    """(Ex, Ey, Ez) = -grad phi at the cells with three interior indices, 0 on
    the outer layer; each difference divided by 2 h as the reference writes it."""
    nx, ny, nz = phi.shape
    hx, hy, hz = (float(e) / c for e, c in zip(extent, phi.shape))
    ex, ey, ez = (np.zeros(phi.shape) for _ in range(3))
    inner = (slice(1, nx - 1), slice(1, ny - 1), slice(1, nz - 1))
    ex[inner] = -(phi[2:, 1:-1, 1:-1] - phi[:-2, 1:-1, 1:-1]) / (2 * hx)
    ey[inner] = -(phi[1:-1, 2:, 1:-1] - phi[1:-1, :-2, 1:-1]) / (2 * hy)
    ez[inner] = -(phi[1:-1, 1:-1, 2:] - phi[1:-1, 1:-1, :-2]) / (2 * hz)
    return ex, ey, ez


def solve(particles, charges, extent, cells, iterative_tol=None):
    """(phi, Ex, Ey, Ez): deposition onto the nodes, the rho array taken as the
    cells' density (as the reference does), the operator solved directly, or
    by conjugate gradients to ``iterative_tol`` for large meshes."""
    rho = bin_particles_cic(particles, charges, extent, cells).reshape(-1)
    b = rho / EPS0
    a = assemble_matrix(extent, cells)
    if iterative_tol is None:
        x = spsolve(a.tocsc(), b)
    else:
        x, _ = cg(a, b, rtol=iterative_tol, atol=0.0, maxiter=20 * max(cells))
    phi = x.reshape([int(c) for c in cells])
    return (phi,) + field_from_potential(phi, extent)
