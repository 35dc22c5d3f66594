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


# ---------------------------------------------------------------------------
# Conductor cells (poisson_amg.py:241-443)
# ---------------------------------------------------------------------------

INTERIOR, BOUNDARY, CONDUCTOR = 0, 1, 2     # CellType (poisson_amg.py:86-90)


def axis_ray_hits(points, vertices, triangles):
    """(min_dist (n,6), hits (n,6)) of the rays from each point along +x, -x,
    +y, -y, +z, -z: crossings counted over every triangle (Moller-Trumbore,
    t >= 0, each product and sum rounded separately), distance to the nearest."""
    p = np.asarray(points, dtype=np.float64).reshape(-1, 3)
    v = np.asarray(vertices, dtype=np.float64)
    t = np.asarray(triangles, dtype=np.int64)
    v0 = v[t[:, 0]]
    e1 = v[t[:, 1]] - v0
    e2 = v[t[:, 2]] - v0
    dist = np.full((p.shape[0], 6), np.inf)
    hits = np.zeros((p.shape[0], 6), dtype=np.int32)

    def cross(a, b):
        return np.stack([a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1],
                         a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                         a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]], axis=-1)

    def dot(a, b):
        return a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1] + a[..., 2] * b[..., 2]

    for direction in range(6):
        d = np.zeros(3)
        d[direction // 2] = -1.0 if direction % 2 else 1.0
        pv = cross(d[None, :], e2)                        # per triangle
        det = dot(e1, pv)
        with np.errstate(divide="ignore", invalid="ignore"):
            inv = 1.0 / det
            for s in range(0, p.shape[0], 2048):
                tv = p[s:s + 2048, None, :] - v0[None]
                u = dot(tv, pv[None]) * inv[None]
                qv = cross(tv, e1[None])
                w = dot(d[None, None, :], qv) * inv[None]
                tt = dot(e2[None], qv) * inv[None]
                ok = (det != 0.0)[None] & (u >= 0.0) & (u <= 1.0) & (w >= 0.0) & (u + w <= 1.0) & (tt >= 0.0)
                hits[s:s + 2048, direction] = ok.sum(axis=1)
                dist[s:s + 2048, direction] = np.where(ok, tt, np.inf).min(axis=1)
    return dist, hits


def classify_cells(min_dist, hits, h):
    """Cell types (poisson_amg.py:258-281): a conductor where a ray crosses the
    surface an odd number of times in any direction; a boundary cell where a
    crossing is within one cell size (compared with the sizes as float32)."""
    is_cond = (hits % 2 != 0).any(axis=1)
    sizes = np.array([h[0], h[0], h[1], h[1], h[2], h[2]], dtype=np.float32)
    is_bnd = (min_dist <= sizes).any(axis=1) & ~is_cond
    out = np.full(hits.shape[0], INTERIOR, dtype=np.int32)
    out[is_bnd] = BOUNDARY
    out[is_cond] = CONDUCTOR
    return out


def assemble_reduced(extent, cells, cell_type, dist):
    """(A, keep): the reference's reduced system over the non-conductor cells,
    row by row as its assembly loop writes them (Shortley-Weller distances
    towards conductor neighbours, at least h / 1000)."""
    n = [int(c) for c in cells]
    h = [float(e) / c for e, c in zip(extent, n)]
    m = n[0] * n[1] * n[2]
    keep = np.nonzero(cell_type != CONDUCTOR)[0]
    new = np.full(m, -1, dtype=np.int64)
    new[keep] = np.arange(keep.size)
    strides = (n[1] * n[2], n[2], 1)
    rows, cols, vals = [], [], []
    for c in keep:
        ijk = (c // strides[0], (c // strides[1]) % n[1], c % n[2])
        diag = 0.0
        for a in range(3):
            has_pos, has_neg = ijk[a] + 1 < n[a], ijk[a] > 0
            pos, neg = c + strides[a], c - strides[a]
            cond_pos = has_pos and cell_type[pos] == CONDUCTOR
            cond_neg = has_neg and cell_type[neg] == CONDUCTOR
            hp = max(dist[c, 2 * a], h[a] * 1e-3) if cond_pos else h[a]
            hn = max(dist[c, 2 * a + 1], h[a] * 1e-3) if cond_neg else h[a]
            diag += 2.0 / (hp * hn)
            if has_pos and not cond_pos:
                rows.append(new[c]); cols.append(new[pos]); vals.append(-2.0 / (hp * (hp + hn)))
            if has_neg and not cond_neg:
                rows.append(new[c]); cols.append(new[neg]); vals.append(-2.0 / (hn * (hp + hn)))
        rows.append(new[c]); cols.append(new[c]); vals.append(diag)
    a = sp.csr_matrix((vals, (rows, cols)), shape=(keep.size, keep.size))
    a.eliminate_zeros()
    return a, keep
