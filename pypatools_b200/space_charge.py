"""Space-charge field of a bunch on the GPU: charge deposition, Poisson solve
and E = -grad phi, with the API of the reference's ``PyAMGPoissonSolver``
(src/PyPATools/poisson_amg.py:58-84, :133-797).

    config = PoissonSolverConfig(domain_extent=(Lx, Ly, Lz), mesh_cells=(nx, ny, nz))
    solver = SpaceChargeSolver(config)
    phi_3d, e_field = solver.solve(particles, charges)   # (nx,ny,nz) V, Field in V/m

As in the reference: the charge is deposited by cloud-in-cell onto nodes
spaced extent / cells from -extent / 2 (``_bin_particles_cic_cpu``, :849-911)
and the resulting array is used as the density of the solver's cells, centred
at -extent / 2 + (i + 1/2) h, half a cell away (the two grids are not aligned
in the reference; that is kept); the operator is the 7-point Laplacian with
zero potential beyond the box; the field is central differences on the
interior, zero on the outer layer; ``e_field`` is a trilinear ``Field`` on
the cell centres.  The linear solve is conjugate gradients to
``solver_tol`` (the reference: GMRES with an AMG preconditioner to the same
relative residual).

With an electrode assembly (an ``ElectrodeSurface`` or any object with
``vertices`` / ``triangles``), the cells are classified as the reference
does (:241-291) from rays cast along the six axis directions from every cell
centre (``ppt_surface_axis_rays``): conductor where some ray crosses the
surface an odd number of times, boundary where a crossing lies within one
cell size.  Conductor cells hold zero potential; the rows next to them use the
distances to the surface (Shortley-Weller, :293-443); that operator is not
symmetric, so the solve is BiCGSTAB (``ppt_poisson_solve_coef``).
"""
import time

import numpy as np
from scipy import constants as _const

from . import _lib

EPS0 = _const.epsilon_0

INTERIOR, BOUNDARY, CONDUCTOR = 0, 1, 2   # the reference's CellType (poisson_amg.py:86-90)


def classify_cells(min_dist, hits, h):
    """Cell types from the six axis rays of each cell centre
    (poisson_amg.py:258-281); the cell sizes are compared as float32, as there."""
    conductor = (hits % 2 != 0).any(axis=1)
    sizes = np.array([h[0], h[0], h[1], h[1], h[2], h[2]], dtype=np.float32)
    boundary = (min_dist <= sizes).any(axis=1) & ~conductor
    kind = np.full(hits.shape[0], INTERIOR, dtype=np.int32)
    kind[boundary] = BOUNDARY
    kind[conductor] = CONDUCTOR
    return kind


def operator_coefficients(cells, h, cell_type, dist):
    """(m, 7) rows of the operator: diagonal and +x, -x, +y, -y, +z, -z
    couplings, as the reference's assembly loop forms them (poisson_amg.py:
    322-437): towards a conductor neighbour the spacing is the distance to the
    surface (at least h / 1000) and the coupling is dropped; a conductor cell's
    row is the identity."""
    n = tuple(int(c) for c in cells)
    kind = np.asarray(cell_type).reshape(n)
    cond = kind == CONDUCTOR
    d = np.asarray(dist, dtype=np.float64).reshape(n + (6,))
    coef = np.zeros(n + (7,))
    diag = np.zeros(n)
    for a in range(3):
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[a], hi[a] = slice(0, n[a] - 1), slice(1, n[a])
        lo, hi = tuple(lo), tuple(hi)
        has_pos = np.zeros(n, dtype=bool)
        has_pos[lo] = True
        has_neg = np.zeros(n, dtype=bool)
        has_neg[hi] = True
        cond_pos = np.zeros(n, dtype=bool)
        cond_pos[lo] = cond[hi]
        cond_neg = np.zeros(n, dtype=bool)
        cond_neg[hi] = cond[lo]
        floor = h[a] * 1e-3
        hp = np.where(cond_pos, np.maximum(d[..., 2 * a], floor), h[a])
        hn = np.where(cond_neg, np.maximum(d[..., 2 * a + 1], floor), h[a])
        diag = diag + 2.0 / (hp * hn)
        coef[..., 1 + 2 * a] = np.where(has_pos & ~cond_pos, -2.0 / (hp * (hp + hn)), 0.0)
        coef[..., 2 + 2 * a] = np.where(has_neg & ~cond_neg, -2.0 / (hn * (hp + hn)), 0.0)
    coef[..., 0] = diag
    coef[cond] = 0.0
    coef[cond, 0] = 1.0
    return coef.reshape(-1, 7)


class PoissonSolverConfig:
    """The reference's ``PyAMGSolverConfig`` fields that apply here."""

    def __init__(self, domain_extent, mesh_cells, solver_tol=1e-6, max_iterations=None, use_gpu=True,
                 interpolator_backend="auto"):
        self.domain_extent = tuple(float(v) for v in domain_extent)
        self.mesh_cells = tuple(int(v) for v in mesh_cells)
        self.solver_tol = float(solver_tol)
        # conjugate gradients without a preconditioner needs O(n) iterations
        self.max_iterations = int(max_iterations) if max_iterations is not None else 20 * max(self.mesh_cells)
        self.use_gpu = use_gpu
        self.interpolator_backend = interpolator_backend


def check_device_inputs(particles, charges, device):
    """(particles, charges) as the deposit kernel reads them: float64 tensors
    on ``device``, (M, 3) row-major and (M,), contiguous.  Anything else is
    refused here (a float32 or host array would be read past its end)."""
    import torch
    if not (torch.is_tensor(particles) and torch.is_tensor(charges)):
        raise TypeError("particles and charges must be torch tensors on the solver's device "
                        "(solve() takes numpy arrays)")
    if particles.dtype != torch.float64 or charges.dtype != torch.float64:
        raise TypeError(f"particles and charges must be float64, got {particles.dtype} and {charges.dtype}")
    if particles.dim() != 2 or particles.shape[1] != 3 or tuple(charges.shape) != (particles.shape[0],):
        raise ValueError(f"particles must be (M, 3) and charges (M,), got {tuple(particles.shape)} and "
                         f"{tuple(charges.shape)}")
    if particles.device != device or charges.device != device:
        raise ValueError(f"particles and charges must be on {device}, got {particles.device} and {charges.device}")
    return particles.contiguous(), charges.contiguous()


class SpaceChargeSolver:
    """GPU counterpart of ``PyAMGPoissonSolver`` (conductor cells from an
    optional electrode assembly)."""

    def __init__(self, config, electrode_assembly=None, device=None):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("the space-charge solver runs on the GPU (no CPU fallback)")
        self.config = config
        self.lib = _lib.load()
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.Lx, self.Ly, self.Lz = config.domain_extent
        self.nx, self.ny, self.nz = config.mesh_cells
        self.hx, self.hy, self.hz = self.Lx / self.nx, self.Ly / self.ny, self.Lz / self.nz
        self.n_dofs = self.nx * self.ny * self.nz
        self.mesh = _lib.MeshDesc()
        for a, (e, c) in enumerate(zip(config.domain_extent, config.mesh_cells)):
            self.mesh.extent[a] = e
            self.mesh.cells[a] = c
        shape = (self.nx, self.ny, self.nz)
        self.cell_type = None
        self._coef = None
        self._conductor = None
        if electrode_assembly is not None:
            self._classify(electrode_assembly)
        nbytes = (self.lib.ppt_poisson_coef_scratch_bytes if self._coef is not None
                  else self.lib.ppt_poisson_scratch_bytes)(self.mesh)
        if nbytes < 0:
            _lib.check(-1)
        self._scratch = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        self._rho = torch.empty(shape, dtype=torch.float64, device=self.device)
        self.phi = torch.zeros(shape, dtype=torch.float64, device=self.device)
        self.e = torch.empty((3,) + shape, dtype=torch.float64, device=self.device)
        self.turn_count = 0
        self.solve_times = []
        self.last_iterations = 0
        self.last_residual = 0.0

    def _classify(self, electrode_assembly):
        """Cell types and operator rows from the electrode surfaces (the
        reference's one-time setup, poisson_amg.py:241-443)."""
        import torch
        from .electrodes import ElectrodeSurface
        surf = ElectrodeSurface.from_assembly(electrode_assembly)
        gx, gy, gz = self.cell_centres()
        xx, yy, zz = np.meshgrid(gx, gy, gz, indexing="ij")
        nodes = torch.from_numpy(np.column_stack([xx.ravel(), yy.ravel(), zz.ravel()])).to(self.device)
        dist = torch.empty((self.n_dofs, 6), dtype=torch.float64, device=self.device)
        hits = torch.empty((self.n_dofs, 6), dtype=torch.int32, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.ppt_surface_axis_rays(surf.handle(self.device), self.n_dofs, nodes.data_ptr(),
                                                      dist.data_ptr(), hits.data_ptr(), _lib.stream_handle()))
        self.boundary_distances = dist.cpu().numpy()
        self.hit_counts = hits.cpu().numpy()
        h = (self.hx, self.hy, self.hz)
        self.cell_type = classify_cells(self.boundary_distances, self.hit_counts, h)
        coef = operator_coefficients((self.nx, self.ny, self.nz), h, self.cell_type, self.boundary_distances)
        self._coef = torch.from_numpy(coef).to(self.device)
        self._conductor = torch.from_numpy(self.cell_type == CONDUCTOR).to(self.device).reshape(
            self.nx, self.ny, self.nz)

    def cell_centres(self):
        """The solver's cell-centre coordinates per axis (poisson_amg.py:229-231)."""
        return tuple(np.linspace(-L / 2 + h / 2, L / 2 - h / 2, n)
                     for L, h, n in ((self.Lx, self.hx, self.nx), (self.Ly, self.hy, self.ny),
                                     (self.Lz, self.hz, self.nz)))

    def solve_device(self, particles, charges, stream=None):
        """Deposit, solve and differentiate on the device.  particles: (M,3)
        float64 CUDA tensor, charges: (M,) float64 CUDA tensor.  Leaves phi in
        ``self.phi`` and (Ex, Ey, Ez) in ``self.e``; returns them.  Everything
        runs on ``stream`` (default: the current stream)."""
        import torch
        particles, charges = check_device_inputs(particles, charges, self._rho.device)
        if stream is not None:
            with torch.cuda.stream(stream):
                return self.solve_device(particles, charges)
        st = _lib.stream_handle()
        m = int(particles.shape[0])
        _lib.check(self.lib.ppt_deposit_cic(m, particles.data_ptr() if m else None,
                                            charges.data_ptr() if m else None, self.mesh, self._rho.data_ptr(), st))
        self._rho.div_(EPS0)                 # rhs = rho / eps0 (poisson_amg.py:917)
        self.phi.zero_()                     # the reference starts GMRES from zero
        iters, res = _lib.c_int64(), _lib.c_double()
        if self._coef is None:
            _lib.check(self.lib.ppt_poisson_solve(self.mesh, self._rho.data_ptr(), self.phi.data_ptr(),
                                                  self._scratch.data_ptr(), self.config.solver_tol,
                                                  self.config.max_iterations, iters, res, st))
        else:
            # conductor cells: zero potential, their charge dropped (:919-921, :727-729)
            self._rho.masked_fill_(self._conductor, 0.0)
            _lib.check(self.lib.ppt_poisson_solve_coef(self.mesh, self._coef.data_ptr(), self._rho.data_ptr(),
                                                       self.phi.data_ptr(), self._scratch.data_ptr(),
                                                       self.config.solver_tol, self.config.max_iterations,
                                                       iters, res, st))
            self.phi.masked_fill_(self._conductor, 0.0)
        self.last_iterations, self.last_residual = iters.value, res.value
        _lib.check(self.lib.ppt_field_from_potential(self.mesh, self.phi.data_ptr(), self.e[0].data_ptr(),
                                                     self.e[1].data_ptr(), self.e[2].data_ptr(), st))
        return self.phi, self.e

    def solve_field_device(self, particles, charges, stream=None):
        """(phi tensor, E Field) with the field's node values left on the
        device: a tracker built from it copies them into its map device to
        device, so a space-charge step feeds the next push without a host
        round trip.  particles / charges: CUDA tensors."""
        from .field import Field
        phi, e = self.solve_device(particles, charges, stream)
        gx, gy, gz = self.cell_centres()
        field = Field.from_arrays({"x": gx, "y": gy, "z": gz}, {"x": e[0].clone(), "y": e[1].clone(), "z": e[2].clone()},
                                  label=f"Space-charge E-field (turn {self.turn_count})", dim=3, scaling=1.0,
                                  units="m", method="linear", interpolator_backend="auto")
        self.turn_count += 1
        return phi.clone(), field

    def solve(self, particles, charges):
        """(phi_3d (nx, ny, nz) numpy [V], E_field Field [V/m]) as the
        reference's ``solve`` returns (poisson_amg.py:616-797)."""
        import torch
        from .field import Field
        t0 = time.time()
        p = particles if torch.is_tensor(particles) else torch.from_numpy(
            np.ascontiguousarray(particles, dtype=np.float64))
        q = charges if torch.is_tensor(charges) else torch.from_numpy(np.ascontiguousarray(charges, dtype=np.float64))
        with torch.cuda.device(self.device):
            phi, e = self.solve_device(p.to(self.device).contiguous(), q.to(self.device).contiguous())
            phi_h = phi.cpu().numpy()
            e_h = e.cpu().numpy()
        gx, gy, gz = self.cell_centres()
        field = Field.from_arrays({"x": gx, "y": gy, "z": gz}, {"x": e_h[0], "y": e_h[1], "z": e_h[2]},
                                  label=f"Space-charge E-field (turn {self.turn_count})", dim=3, scaling=1.0,
                                  units="m", method="linear",
                                  interpolator_backend="auto")
        self.solve_times.append(time.time() - t0)
        self.turn_count += 1
        return phi_h, field
