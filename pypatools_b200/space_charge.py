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
relative residual).  Conductor cells (electrode geometry from py_electrodes,
Shortley-Weller boundaries) are not on the GPU path: an electrode assembly
raises ``NotImplementedError``.
"""
import time

import numpy as np
from scipy import constants as _const

from . import _lib

EPS0 = _const.epsilon_0


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


class SpaceChargeSolver:
    """GPU counterpart of ``PyAMGPoissonSolver`` for a domain without conductors."""

    def __init__(self, config, electrode_assembly=None, device=None):
        import torch
        if electrode_assembly is not None:
            raise NotImplementedError("conductor cells (electrode geometry) are not on the GPU Poisson path")
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
        nbytes = self.lib.ppt_poisson_scratch_bytes(self.mesh)
        if nbytes < 0:
            _lib.check(-1)
        shape = (self.nx, self.ny, self.nz)
        self._scratch = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        self._rho = torch.empty(shape, dtype=torch.float64, device=self.device)
        self.phi = torch.zeros(shape, dtype=torch.float64, device=self.device)
        self.e = torch.empty((3,) + shape, dtype=torch.float64, device=self.device)
        self.turn_count = 0
        self.solve_times = []
        self.last_iterations = 0
        self.last_residual = 0.0

    def cell_centres(self):
        """The solver's cell-centre coordinates per axis (poisson_amg.py:229-231)."""
        return tuple(np.linspace(-L / 2 + h / 2, L / 2 - h / 2, n)
                     for L, h, n in ((self.Lx, self.hx, self.nx), (self.Ly, self.hy, self.ny),
                                     (self.Lz, self.hz, self.nz)))

    def solve_device(self, particles, charges, stream=None):
        """Deposit, solve and differentiate on the device.  particles: (M,3)
        float64 CUDA tensor, charges: (M,) float64 CUDA tensor.  Leaves phi in
        ``self.phi`` and (Ex, Ey, Ez) in ``self.e``; returns them."""
        st = _lib.stream_handle(stream)
        m = int(particles.shape[0])
        _lib.check(self.lib.ppt_deposit_cic(m, particles.data_ptr() if m else None,
                                            charges.data_ptr() if m else None, self.mesh, self._rho.data_ptr(), st))
        self._rho.div_(EPS0)                 # rhs = rho / eps0 (poisson_amg.py:917)
        self.phi.zero_()                     # the reference starts GMRES from zero
        iters, res = _lib.c_int64(), _lib.c_double()
        _lib.check(self.lib.ppt_poisson_solve(self.mesh, self._rho.data_ptr(), self.phi.data_ptr(),
                                              self._scratch.data_ptr(), self.config.solver_tol,
                                              self.config.max_iterations, iters, res, st))
        self.last_iterations, self.last_residual = iters.value, res.value
        _lib.check(self.lib.ppt_field_from_potential(self.mesh, self.phi.data_ptr(), self.e[0].data_ptr(),
                                                     self.e[1].data_ptr(), self.e[2].data_ptr(), st))
        return self.phi, self.e

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
