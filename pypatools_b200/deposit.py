"""Cloud-in-cell charge deposition on the GPU: the particle -> mesh step of the
reference's space-charge solver (``PyAMGPoissonSolver._bin_particles_cic_cpu``,
src/PyPATools/poisson_amg.py:849-911), through ``ppt_deposit_cic``.

    rho = bin_particles_cic(particles, charges, domain_extent, mesh_cells)

``particles`` (M, 3) positions [m] and ``charges`` (M,) [C], as NumPy arrays
(rho comes back as NumPy, like the reference's CPU path) or CUDA tensors (rho
stays on the device).  ``domain_extent`` and ``mesh_cells`` are the reference's
``PyAMGSolverConfig`` fields: a mesh of ``mesh_cells`` nodes per axis spaced
``extent / cells`` from ``-extent / 2``.  rho is the charge per cell volume,
flat in [i][j][k] order (k fastest), as the reference returns it.
"""
import numpy as np

from . import _lib


def _mesh(domain_extent, mesh_cells):
    m = _lib.MeshDesc()
    ext = [float(e) for e in domain_extent]
    cells = [int(c) for c in mesh_cells]
    if len(ext) != 3 or len(cells) != 3:
        raise ValueError("domain_extent and mesh_cells need 3 entries each")
    for a in range(3):
        m.extent[a] = ext[a]
        m.cells[a] = cells[a]
    return m, cells


def bin_particles_cic(particles, charges, domain_extent, mesh_cells, stream=None):
    import torch
    lib = _lib.load()
    mesh, cells = _mesh(domain_extent, mesh_cells)
    on_device = isinstance(particles, torch.Tensor) and particles.is_cuda
    if on_device:
        dev = particles.device
        r = particles.to(torch.float64).reshape(-1, 3).contiguous()
        q = torch.as_tensor(charges, dtype=torch.float64, device=dev).reshape(-1).contiguous()
    else:
        if not torch.cuda.is_available():
            raise RuntimeError("bin_particles_cic needs a CUDA device (there is no CPU fallback)")
        dev = torch.device("cuda", torch.cuda.current_device())
        r = torch.from_numpy(np.ascontiguousarray(particles, dtype=np.float64).reshape(-1, 3)).to(dev)
        q = torch.from_numpy(np.ascontiguousarray(charges, dtype=np.float64).reshape(-1)).to(dev)
    if r.shape[0] != q.shape[0]:
        raise ValueError("particles and charges must have the same length")
    rho = torch.empty(cells[0] * cells[1] * cells[2], dtype=torch.float64, device=dev)
    with torch.cuda.device(dev):
        _lib.check(lib.ppt_deposit_cic(r.shape[0], r.data_ptr() if r.numel() else None,
                                       q.data_ptr() if q.numel() else None, mesh, rho.data_ptr(),
                                       _lib.stream_handle(stream)))
    return rho if on_device else rho.cpu().numpy()
