"""Bunch moments on the GPU in float64 (``ppt_moments``).

Restates the statistics of the reference's ``ParticleDistribution``
(src/PyPATools/particles.py:693-719 centroid / standard deviations /
x-x' correlations, :761-788 1-rms emittances, :507-525 and :701-705 kinetic
energy mean and spread, :600-605 mean |beta gamma|) for positions and
velocities that are already on the device, e.g. a snapshot row of
``PusherGPU.track_batch(..., snapshot='device')``.
"""
import numpy as np

from . import _lib


def _as_device(a, torch, device):
    if isinstance(a, torch.Tensor):
        t = a
        if t.device.type != "cuda":
            t = t.to(device)
    else:
        t = torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=np.float64))).to(device)
    if t.dtype != torch.float64 or t.ndim != 2 or t.shape[1] != 3:
        raise ValueError("positions and velocities must be (n, 3) float64")
    return t.contiguous()


def raw_moments(r, v, mass_mev, device=None, stream=None):
    """The PPT_MOMENTS_LEN float64 values of ``ppt_moments`` (see include/ppt.h)."""
    import torch
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    lib = _lib.load()
    dr = _as_device(r, torch, dev)
    dv = _as_device(v, torch, dev)
    n = dr.shape[0]
    if dv.shape[0] != n:
        raise ValueError("positions and velocities must have the same length")
    if n == 0:
        raise ValueError("moments of an empty bunch")
    out = torch.empty(_lib.MOMENTS_LEN, dtype=torch.float64, device=dr.device)
    scratch = torch.empty(lib.ppt_moments_scratch_bytes(n), dtype=torch.uint8, device=dr.device)
    with torch.cuda.device(dr.device):
        _lib.check(lib.ppt_moments(n, dr.data_ptr(), dv.data_ptr(), float(mass_mev), out.data_ptr(),
                                   scratch.data_ptr(), _lib.stream_handle(stream)))
    return out


def unpack(raw):
    """Dict of named moments from the raw vector (host side, scalars)."""
    m = raw.cpu().numpy() if hasattr(raw, "cpu") else np.asarray(raw)
    x_std, xp_std = m[3:6], m[6:9]
    xxp, yyp, xyp, yxp = m[12:16]
    mean_p = m[16]
    e_raw = np.array([(x_std[0] * xp_std[0]) ** 2 - xxp ** 2,
                      (x_std[1] * xp_std[1]) ** 2 - yyp ** 2,
                      (x_std[0] * xp_std[1]) ** 2 - xyp ** 2,
                      (x_std[1] * xp_std[0]) ** 2 - yxp ** 2])
    with np.errstate(invalid="ignore"):
        emit = np.sqrt(e_raw)
    return {"centroid": m[0:3].copy(), "x_std": x_std.copy(), "xp_std": xp_std.copy(),
            "xp_mean": m[9:12].copy(), "xxp": xxp, "yyp": yyp, "xyp": xyp, "yxp": yxp,
            "mean_p": mean_p, "mean_momentum": m[17:20].copy(), "emittance": emit,
            "emittance_n": emit * mean_p, "ekin_mean": m[20], "ekin_std": m[21]}


def bunch_moments(r, v, mass_mev, device=None):
    """Named float64 bunch moments of positions r [m] and velocities v [m/s]."""
    return unpack(raw_moments(r, v, mass_mev, device))
