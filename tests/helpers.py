"""Shared test helpers: error metrics and building equivalent field objects
for the GPU package and the CPU oracle from one workload."""
import numpy as np

from oracle import pusher_oracle as orc


def rel_pos_err(r, r_ref, half_width):
    """Per-particle |r - r_ref| / max(|r_ref|, half_width) (max over rows)."""
    r = np.asarray(r).reshape(-1, 3)
    r_ref = np.asarray(r_ref).reshape(-1, 3)
    num = np.linalg.norm(r - r_ref, axis=1)
    den = np.maximum(np.linalg.norm(r_ref, axis=1), half_width)
    return float(np.max(num / den)) if num.size else 0.0


def rel_vel_err(v, v_ref):
    v = np.asarray(v).reshape(-1, 3)
    v_ref = np.asarray(v_ref).reshape(-1, 3)
    num = np.linalg.norm(v - v_ref, axis=1)
    den = np.maximum(np.linalg.norm(v_ref, axis=1), 1e-300)
    return float(np.max(num / den)) if num.size else 0.0


def gpu_fields(wl):
    from pypatools_b200 import Field
    g = {"x": wl.grid[0], "y": wl.grid[1], "z": wl.grid[2]}
    e = Field.zero(3) if wl.e_values is None else Field.from_arrays(g, wl.e_values)
    b = Field.zero(3) if wl.b_values is None else Field.from_arrays(g, wl.b_values)
    return e, b


def oracle_fields(wl):
    e = orc.ZeroField() if wl.e_values is None else orc.MapField(wl.grid, wl.e_values)
    b = orc.ZeroField() if wl.b_values is None else orc.MapField(wl.grid, wl.b_values)
    return e, b


def half_width(wl):
    return 0.5 * float(wl.grid[0][-1] - wl.grid[0][0])
