"""CPU restatement of the cylindrical-map resampling of the reference's
loaders (src/PyPATools/field_src/field_loaders.py:612-640 for the OPAL
midplane, :836-899 for AIMA AGORA): scipy's RegularGridInterpolator on the
(r, theta) node grid, evaluated at the Cartesian nodes' (r, theta), then the
rotation of (B_r, B_theta) into (B_x, B_y).

TEST INFRASTRUCTURE ONLY: used by tests/ and by bench.py's CPU baseline of the
loader leg, as the checker; nothing in the product imports it.
"""
import numpy as np
from scipy.interpolate import RegularGridInterpolator


def polar_to_cartesian(r_nodes, theta_nodes, comps, x, y, r_scale=1.0):
    """[B_x, B_y, B_z] on the (len(x), len(y)) Cartesian grid; ``comps`` are
    (B_r, B_theta, B_z) on the (r, theta [deg]) grid, None for zero."""
    gx, gy = np.meshgrid(x, y, indexing="ij")
    r = np.sqrt(gx ** 2 + gy ** 2) * r_scale
    th = np.rad2deg(np.arctan2(gy, gx))
    th = np.where(th < 0, th + 360.0, th)
    pts = np.column_stack([r.ravel(), th.ravel()])
    vals = []
    for c in comps:
        if c is None:
            vals.append(np.zeros(gx.shape))
            continue
        f = RegularGridInterpolator((r_nodes, theta_nodes), c, method="linear", bounds_error=False,
                                    fill_value=0.0)
        vals.append(f(pts).reshape(gx.shape))
    rad = np.deg2rad(th)
    cos, sin = np.cos(rad), np.sin(rad)
    return [vals[0] * cos - vals[1] * sin, vals[0] * sin + vals[1] * cos, vals[2]]
