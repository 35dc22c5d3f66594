"""Generate the per-particle time-step fixture (dt_golden.npz) by running the reference.

The reference's batch RK4 step takes ``dt`` either as a float or as one value
per particle: an array is broadcast over the three components of each
particle's stages (``Pusher._rk4_step_batch``, src/PyPATools/pusher.py:815-816),
so ``push_batch`` and ``track_batch`` with 'rk4' / 'rk4_rel' accept an (M,)
array.  This script runs those two entry points on seeded inputs with an
array ``dt`` and stores the results.

    PYPATOOLS_REFERENCE_SRC=<checkout>/src python tests/golden/make_golden_dt.py
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
from make_golden import load_reference  # noqa: E402

REPO = HERE.parents[1]


def main():
    sys.path.insert(0, str(REPO))
    from pypatools_b200 import workloads

    pusher, field, species, particles = load_reference()
    Pusher, Field = pusher.Pusher, field.Field
    out = {}
    # quadrupole-solenoid protons (B only) and radial-E / solenoid electrons (E and B)
    wl = workloads.quad_solenoid_protons(n=96, nsteps=400, seed=21)
    wl2 = workloads.radial_e_solenoid_electrons(n=64, nsteps=800, seed=22)
    rng = np.random.default_rng(23)
    for tag, w, steps, rec in (("quad", wl, 400, 40), ("radial", wl2, 800, 100)):
        g = {"x": w.grid[0], "y": w.grid[1], "z": w.grid[2]}
        ef = Field.zero(dim=3) if w.e_values is None else Field.from_arrays(g, w.e_values)
        bf = Field.from_arrays(g, w.b_values)
        dt = w.dt * rng.uniform(0.5, 1.5, w.n)
        out[f"{tag}/r0"], out[f"{tag}/v0"], out[f"{tag}/dt"] = w.r0, w.v0, dt
        out[f"{tag}/nsteps"], out[f"{tag}/rec"] = np.int64(steps), np.int64(rec)
        for alg in ("rk4", "rk4_rel"):
            p = Pusher(w.species, alg)
            rh, vh, act = p.track_batch(w.r0, w.v0, ef, bf, steps, dt, rec)
            out[f"{tag}/{alg}/r_hist"], out[f"{tag}/{alg}/v_hist"] = rh, vh
            rn, vn = p.push_batch(w.r0, w.v0, ef, bf, dt)
            out[f"{tag}/{alg}/push_r"], out[f"{tag}/{alg}/push_v"] = rn, vn
            print(tag, alg, "done")
    dest = HERE / "dt_golden.npz"
    np.savez_compressed(dest, **out)
    print("wrote", dest, dest.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
