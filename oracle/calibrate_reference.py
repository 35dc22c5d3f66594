"""Calibrate the CPU port against the reference's own Numba path (TEST/BENCH
INFRASTRUCTURE ONLY: runs where the reference checkout is, never on the GPU
host, and is not imported by bench.py).

The reference is Python + Numba; its checkout does not travel with this
repository, so ``bench.py --impl reference`` times the C restatement
(``ppt_oracle.c``) instead.  This script shows what that stands in for: it times
the reference's ``Pusher('boris').track_batch`` (pusher.py:894-1012, Numba
``prange`` kernels, all threads) and the C port (OpenMP, the same threads) on
the same bunch sample of the RF-gap workload, in the map and past it, with the
static fields (the reference has no RF modulation; the port runs with omega =
0 here), and prints one JSON line with both rates.

    PYPATOOLS_REFERENCE_SRC=<checkout>/src python -m oracle.calibrate_reference
"""
import json
import os
import sys
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[1]


def _reference():
    sys.path.insert(0, str(REPO / "tests" / "golden"))
    from make_golden import load_reference
    return load_reference()


def _best(fn, reps):
    best = float("inf")
    for _ in range(reps):
        t = time.perf_counter()
        fn()
        best = min(best, time.perf_counter() - t)
    return best


def main(n=20_000, steps=20, reps=3):
    sys.path.insert(0, str(REPO))
    from pypatools_b200 import workloads
    from oracle import cpu_baseline
    import numba

    pusher, field, species, _ = _reference()
    threads = os.cpu_count()
    numba.set_num_threads(threads)
    wl = workloads.rf_gap_protons(n=n, nsteps=steps)
    g = {"x": wl.grid[0], "y": wl.grid[1], "z": wl.grid[2]}
    ef = field.Field.from_arrays(g, {c: np.asarray(wl.e_values[c], dtype=np.float64) for c in "xyz"})
    bf = field.Field.from_arrays(g, {c: np.asarray(wl.b_values[c], dtype=np.float64) for c in "xyz"})

    class Ion:
        q_over_m = wl.species.q_over_m

    ref = pusher.Pusher(Ion(), "boris", use_numba=True)
    omap, keep = cpu_baseline.make_map(wl.grid, wl.e_values, wl.b_values)
    r_out = wl.r0.copy()
    r_out[:, 2] += 0.35
    res = {"sample": f"{n} protons x {steps} Boris steps, RF-gap map (256^3 Ez, Bz) with static fields",
           "threads": threads, "cpu": cpu_baseline._cpu_model()}
    ref.track_batch(wl.r0[:64], wl.v0[:64], ef, bf, 2, wl.dt, 2)            # Numba compile
    cpu_baseline.track("boris", wl.r0[:64], wl.v0[:64], omap, 2, wl.dt, wl.species.q_over_m, rec=2)
    for phase, r0 in (("in_map", wl.r0), ("drift", r_out)):
        t_ref = _best(lambda: ref.track_batch(r0, wl.v0, ef, bf, steps, wl.dt, steps), reps)
        t_port = _best(lambda: cpu_baseline.track("boris", r0, wl.v0, omap, steps, wl.dt, wl.species.q_over_m,
                                                   rec=steps), reps)
        r_ref, _, _ = ref.track_batch(r0, wl.v0, ef, bf, steps, wl.dt, steps)
        r_port, _ = cpu_baseline.track("boris", r0, wl.v0, omap, steps, wl.dt, wl.species.q_over_m, rec=steps)
        res[phase] = {"reference_numba_particle_steps_per_s": n * steps / t_ref,
                      "port_particle_steps_per_s": n * steps / t_port,
                      "port_over_reference": t_ref / t_port,
                      "max_abs_position_difference_m": float(np.max(np.abs(r_ref - r_port)))}
    del keep
    res["electron_sweep"] = electron_sweep(pusher, field, n=max(2000, n // 10), steps=steps, reps=reps)
    print(json.dumps(res))


def electron_sweep(pusher, field, n=2000, steps=20, reps=3):
    """The electron sweep's three reference pushers (boris, vay_rel,
    rk4_rel) on its bunch and 129^3 map (radial E, solenoid B), reference
    Numba against the C restatement, the same threads."""
    from pypatools_b200 import workloads
    from oracle import cpu_baseline
    wl = workloads.radial_e_solenoid_electrons(n=n, nsteps=steps)
    g = {"x": wl.grid[0], "y": wl.grid[1], "z": wl.grid[2]}
    ef = field.Field.from_arrays(g, {c: np.asarray(wl.e_values[c], dtype=np.float64) for c in "xyz"})
    bf = field.Field.from_arrays(g, {c: np.asarray(wl.b_values[c], dtype=np.float64) for c in "xyz"})
    omap, keep = cpu_baseline.make_map(wl.grid, wl.e_values, wl.b_values)

    class Ion:
        q_over_m = wl.species.q_over_m

    out = {"sample": f"{n} electrons x {steps} steps, 129^3 map (radial E, solenoid B)"}
    for alg in ("boris", "vay_rel", "rk4_rel"):
        ref = pusher.Pusher(Ion(), alg, use_numba=True)
        ref.track_batch(wl.r0[:64], wl.v0[:64], ef, bf, 2, wl.dt, 2)                 # Numba compile
        t_ref = _best(lambda: ref.track_batch(wl.r0, wl.v0, ef, bf, steps, wl.dt, steps), reps)
        t_port = _best(lambda: cpu_baseline.track(alg, wl.r0, wl.v0, omap, steps, wl.dt, wl.species.q_over_m,
                                                   rec=steps), reps)
        r_ref, _, _ = ref.track_batch(wl.r0, wl.v0, ef, bf, steps, wl.dt, steps)
        r_port, _ = cpu_baseline.track(alg, wl.r0, wl.v0, omap, steps, wl.dt, wl.species.q_over_m, rec=steps)
        out[alg] = {"reference_numba_particle_steps_per_s": n * steps / t_ref,
                    "port_particle_steps_per_s": n * steps / t_port,
                    "port_over_reference": t_ref / t_port,
                    "max_abs_position_difference_m": float(np.max(np.abs(r_ref - r_port)))}
    del keep
    return out


if __name__ == "__main__":
    main()
