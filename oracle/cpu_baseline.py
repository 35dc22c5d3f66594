"""CPU baseline: the C restatement of the reference's tracking loop, timed on
the host cores (TEST/BENCH INFRASTRUCTURE ONLY; bench.py's cpu_baseline leg
and its --impl reference arm).

The reference itself (Python + Numba) cannot run on the benchmark host, so
the restatement in ppt_oracle.c stands in for it: same per-step structure
(per-component interpolation passes with bisection cell search, a push pass,
a position pass), OpenMP threads over particles like Numba's prange.
"""
import ctypes
import json
import os
import time

import numpy as np

from .build_oracle import build, LIB

ALG = {"leapfrog": 0, "boris": 1, "rk4": 2, "vay_rel": 4, "rk4_rel": 5}


class OracleMap(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64 * 3), ("axis", ctypes.c_void_p * 3), ("comp", ctypes.c_void_p * 6)]


_lib = None


def load():
    global _lib
    if _lib is None:
        build()
        lib = ctypes.CDLL(str(LIB))
        lib.oracle_track.restype = ctypes.c_int
        lib.oracle_track.argtypes = [ctypes.c_int, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.POINTER(OracleMap), ctypes.c_int64, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_int64, ctypes.c_double, ctypes.c_void_p, ctypes.c_double,
                                     ctypes.c_void_p, ctypes.c_void_p]
        lib.oracle_threads.restype = ctypes.c_int
        _lib = lib
    return _lib


def make_map(grid, e_values, b_values):
    """OracleMap over float64 copies of the node values (all-zero
    components passed as NULL).  Returns (struct, keep-alive list)."""
    m = OracleMap()
    keep = []
    for d in range(3):
        a = np.ascontiguousarray(grid[d], dtype=np.float64)
        keep.append(a)
        m.n[d] = a.shape[0]
        m.axis[d] = a.ctypes.data
    for f, vals in enumerate((e_values, b_values)):
        for c, key in enumerate("xyz"):
            v = None if vals is None else vals.get(key)
            if v is None or not np.any(v):
                m.comp[3 * f + c] = None
                continue
            a = np.ascontiguousarray(v, dtype=np.float64)
            keep.append(a)
            m.comp[3 * f + c] = a.ctypes.data
    return m, keep


def track(alg, r0, v0, omap, nsteps, dt, qm, rec=None, omega=0.0, phase=None, t0=0.0, record=True):
    lib = load()
    r0 = np.ascontiguousarray(r0, dtype=np.float64)
    v0 = np.ascontiguousarray(v0, dtype=np.float64)
    n = r0.shape[0]
    rec = rec or max(nsteps, 1)
    n_rec = nsteps // rec + 1
    rh = np.empty((n_rec, n, 3)) if record else None
    vh = np.empty((n_rec, n, 3)) if record else None
    ph = None if phase is None else np.ascontiguousarray(np.broadcast_to(phase, (n,)), dtype=np.float64)
    rc = lib.oracle_track(ALG[alg], n, r0.ctypes.data, v0.ctypes.data, omap, nsteps, dt, qm, rec, omega,
                          None if ph is None else ph.ctypes.data, t0,
                          None if rh is None else rh.ctypes.data, None if vh is None else vh.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"oracle_track failed ({rc})")
    return rh, vh


def _time_window(wl, omap, r0, v0, phase, steps):
    t = time.perf_counter()
    track("boris", r0, v0, omap, steps, wl.dt, wl.species.q_over_m, rec=steps,
          omega=2 * np.pi * wl.rf_frequency, phase=phase)
    return time.perf_counter() - t


# RF-gap job: 2e4 steps; every proton has left the 20 cm map within its
# first ~1300 steps (it enters at z in +-6.9 cm at 1.4e7 m/s).
RF_GAP_STEPS = 20_000


def in_map_fraction(n_sample=2000, window=1600, job_steps=RF_GAP_STEPS):
    """Share of the RF-gap job's particle-steps whose field evaluation falls
    inside the map, from the oracle's own tracks: the steps of a bunch sample
    whose start position lies in the map's node box, over the first
    ``window`` steps (the sample must have left the map by then: checked),
    divided by the job's particle-steps."""
    from pypatools_b200 import workloads
    wl = workloads.rf_gap_protons(n=n_sample, nsteps=window)
    omap, keep = make_map(wl.grid, wl.e_values, wl.b_values)
    rh, _ = track("boris", wl.r0, wl.v0, omap, window, wl.dt, wl.species.q_over_m, rec=1,
                  omega=2 * np.pi * wl.rf_frequency, phase=wl.rf_phase)
    lo = np.array([g[0] for g in wl.grid])
    hi = np.array([g[-1] for g in wl.grid])
    inside = np.all((rh >= lo) & (rh <= hi), axis=2)          # (window + 1, n)
    if inside[-1].any():
        raise RuntimeError("in_map_fraction: particles still in the map after the window")
    del keep
    return float(inside[:-1].sum()) / (n_sample * job_steps)


def blended_sample(n_sample=20_000, steps=20, fraction=None):
    """Boris on the RF-gap workload: a window of ``steps`` steps of
    ``n_sample`` particles in the map (the bunch's start) and the same window
    after the bunch has left it (the drift that makes up most of the job),
    combined by the job's in-map fraction (``in_map_fraction()`` unless
    given): seconds per ``n_sample x steps`` particle-steps of the job's mix,
    and the two phase rates."""
    from pypatools_b200 import workloads
    wl = workloads.rf_gap_protons(n=n_sample, nsteps=steps)
    omap, keep = make_map(wl.grid, wl.e_values, wl.b_values)
    load()
    f = in_map_fraction() if fraction is None else float(fraction)
    _time_window(wl, omap, wl.r0[:64], wl.v0[:64], wl.rf_phase[:64], 2)     # warm caches / threads
    t_in = _time_window(wl, omap, wl.r0, wl.v0, wl.rf_phase, steps)
    r_out = wl.r0.copy()
    r_out[:, 2] += 0.35                                                     # past the 20 cm map
    t_out = _time_window(wl, omap, r_out, wl.v0, wl.rf_phase, steps)
    del keep
    ps = n_sample * steps
    return {"seconds": f * t_in + (1.0 - f) * t_out, "particle_steps": ps, "fraction": f,
            "rate_in_map": ps / t_in, "rate_drift": ps / t_out}


def _describe(n_sample, steps, f):
    return (f"boris, float64, RF gap workload: {n_sample} particles x {steps} steps in the map and x {steps} "
            f"steps past it, combined by the job's in-map fraction {f:.4f} (from the oracle's own tracks)")


def sample(n_sample=20_000, steps=20, in_map_fraction=None):
    """The bench line's cpu_baseline object: the job-mix rate of
    ``blended_sample``."""
    b = blended_sample(n_sample, steps, in_map_fraction)
    return {"value": b["particle_steps"] / b["seconds"], "unit": "particle-steps/s",
            "cores": int(load().oracle_threads()), "kind": "port",
            "sample": _describe(n_sample, steps, b["fraction"]),
            "in_map_fraction": b["fraction"], "rate_in_map": b["rate_in_map"], "rate_drift": b["rate_drift"],
            "cpu": _cpu_model()}


def _cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_reference_arm(metric, config, steps, warmup):
    """bench.py --impl reference: the CPU port of the reference algorithm on
    all host threads.  Each bench step is a bounded sample of the RF-gap job
    with the job's phase mix (``blended_sample``); ``metric`` and ``config``
    are the GPU arm's, so the two lines describe the same workload."""
    n_sample, window = 200_000, 50     # ~0.5 s of work per bench step on 16 host threads
    f = in_map_fraction()
    for _ in range(max(1, warmup)):
        blended_sample(2000, 2, f)
    runs = [blended_sample(n_sample, window, f) for _ in range(steps)]
    total = sum(r["seconds"] for r in runs)
    value = n_sample * window * steps / total
    cores = int(load().oracle_threads())
    res = {"impl": "reference", "metric": metric,
           "value": value, "unit": "particle-steps/s", "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
           "steps": steps, "warmup": warmup, "ms_per_step": 1e3 * total / steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded pypatools_b200.workloads.rf_gap_protons)",
           "config": config,
           "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": cores, "kind": "port",
                            "sample": _describe(n_sample, window, f), "in_map_fraction": f,
                            "rate_in_map": sum(r["rate_in_map"] for r in runs) / steps,
                            "rate_drift": sum(r["rate_drift"] for r in runs) / steps, "cpu": _cpu_model()},
           "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    return res


if __name__ == "__main__":
    print(json.dumps(sample()))
