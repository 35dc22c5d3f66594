"""Benchmark: particle-steps/s of the fused push + trilinear gather.

Workload (default): RF-gap protons -- 1e7 protons, 1 MeV +-1 %, 256^3 float32
E+B map over a 20 cm cube (Ez = 5 MV/m gap profile, Bz = 0.2 T), E modulated
by cos(2 pi 100 MHz t + phi_i), dt = 1e-11 s, 2e4 steps, snapshots every 500
steps.  One bench "step" is one whole tracking job of that workload (all
2e4 pushes of all particles, 41 snapshot writes), restarted from the same
initial state, with inputs resident in HBM.  ``value`` is the mixed-precision
form; the float64 plain form is timed the same way and reported beside it
with the ratio and the mixed form's error against it (the float64 GPU path
matches the reference to 1e-10).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun with N > 1 every rank runs an independent replica of the job
(particles are independent: no data-path collective); value = total
particle-steps of all ranks / max over ranks of the device time.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["rf_gap", "pusher_sweep", "sector_ring", "rf_gap_phases"],
                    default="rf_gap",
                    help="rf_gap: the headline line (default); pusher_sweep: 1e6 electrons, Boris / vay_rel "
                         "/ rk4_rel / boris_rel / vay in both forms; sector_ring: 1e8 protons on a 512^3 Bz map; "
                         "rf_gap_phases: the RF-gap job's map crossing and field-free drift on their own "
                         "(--n particles, --nsteps steps per drift launch)")
    ap.add_argument("--n", type=int, default=None, help="particles (default: the workload's)")
    ap.add_argument("--nsteps", type=int, default=None, help="steps per job (default: the workload's)")
    ap.add_argument("--e2e-steps", type=int, default=3,
                    help="timed track_batch calls of the e2e figure (their mean)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--long-chunk", type=int, default=1000,
                    help="steps per launch once the bunch has left the map (no sorts then)")
    ap.add_argument("--free-chunk", type=int, default=None,
                    help="steps per launch once the bunch is back in row order and met no map "
                         "(default 10 x --long-chunk)")
    ap.add_argument("--sort-every", type=int, default=None,
                    help="cell re-sort interval in steps while the map is populated (also the launch length "
                         "then); 0 = never; default 300 for rf_gap (best of a 50-1000 sweep), 100 otherwise "
                         "(the sector-ring configuration's interval)")
    ap.add_argument("--serve-jobs", type=int, default=2000,
                    help="jobs of the serving stream per form (default: the whole 2000-job stream); 0 skips it")
    ap.add_argument("--no-sweep", action="store_true",
                    help="skip the electron pusher sweep object of the default line")
    ap.add_argument("--no-sector-ring", action="store_true",
                    help="skip the large-scale sector-ring object of the default line")
    ap.add_argument("--no-legs", action="store_true",
                    help="skip the deposition, space-charge, electrode and loader objects")
    args = ap.parse_args()
    defaults = {"rf_gap": (10_000_000, 20_000), "pusher_sweep": (1_000_000, 10_000),
                "sector_ring": (100_000_000, 50_000), "rf_gap_phases": (1_000_000, 1000)}[args.workload]
    args.n = args.n or defaults[0]
    args.nsteps = args.nsteps or defaults[1]
    if args.sort_every is None:
        args.sort_every = 300 if args.workload == "rf_gap" else 100
    return args


# DRAM bytes per particle per launch of the mixed track kernel, from the ncu
# captures of `bench.py --workload rf_gap_phases` at 1e6 protons: a 100-step
# launch inside the map (the 60 B state read and written; the map's occupied
# cells stay in L1/L2) and a 1000-step field-free launch (the state and two
# 48 B snapshot rows).
MIXED_DRAM_BYTES_PER_PARTICLE_LAUNCH = {"map": 131.0, "drift": 167.4}
# Warp-instructions issued per warp-step (32 particle-steps) by the mixed
# Boris kernel on the RF-gap layout, in the map and in field-free drift
# (ncu smsp__inst_executed of those launches / warps / steps).
WARP_INST_PER_WARP_STEP = {"map": 213.7, "drift": 1.42}
MIXED_STATE_BYTES = 60


def _timed_track(tr, r0, v0, nsteps, sort_every, phase=None):
    """Load and run one whole track; device milliseconds."""
    import torch
    tr.step = 0
    tr.order = None
    if phase is not None:
        tr.rf_phase.copy_(phase)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record()
    tr.load(r0, v0)
    tr.run(nsteps, sort_every or nsteps, sort_every=sort_every)
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b)


def _rel_err(r, r64, floor):
    """Per-particle worst |r - r64| / max(|r64|, floor) over the records."""
    import torch
    num = torch.linalg.vector_norm(r - r64, dim=-1)
    den = torch.clamp(torch.linalg.vector_norm(r64, dim=-1), min=floor)
    rel = (num / den).amax(dim=0)
    srt = torch.sort(rel.flatten()).values
    q = lambda p: float(srt[min(srt.numel() - 1, int(p * srt.numel()))])
    return {"p50": q(0.5), "p99": q(0.99), "max": float(srt[-1]), "over_1e-6": int((srt > 1e-6).sum())}


def run_pusher_sweep(dev, n=1_000_000, nsteps=10_000, sort_every=100):
    """1e6 electrons (10 keV-10 MeV, isotropic) in a radial 1 MV/m E and a
    0.5 T cos(pi z / 0.2 m) solenoid B on a 129^3 map, dt = 1e-12 s, 1e4
    steps: the reference's Boris, vay_rel and rk4_rel and the added
    relativistic Boris and Vay (2008), each in both forms, with the mixed
    form's error against the float64 form (which matches the oracle to 1e-10)."""
    import torch
    from pypatools_b200 import workloads, Field
    from pypatools_b200.device_fields import DeviceFields
    from pypatools_b200.pusher import DeviceTracker
    wl = workloads.radial_e_solenoid_electrons(n=n, nsteps=nsteps)
    g = {"x": wl.grid[0], "y": wl.grid[1], "z": wl.grid[2]}
    ef, bf = Field.from_arrays(g, wl.e_values), Field.from_arrays(g, wl.b_values)
    r0, v0 = torch.from_numpy(wl.r0).to(dev), torch.from_numpy(wl.v0).to(dev)
    out = {}
    for alg in ("boris", "vay_rel", "rk4_rel", "boris_rel", "vay"):
        res, hist = {}, {}
        for form in ("fp64", "mixed"):
            df = DeviceFields(ef, bf, form, dev)
            tr = DeviceTracker(alg, wl.species.q_over_m, df, wl.n, wl.nsteps, wl.dt, wl.rec_every, form,
                               device=dev)
            warm = DeviceTracker(alg, wl.species.q_over_m, df, min(wl.n, 4096), 50, wl.dt, 50, form, device=dev)
            _timed_track(warm, r0[:warm.n], v0[:warm.n], 50, sort_every)
            ms = _timed_track(tr, r0, v0, wl.nsteps, sort_every)
            res[form] = {"particle_steps_per_s": wl.n * wl.nsteps / (ms / 1e3), "ms": ms}
            hist[form] = tr.r_hist
            del tr, warm
        res["mixed_over_fp64"] = res["fp64"]["ms"] / res["mixed"]["ms"]
        res["error_vs_fp64"] = _rel_err(hist["mixed"], hist["fp64"], 0.1)
        out[alg] = res
        del hist
        torch.cuda.empty_cache()
    cpu = _sweep_cpu_baseline(wl)
    for alg, rate in cpu["particle_steps_per_s"].items():
        out[alg]["cpu_port_particle_steps_per_s"] = rate
    return {"metric": "particle-steps/s per pusher, mixed vs float64, and the mixed form's error",
            "workload": "radial_e_solenoid_electrons", "particles": wl.n, "steps": wl.nsteps, "dt": wl.dt,
            "map": "129^3 over a 20 cm cube: E radial 1 MV/m at r = 0.1 m, Bz = 0.5 T cos(pi z / 0.2 m)",
            "error_metric": "per particle max over the start and end records of |r - r64| / max(|r64|, 0.1 m)",
            "sort_every": sort_every, "cpu_baseline": cpu["describe"], "results": out}


def _sweep_cpu_baseline(wl, n_sample=100_000, steps=20):
    """The C restatement of the reference's three pushers (boris, vay_rel,
    rk4_rel) on the first n_sample electrons of the sweep, all host threads:
    the per-pusher CPU baseline."""
    import time
    from oracle import cpu_baseline
    omap, keep = cpu_baseline.make_map(wl.grid, wl.e_values, wl.b_values)
    r0, v0 = wl.r0[:n_sample], wl.v0[:n_sample]
    rates = {}
    for alg in ("boris", "vay_rel", "rk4_rel"):
        cpu_baseline.track(alg, r0[:64], v0[:64], omap, 2, wl.dt, wl.species.q_over_m, rec=2)
        t = time.perf_counter()
        cpu_baseline.track(alg, r0, v0, omap, steps, wl.dt, wl.species.q_over_m, rec=steps)
        rates[alg] = n_sample * steps / (time.perf_counter() - t)
    del keep
    return {"particle_steps_per_s": rates,
            "describe": {"kind": "port", "cores": int(cpu_baseline.load().oracle_threads()),
                         "sample": f"{n_sample} electrons x {steps} steps per pusher (the C restatement)"}}


def run_phases(dev, n=1_000_000, nsteps=1000, sort_every=0, launches=4):
    """The two phases of the RF-gap job, each on its own, for both forms:
    the bunch as generated, every particle inside the map (100-step
    launches after one cell sort, as the job's schedule runs the crossing),
    and the same bunch moved 35 cm past the map, moving away (launches of
    ``nsteps`` field-free steps, snapshots every 500 as in the job).  Device
    time per launch (CUDA events); the last of ``launches`` launches is the
    figure (the first ones warm up).  Snapshot rows are written as in the
    job, so the drift figure is that of the job's 1000-step launches."""
    import numpy as np
    import torch
    from pypatools_b200 import workloads, Field
    from pypatools_b200.device_fields import DeviceFields
    from pypatools_b200.pusher import DeviceTracker
    phases = {"map": 100, "drift": nsteps}
    wl = workloads.rf_gap_protons(n=n, nsteps=launches * max(phases.values()), rec_every=500)
    g = {"x": wl.grid[0], "y": wl.grid[1], "z": wl.grid[2]}
    ef, bf = Field.from_arrays(g, wl.e_values), Field.from_arrays(g, wl.b_values)
    out = {}
    for form in ("mixed", "fp64"):
        df = DeviceFields(ef, bf, form, dev)
        for phase, k in phases.items():
            r0 = wl.r0.copy()
            if phase == "drift":
                r0[:, 2] += 0.35
            tr = DeviceTracker("boris", wl.species.q_over_m, df, n, launches * k, wl.dt, 500, form,
                               rf_omega=2 * np.pi * wl.rf_frequency, rf_phase=torch.from_numpy(wl.rf_phase),
                               device=dev)
            tr.load(torch.from_numpy(r0).to(dev), torch.from_numpy(wl.v0).to(dev))
            if phase == "map":
                tr.sort()
            ms = []
            for _ in range(launches):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record()
                tr.advance(k)
                b.record()
                torch.cuda.synchronize()
                ms.append(a.elapsed_time(b))
            out.setdefault(form, {})[phase] = {"steps_per_launch": k, "ms_per_launch": ms[-1],
                                               "particle_steps_per_s": n * k / (ms[-1] / 1e3), "all_ms": ms}
            del tr
        del df
        torch.cuda.empty_cache()
    for phase in phases:
        out[f"mixed_over_fp64_{phase}"] = (out["mixed"][phase]["particle_steps_per_s"] /
                                           out["fp64"][phase]["particle_steps_per_s"])
    return {"metric": "particle-steps/s per phase of the RF-gap job, mixed vs float64",
            "workload": "rf_gap_protons", "particles": n, "launches": launches,
            "phases": {"map": "the bunch as generated, inside the 256^3 map, cell-sorted once",
                       "drift": "the bunch 35 cm past the map, moving away: every step field-free"},
            "results": out}


def run_sector_ring(dev, n=100_000_000, nsteps=50_000, sort_every=100):
    """1e8 protons (5 MeV +-0.5 %) circulating in a four-sector Bz map
    (512^3 float32 over a 1 m cube, 1 T (1 + 0.1 cos 4 theta) - 0.05 T/m r),
    dt = 1e-10 s, 5e4 steps, cell re-sort every 100 steps.  Mixed form over
    the whole job; the float64 form timed on the first 1/10 of the steps at
    full size; the mixed form's error against the float64 form on a
    1e5-particle subsample over the whole job."""
    import torch
    from pypatools_b200 import workloads, Field
    from pypatools_b200.device_fields import DeviceFields
    from pypatools_b200.pusher import DeviceTracker
    wl = workloads.sector_ring_protons(n=n, nsteps=nsteps)
    g = {"x": wl.grid[0], "y": wl.grid[1], "z": wl.grid[2]}
    bf = Field.from_arrays(g, wl.b_values)
    r0, v0 = torch.from_numpy(wl.r0).to(dev), torch.from_numpy(wl.v0).to(dev)
    sub = min(wl.n, 100_000)
    qm = wl.species.q_over_m
    out = {}
    dfm = DeviceFields(None, bf, "mixed", dev)
    warm = DeviceTracker("boris", qm, dfm, min(wl.n, 4096), 50, wl.dt, 50, "mixed", device=dev)
    _timed_track(warm, r0[:warm.n], v0[:warm.n], 50, sort_every)
    tr = DeviceTracker("boris", qm, dfm, wl.n, wl.nsteps, wl.dt, wl.rec_every, "mixed", device=dev)
    ms = _timed_track(tr, r0, v0, wl.nsteps, sort_every)
    out["mixed"] = {"particle_steps_per_s": wl.n * wl.nsteps / (ms / 1e3), "ms_job": ms}
    r_mixed_sub = tr.r_hist[:, :sub].clone()
    del tr
    torch.cuda.empty_cache()
    df64 = DeviceFields(None, bf, "fp64", dev)
    window = max(1, wl.nsteps // 10)
    tr = DeviceTracker("boris", qm, df64, wl.n, window, wl.dt, window, "fp64", device=dev)
    ms64 = _timed_track(tr, r0, v0, window, sort_every)
    out["fp64"] = {"particle_steps_per_s": wl.n * window / (ms64 / 1e3), "ms": ms64, "steps_timed": window}
    del tr
    torch.cuda.empty_cache()
    tr = DeviceTracker("boris", qm, df64, sub, wl.nsteps, wl.dt, wl.rec_every, "fp64", device=dev)
    _timed_track(tr, r0[:sub].contiguous(), v0[:sub].contiguous(), wl.nsteps, sort_every)
    out["mixed_over_fp64"] = out["mixed"]["particle_steps_per_s"] / out["fp64"]["particle_steps_per_s"]
    out["error_vs_fp64"] = _rel_err(r_mixed_sub, tr.r_hist, 0.5)
    out["error_vs_fp64"]["sample"] = f"first {sub} particles, whole job"
    # particles that leave the map (no vertical focusing in a Bz-only map)
    # fly straight on: a one-step difference in the exit makes a different line
    end = tr.r_hist[-1]
    inside = (end.abs() <= 0.5).all(dim=1)
    out["left_map_fraction"] = float(1.0 - inside.double().mean())
    if bool(inside.any()):
        e_in = _rel_err(r_mixed_sub[:, inside], tr.r_hist[:, inside], 0.5)
        out["error_vs_fp64_inside"] = e_in
    return {"metric": "particle-steps/s, mixed vs float64, and the mixed form's error (large-scale sector ring)",
            "workload": "sector_ring_protons", "particles": wl.n, "steps": wl.nsteps, "dt": wl.dt,
            "map": "512^3 float32 Bz over a 1 m cube (Bx = By = 0: the Bz-only record layout)",
            "sort_every": sort_every, "map_bytes_mixed": dfm.map_bytes,
            "error_metric": "per particle max over the start and end records of |r - r64| / max(|r64|, 0.5 m)",
            "results": out}


def run_deposit(r, dev, mesh_extent=(0.02, 0.02, 0.3), mesh_cells=(32, 32, 128), reps=5):
    """Cloud-in-cell deposition of the bunch (positions r, (n,3) CUDA float64,
    unit charges) onto a space-charge mesh around it, in the given particle order
    and sorted by mesh cell; device time per deposit (best of reps), the bytes
    it must move at HBM bandwidth, and the NumPy oracle on a 1e6 sample."""
    import torch
    from pypatools_b200 import _lib
    from oracle.deposit_oracle import bin_particles_cic as oracle_cic
    lib = _lib.load()
    n = r.shape[0]
    q = torch.full((n,), 1.602176634e-19, dtype=torch.float64, device=dev)
    mesh = _lib.MeshDesc()
    for a in range(3):
        mesh.extent[a] = mesh_extent[a]
        mesh.cells[a] = mesh_cells[a]
    nodes = mesh_cells[0] * mesh_cells[1] * mesh_cells[2]
    rho = torch.empty(nodes, dtype=torch.float64, device=dev)
    h = torch.tensor([e / c for e, c in zip(mesh_extent, mesh_cells)], dtype=torch.float64, device=dev)
    key = torch.floor((r + torch.tensor(mesh_extent, dtype=torch.float64, device=dev) / 2) / h).to(torch.int64)
    key = key.clamp(min=0)
    lin = (key[:, 0] * mesh_cells[1] + key[:, 1]) * mesh_cells[2] + key[:, 2]
    r_sorted = r[torch.argsort(lin)].contiguous()
    out = {}
    for name, rr in (("given_order", r), ("cell_sorted", r_sorted)):
        best = None
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            _lib.check(lib.ppt_deposit_cic(n, rr.data_ptr(), q.data_ptr(), mesh, rho.data_ptr(),
                                           _lib.stream_handle()))
            b.record()
            torch.cuda.synchronize()
            ms = a.elapsed_time(b)
            best = ms if best is None or ms < best else best
        out[name] = {"ms": best, "particles_per_s": n / (best / 1e3)}
    peak, peak_kind = measured_peaks()
    alg_bytes = n * 32 + 3 * nodes * 8       # positions + charges in; rho zeroed, written, divided
    ms = out["cell_sorted"]["ms"]
    out["roofline"] = {"bound": "hbm", "achieved": alg_bytes / (ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                       "frac": alg_bytes / (ms / 1e3) / 1e9 / peak, "peak_kind": f"{peak_kind} hbm_gbs"}
    sample = min(n, 1_000_000)
    rs = r[:sample].cpu().numpy()
    qs = np.full(sample, 1.602176634e-19)
    t = time.perf_counter()
    oracle_cic(rs, qs, mesh_extent, mesh_cells)
    out["cpu_oracle_particles_per_s"] = sample / (time.perf_counter() - t)
    out["mesh"] = f"{mesh_cells[0]}x{mesh_cells[1]}x{mesh_cells[2]} nodes over {mesh_extent} m"
    out["particles"] = n
    return out


def run_electrodes(dev, n=1_000_000, nsteps=1000, reps=3):
    """Electrode collision termination (float64 Boris): the quadrupole-solenoid
    bunch through an aperture plate (5 mm hole) at z = 3 cm inside a 12 mm beam
    pipe (2.4e3 triangles); device time of one 1000-step launch with and
    without the surface, and the oracle's rate on a small sample."""
    import torch
    from pypatools_b200 import ElectrodeSurface, Field, workloads
    from pypatools_b200.device_fields import DeviceFields
    from pypatools_b200.pusher import DeviceTracker
    from oracle import pusher_oracle as orc
    wl = workloads.quad_solenoid_protons(n=n, nsteps=nsteps, rec_every=nsteps)
    g = {"x": wl.grid[0], "y": wl.grid[1], "z": wl.grid[2]}
    df = DeviceFields(Field.zero(3), Field.from_arrays(g, wl.b_values), "fp64", dev)
    surf = ElectrodeSurface.aperture_plate(0.03, 0.005, 0.02, n_phi=48, n_r=3) + \
        ElectrodeSurface.tube(0.012, -0.05, 0.06, n_phi=48, n_z=22)
    r0 = torch.from_numpy(wl.r0).to(dev)
    v0 = torch.from_numpy(wl.v0).to(dev)
    out = {}
    stopped = None
    for name, sf in (("without_surface", None), ("with_surface", surf)):
        best = None
        for _ in range(reps):
            tr = DeviceTracker("boris", wl.species.q_over_m, df, n, nsteps, wl.dt, nsteps, "fp64", device=dev,
                               surface=sf)
            tr.load(r0, v0)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            tr.advance(nsteps)
            b.record()
            torch.cuda.synchronize()
            ms = a.elapsed_time(b)
            best = ms if best is None or ms < best else best
            if sf is not None:
                stopped = int(n - tr.active.sum().item())
            del tr
        out[name] = {"ms": best, "particle_steps_per_s": n * nsteps / (best / 1e3)}
    out["overhead"] = out["with_surface"]["ms"] / out["without_surface"]["ms"]
    out["stopped_fraction"] = stopped / n
    out["triangles"] = int(surf.triangles.shape[0])
    out["cells"] = surf.info(dev)["cells"]
    sample, steps = 500, 40
    e, bo = orc.ZeroField(), orc.MapField(wl.grid, wl.b_values)
    t = time.perf_counter()
    orc.track_batch("boris", wl.species.q_over_m, wl.r0[:sample], wl.v0[:sample], e, bo, steps, wl.dt, steps,
                    surface=(surf.vertices, surf.triangles))
    out["cpu_oracle_particle_steps_per_s"] = sample * steps / (time.perf_counter() - t)
    out["workload"] = f"quad_solenoid_protons n={n}, {nsteps} steps, float64 boris, one launch"
    return out


def run_loaders(dev, nr=200, nt=360, res=1000, reps=3):
    """The cylindrical-map loaders' resampling (AIMA AGORA / OPAL midplane):
    one z slice of (B_r, B_theta, B_z) on a 200 x 360 polar grid onto a
    1000 x 1000 Cartesian grid through the public helper (host arrays in and
    out, copies included), against the oracle's RegularGridInterpolator
    restatement of the reference's CPU resampling on the same slice."""
    import torch
    from pypatools_b200 import loaders
    from oracle import loader_oracle
    rng = np.random.default_rng(9)
    r = np.linspace(0.0, 100.0, nr, endpoint=False)
    th = np.linspace(0.0, 360.0, nt, endpoint=False)
    comps = [rng.normal(0, 1, (nr, nt)) for _ in range(3)]
    x = np.linspace(-r[-1], r[-1], res)
    loaders.polar_to_cartesian(r, th, comps, x, x)      # warm-up
    best = None
    for _ in range(reps):
        torch.cuda.synchronize()
        t = time.perf_counter()
        got = loaders.polar_to_cartesian(r, th, comps, x, x)
        dt = time.perf_counter() - t
        best = dt if best is None or dt < best else best
    t = time.perf_counter()
    ref = loader_oracle.polar_to_cartesian(r, th, comps, x, x)
    cpu = time.perf_counter() - t
    err = max(float(np.max(np.abs(g - o))) for g, o in zip(got, ref))
    return {"workload": f"polar {nr}x{nt} -> cartesian {res}x{res}, 3 components, one slice",
            "gpu_ms": best * 1e3, "nodes_per_s": res * res / best, "cpu_oracle_ms": cpu * 1e3,
            "cpu_oracle_nodes_per_s": res * res / cpu, "max_abs_diff_vs_oracle": err}


def run_space_charge(r, dev, extent=(0.02, 0.02, 0.3), cells=(64, 64, 128), reps=3):
    """The space-charge step of the reference's solver (poisson_amg.py:616-797)
    for the bunch (positions r, unit charges x 1e4): deposition, Poisson solve
    to its default 1e-6 relative residual and E = -grad phi on the 64 x 64 x 128
    mesh, device time; the oracle's CPU solve (scipy conjugate gradients to the
    same residual) of the same right-hand side for comparison."""
    import torch
    from pypatools_b200.space_charge import PoissonSolverConfig, SpaceChargeSolver
    from oracle import space_charge_oracle as sco
    n = r.shape[0]
    q = torch.full((n,), 1.602176634e-19 * 1e4, dtype=torch.float64, device=dev)
    solver = SpaceChargeSolver(PoissonSolverConfig(extent, cells, solver_tol=1e-6), device=dev)
    solver.solve_device(r, q)                       # warm-up
    best = None
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        solver.solve_device(r, q)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        best = ms if best is None or ms < best else best
    rhs = solver._rho.cpu().numpy().ravel()
    t = time.perf_counter()
    x, _ = sco.cg(sco.assemble_matrix(extent, cells), rhs, rtol=1e-6, atol=0.0, maxiter=20 * max(cells))
    cpu = time.perf_counter() - t
    phi = solver.phi.cpu().numpy().ravel()
    out = {"mesh": f"{cells[0]}x{cells[1]}x{cells[2]} cells over {extent} m", "particles": n,
           "ms": best, "cg_iterations": solver.last_iterations, "rel_residual": solver.last_residual,
           "cpu_oracle_solve_ms": cpu * 1e3,
           "max_rel_diff_vs_cpu_solve": float(np.abs(phi - x).max() / max(np.abs(x).max(), 1e-300))}
    # with conductors: a thick beam pipe (wall 8-9.5 mm) and a 2 mm thick
    # aperture plate (3 mm hole) at z = 5 cm, both closed solids
    from pypatools_b200 import ElectrodeSurface
    surf = ElectrodeSurface.annular_cylinder(0.008, 0.0095, -0.15, 0.15, n_phi=64, n_z=60) + \
        ElectrodeSurface.annular_cylinder(0.003, 0.008, 0.049, 0.051, n_phi=64, n_z=1, n_r=4)
    torch.cuda.synchronize()
    t = time.perf_counter()
    solver_c = SpaceChargeSolver(PoissonSolverConfig(extent, cells, solver_tol=1e-6), electrode_assembly=surf,
                                 device=dev)
    setup = time.perf_counter() - t
    solver_c.solve_device(r, q)
    best = None
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        solver_c.solve_device(r, q)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        best = ms if best is None or ms < best else best
    kinds = np.bincount(solver_c.cell_type, minlength=3)
    out["conductors"] = {"electrodes": f"thick pipe + aperture plate, {surf.triangles.shape[0]} triangles",
                         "setup_s": setup, "ms": best, "bicgstab_iterations": solver_c.last_iterations,
                         "rel_residual": solver_c.last_residual,
                         "cells": {"interior": int(kinds[0]), "boundary": int(kinds[1]), "conductor": int(kinds[2])}}
    return out


def run_serving(n_jobs, device, rate=50.0):
    """The serving stream (Poisson arrivals at 50 jobs/s, 1e3-1e6 protons,
    Boris / Vay / RK4, 1000-10000 steps, 4 resident float32 maps 64^3-256^3,
    120 GB admission budget) in real time, mixed then float64."""
    import torch
    from pypatools_b200 import Field, IonSpecies, workloads
    from pypatools_b200.serving import TrackingJob, TrackingServer

    ion = IonSpecies("proton")
    fields = []
    for grid, e, b in workloads.serving_maps():
        g = {"x": grid[0], "y": grid[1], "z": grid[2]}
        fields.append((Field.zero(3) if e is None else Field.from_arrays(g, e), Field.from_arrays(g, b)))
    specs = workloads.serving_stream(n_jobs=n_jobs, rate=rate)
    warm_stream = workloads.serving_stream(n_jobs=min(n_jobs, 100), rate=rate, seed=41)
    # one small job per (map, pusher) class: the stream's maps are resident
    # before it starts, and every class kernel has run once
    bunch = workloads.quad_solenoid_protons(n=256, nsteps=1, seed=40, nodes=2)
    algs = ("boris", "vay_rel", "rk4_rel")
    out = {}
    for form in ("mixed", "fp64"):
        def jobs_of(sp):
            return [TrackingJob(s.job_id, ion.q_over_m, s.algorithm, s.r0, s.v0, *fields[s.map_index], s.nsteps,
                                1e-11, precision=form, arrival=s.arrival) for s in sp]
        warm = [TrackingJob(i, ion.q_over_m, algs[i % 3], bunch.r0, bunch.v0, *fields[i // 3], 1200, 1e-11,
                            precision=form, arrival=0.0) for i in range(3 * len(fields))]
        server = TrackingServer(device=device, budget_bytes=120e9, chunk=500)
        server.run(warm, realtime=False)
        # and a short stream of another seed, so the allocators' pools (device
        # and pinned host blocks) hold the stream's sizes, as in a server that
        # has been running
        server.run(jobs_of(warm_stream), realtime=False)
        rep = server.run(jobs_of(specs), realtime=True)
        span = specs[-1].arrival
        rep["offered_particle_steps_per_s"] = sum(s.n * s.nsteps for s in specs) / span if span > 0 else None
        out[form] = rep
        torch.cuda.synchronize()
    return {"stream": f"{n_jobs} jobs, Poisson {rate}/s, 1e3-1e6 protons, boris/vay_rel/rk4_rel, "
                      "1000-10000 steps, maps 64^3/128^3/192^3/256^3 float32, 120 GB budget, chunk 500",
            "mixed": out["mixed"], "fp64": out["fp64"]}


# ---------------------------------------------------------------------------
# clocks sampler (nvidia-smi during the timed region)
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
def measured_peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def d2h_bandwidth(dev, gib=2, reps=3):
    """Device -> pinned host copy rate (GB/s), best of ``reps`` copies of
    ``gib`` GiB: the link the e2e histories cross."""
    import torch
    n = gib << 30
    d = torch.empty(n, dtype=torch.uint8, device=dev)
    h = torch.empty(n, dtype=torch.uint8, pin_memory=True)
    best = None
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        h.copy_(d, non_blocking=True)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        best = ms if best is None or ms < best else best
    del d, h
    return n / (best / 1e3) / 1e9


def max_over_ranks(value, world, device):
    """The slowest rank's device time: replicas report the job as done when
    the last one is (the only collective on the bench path)."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


HEADLINE_METRIC = "particle-steps/s, mixed-precision fused Boris + trilinear E/B (RF gap, 1e7 protons, 256^3 map)"


def headline_config(n, nsteps, world):
    """The ``config`` object of the RF-gap line, the same for both arms."""
    from pypatools_b200 import workloads
    wl = workloads.rf_gap_protons(n=1, nsteps=nsteps)
    nodes = wl.grid[0].shape[0]
    stored = [v for vals in (wl.e_values, wl.b_values) for v in vals.values() if np.any(v)]
    map_mb = nodes ** 3 * len(stored) * 4 / 1e6            # the {Ez, Bz} record layout: 2 x 4 B per node
    n_rec = nsteps // wl.rec_every + 1
    return {"workload": "rf_gap_protons", "particles_per_gpu": n, "steps_per_job": nsteps, "dt": wl.dt,
            "map": f"{nodes}^3 float32 over a 20 cm cube, stored as {{Ez, Bz}} records ({map_mb:.0f} MB)",
            "rf_hz": wl.rf_frequency, "snapshot_every": wl.rec_every, "algorithm": "boris", "precision": "mixed",
            "parallelism": f"replicas x{world}",
            "l2": (f"inputs larger than L2 (map {map_mb:.0f} MB, mixed state {n * 60 / 1e6:.0f} MB, "
                   f"snapshots {2 * n_rec * n * 24 / 1e9:.1f} GB)")}


def run_reference_arm(args, rank, world):
    """The reference's CPU path (the C port of it: the reference is Python
    and its source does not travel) on the host cores, rank 0 only, with
    the GPU arm's metric and config."""
    if rank != 0:
        return
    from oracle import cpu_baseline
    res = cpu_baseline.run_reference_arm(HEADLINE_METRIC, headline_config(args.n, args.nsteps, world),
                                         args.steps, args.warmup)
    print(json.dumps(res), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return

    import torch
    import torch.distributed as dist
    from pypatools_b200 import workloads, PusherGPU, Field, RFModulation
    from pypatools_b200.device_fields import DeviceFields
    from pypatools_b200.pusher import DeviceTracker

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if args.workload != "rf_gap":
        if rank == 0:
            fn = {"pusher_sweep": run_pusher_sweep, "sector_ring": run_sector_ring,
                  "rf_gap_phases": run_phases}[args.workload]
            print(json.dumps(fn(dev, args.n, args.nsteps, args.sort_every)), flush=True)
        return
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    wl = workloads.rf_gap_protons(n=args.n, nsteps=args.nsteps)
    g = {"x": wl.grid[0], "y": wl.grid[1], "z": wl.grid[2]}
    efield = Field.from_arrays(g, wl.e_values)
    bfield = Field.from_arrays(g, wl.b_values)
    omega = 2 * np.pi * wl.rf_frequency
    d_r0 = torch.from_numpy(wl.r0).to(dev)
    d_v0 = torch.from_numpy(wl.v0).to(dev)
    d_phase = torch.from_numpy(wl.rf_phase).to(dev)
    chunk = min(wl.rec_every, args.sort_every) if args.sort_every > 0 else wl.rec_every
    n = wl.n

    def run_form(precision):
        df = DeviceFields(efield, bfield, precision, dev)
        tr = DeviceTracker("boris", wl.species.q_over_m, df, n, wl.nsteps, wl.dt, wl.rec_every, precision,
                           rf_omega=omega, rf_phase=d_phase, record=True, counters=True, device=dev)
        stream = torch.cuda.current_stream()
        launch_ev = []

        def job(time_launches):
            tr.step = 0
            tr.order = None
            tr.rf_phase.copy_(d_phase)
            tr.load(d_r0, d_v0)
            tr.run(wl.nsteps, chunk, sort_every=args.sort_every, long_chunk=args.long_chunk,
                   free_chunk=args.free_chunk, launch_events=launch_ev if time_launches else None)

        for _ in range(args.warmup):
            job(False)
        torch.cuda.synchronize()
        tr.counters.zero_()
        launches0 = tr.launches
        barrier()
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(args.steps):
            job(True)
        t1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ms = max_over_ranks(t0.elapsed_time(t1), world, dev)
        cnt = tr.counter_values()
        launch_ms = [a.elapsed_time(b) for a, b, _, _ in launch_ev]
        launch_step0 = [s0 for _, _, s0, _ in launch_ev]
        out = {"ms_total": ms, "ms_per_job": ms / args.steps, "launch_ms": launch_ms, "launch_step0": launch_step0,
               "counters": cnt, "launches": tr.launches - launches0, "map_bytes": df.map_bytes,
               "n_comp": df.n_components}
        return tr, df, out

    sampler = ClockSampler(local)
    sampler.start()
    results = {}
    r_fp64 = None
    if not args.no_fp64:
        tr64, df64, results["fp64"] = run_form("fp64")
        r_fp64 = tr64.r_hist
        v_fp64 = tr64.v_hist
        del tr64, df64
    trm, dfm, results["mixed"] = run_form("mixed")
    clocks = sampler.stop()

    # mixed-form error against the float64 form (which matches the oracle to 1e-10)
    err = None
    if r_fp64 is not None:
        half = 0.5 * float(wl.grid[0][-1] - wl.grid[0][0])
        num = torch.linalg.vector_norm(trm.r_hist - r_fp64, dim=2)
        den = torch.clamp(torch.linalg.vector_norm(r_fp64, dim=2), min=half)
        rel = (num / den).amax(dim=0)          # per particle, worst record
        vrel = (torch.linalg.vector_norm(trm.v_hist - v_fp64, dim=2) /
                torch.linalg.vector_norm(v_fp64, dim=2)).amax(dim=0)
        srt = torch.sort(rel).values

        def q(p):
            return float(srt[min(srt.numel() - 1, int(p * srt.numel()))])

        err = {"max_rel_pos": float(srt[-1]), "p99_rel_pos": q(0.99), "p99.99_rel_pos": q(0.9999),
               "particles_over_1e-6": int((rel > 1e-6).sum()), "max_rel_vel": float(vrel.max()),
               "metric": "per particle max over the 41 snapshots of |r - r64| / max(|r64|, 0.1 m)",
               "against": "float64 GPU form (pinned to the oracle at 1e-10)"}
        del r_fp64, v_fp64

    # time per phase of the job from the per-launch events: the bunch crosses
    # the map during the first steps (each proton exits after 225-1225 steps,
    # the in-map steps are 3.6 % of the job); the rest is field-free drift
    in_map_steps = 1300

    def phase_ms(res):
        first = [ms for ms, s0 in zip(res["launch_ms"], res["launch_step0"]) if s0 < in_map_steps]
        return sum(first) / args.steps, (sum(res["launch_ms"]) - sum(first)) / args.steps

    phases = {"split_at_step": in_map_steps}
    for form, res in results.items():
        a, b = phase_ms(res)
        phases[form] = {"ms_map_crossing": a, "ms_drift": b}
    if "fp64" in results:
        phases["mixed_over_fp64_map_crossing"] = phases["fp64"]["ms_map_crossing"] / phases["mixed"]["ms_map_crossing"]
        phases["mixed_over_fp64_drift"] = phases["fp64"]["ms_drift"] / phases["mixed"]["ms_drift"]

    total_ps = n * wl.nsteps * args.steps * world
    m = results["mixed"]
    value = total_ps / (m["ms_total"] / 1e3)

    # Roofline of the dominant kernel (the mixed track kernel), in the terms
    # this path's measurement plan defines: algorithmic bytes = in-map
    # gathers x 8 corners x stored components x 4 B + state in/out per
    # launch + snapshot rows written, against the measured HBM copy
    # bandwidth.  The gathers of a cell-sorted bunch are served from L1, so
    # that fraction is a basis, not the kernel's limit: the limit is
    # instruction issue (the "limiter" object below).
    peak, peak_kind = measured_peaks()
    hits = m["counters"]["map_hits"]
    psteps = m["counters"]["particle_steps"]
    n_launch = len(m["launch_ms"])
    gather_b = hits * 8 * m["n_comp"] * 4
    state_b = n_launch * n * 2 * MIXED_STATE_BYTES
    snap_b = args.steps * (wl.nsteps // wl.rec_every + 1) * n * 48
    alg_bytes_per_launch = (gather_b + state_b + snap_b) / max(n_launch, 1)
    kernel_s = float(np.sum(m["launch_ms"])) / 1e3
    avg_launch_s = kernel_s / max(n_launch, 1)
    n_map_launch = sum(1 for s0 in m["launch_step0"] if s0 < in_map_steps)
    traffic_per_launch = n * (n_map_launch * MIXED_DRAM_BYTES_PER_PARTICLE_LAUNCH["map"] +
                              (n_launch - n_map_launch) * MIXED_DRAM_BYTES_PER_PARTICLE_LAUNCH["drift"]) / max(n_launch, 1)
    achieved = alg_bytes_per_launch / avg_launch_s / 1e9
    clk_hz = (clocks.get("sm_mhz") or 1965.0) * 1e6
    n_sm = torch.cuda.get_device_properties(dev).multi_processor_count
    # warp-instructions issued per warp-step in the map and in field-free
    # drift, from the ncu instruction counts of the kernel as built
    # (profiles/track_mixed_kernel_rf_gap_1e6_*.txt)
    inst = (hits * WARP_INST_PER_WARP_STEP["map"] + (psteps - hits) * WARP_INST_PER_WARP_STEP["drift"]) / 32.0
    issue_peak = n_sm * 4 * clk_hz                  # one warp-instruction per scheduler per clock
    l1_peak = n_sm * 128 * clk_hz / 1e9             # 128 B per SM per clock
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "basis": "algorithmic bytes (in-map corner gathers of the stored components + state + snapshot "
                         "rows) at the measured HBM copy bandwidth; the gathers are L1-served, so this is not "
                         "the kernel's limit (see limiter)",
                "traffic": traffic_per_launch,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of a 100-step in-map and a "
                                  "1000-step field-free launch at 1e6 protons "
                                  "(profiles/track_mixed_kernel_rf_gap_1e6_in_map.txt, *_drift.txt), scaled by "
                                  "particle count and averaged over this job's launches of each kind",
                "peak_kind": f"{peak_kind} hbm_gbs",
                "kernel": "track_mixed_kernel<BORIS,RF,Ez|Bz layout>", "avg_launch_ms": avg_launch_s * 1e3,
                "in_map_fraction": hits / max(1, psteps),
                "limiter": {"kind": "instruction issue",
                            "issue_frac": inst / (issue_peak * kernel_s),
                            "warp_inst_per_s": inst / kernel_s, "peak_warp_inst_per_s": issue_peak,
                            "warp_inst_per_warp_step": dict(WARP_INST_PER_WARP_STEP),
                            "l1_gather_gbs": gather_b / kernel_s / 1e9, "l1_peak_gbs": l1_peak,
                            "l1_frac": gather_b / kernel_s / 1e9 / l1_peak,
                            "model": f"({n_sm} SMs x 4 schedulers x median SM clock) for issue; {n_sm} SMs x "
                                     "128 B/clock for L1; instruction counts per warp-step from ncu"}}

    # e2e through the public API with host buffers (H2D of r0/v0/phase, D2H of the histories)
    e2e = None
    if not args.no_e2e:
        del trm, dfm
        torch.cuda.empty_cache()
        pusher = PusherGPU(wl.species, "boris", precision="mixed", steps_per_launch=chunk,
                           sort_every=args.sort_every)
        rf = RFModulation(wl.rf_frequency, wl.rf_phase)
        for _ in range(1):
            pusher.track_batch(wl.r0, wl.v0, efield, bfield, wl.nsteps, wl.dt, wl.rec_every, rf=rf)
        torch.cuda.synchronize()
        barrier()
        t = time.perf_counter()
        rh = vh = None
        for _ in range(args.e2e_steps):
            rh = vh = None            # a caller that is done with the previous call's results
            rh, vh, _ = pusher.track_batch(wl.r0, wl.v0, efield, bfield, wl.nsteps, wl.dt, wl.rec_every, rf=rf)
        # results are on the host when track_batch returns; the job is done
        # when the slowest replica's are
        dt_e2e = max_over_ranks(time.perf_counter() - t, world, dev)
        n_rec = wl.nsteps // wl.rec_every + 1
        # per step: r0 and v0 (n,3) float64 plus the n RF phases in; both
        # (n_rec, n, 3) float64 histories out
        d2h_bytes = 2 * n_rec * n * 24
        d2h_gbs = d2h_bandwidth(dev)
        # the bound this path can reach: the device job, then the histories at the
        # link's measured rate (the copies of early records overlap the job)
        bound = n * wl.nsteps / (m["ms_per_job"] / 1e3 + d2h_bytes / (d2h_gbs * 1e9))
        e2e = {"value": n * wl.nsteps * args.e2e_steps * world / dt_e2e, "unit": "particle-steps/s",
               "h2d_bytes_per_step": int(2 * n * 24 + n * 8),
               "d2h_bytes_per_step": int(d2h_bytes),
               "api": "PusherGPU.track_batch (numpy in, numpy histories out)", "steps": args.e2e_steps,
               "s_per_call": dt_e2e / args.e2e_steps, "d2h_gbs_measured": d2h_gbs,
               "bound_device_plus_d2h": bound, "frac_of_bound": n * wl.nsteps / (dt_e2e / args.e2e_steps) / bound}
        del rh, vh

    deposit = electrodes = loader = space_charge = sweep = ring = None
    # the single-GPU objects (legs, C2, C5, C4) belong to the one-GPU line; a
    # multi-GPU (replica) run reports the RF-gap job alone, so the GPUs it
    # holds are not kept for minutes of work that does not scale
    single = rank == 0 and world == 1
    if single and not args.no_legs:
        deposit = run_deposit(d_r0, dev)
        space_charge = run_space_charge(d_r0, dev)
        electrodes = run_electrodes(dev)
        loader = run_loaders(dev)
    del d_r0, d_v0, d_phase
    torch.cuda.empty_cache()
    if single and not args.no_sweep:
        sweep = run_pusher_sweep(dev)
        torch.cuda.empty_cache()
    if single and not args.no_sector_ring:
        ring = run_sector_ring(dev)
        torch.cuda.empty_cache()

    serving = None
    if single and args.serve_jobs > 0:
        serving = run_serving(args.serve_jobs, dev)

    cpu = None
    if rank == 0:
        from oracle import cpu_baseline
        cpu = cpu_baseline.sample(n_sample=1_000_000, steps=200)    # ~10 s of CPU work on the host
        cpu["in_map_fraction_gpu_counters"] = roofline["in_map_fraction"]

    if rank == 0:
        f64 = results.get("fp64")
        ratio = (f64["ms_total"] / m["ms_total"]) if f64 else None
        targets = {"mixed_over_fp64": ratio, "mixed_over_fp64_target": 5.0,
                   "speed_target_met": (ratio >= 5.0) if ratio is not None else None,
                   "max_rel_pos": err["max_rel_pos"] if err else None, "max_rel_pos_target": 1e-6,
                   "error_target_met": (err["max_rel_pos"] <= 1e-6) if err else None}
        line = {
            "metric": HEADLINE_METRIC,
            "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": m["ms_per_job"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 time/phase, float-float velocity)",
            "data": "synthetic (seeded pypatools_b200.workloads.rf_gap_protons)",
            "config": headline_config(n, wl.nsteps, world),
            "fp64": ({"value": total_ps / (f64["ms_total"] / 1e3), "ms_per_step": f64["ms_per_job"],
                      "launches": f64["launches"]} if f64 else None),
            "mixed_over_fp64": ratio,
            "targets": targets,
            "phases": phases,
            "error_vs_fp64": err,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": m["launches"],
            "clocks": clocks,
            "pusher_sweep": sweep,
            "sector_ring": ring,
            "serving": serving,
            "deposit": deposit,
            "electrodes": electrodes,
            "loaders": loader,
            "space_charge": space_charge,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
