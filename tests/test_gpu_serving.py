"""Serving loop: jobs of uneven size, algorithm, precision form and field map
arrive while others run, are admitted as device memory frees up, and are
advanced together (continuous batching).  Each job's result must be the same
as the same job tracked alone (the per-particle arithmetic is identical, so
the bar is bitwise equality)."""
import numpy as np
import pytest

from pypatools_b200 import PusherGPU, Field, IonSpecies, RFModulation, workloads
from pypatools_b200.serving import TrackingJob, TrackingServer

pytestmark = pytest.mark.gpu


def _map_fields(map_dtype=np.float32):
    out = []
    for grid, e, b in workloads.serving_maps(map_dtype)[:3]:   # 64^3, 128^3, 192^3
        g = {"x": grid[0], "y": grid[1], "z": grid[2]}
        out.append((Field.zero(3) if e is None else Field.from_arrays(g, e), Field.from_arrays(g, b)))
    return out


def _jobs(fields, n_jobs=10, spacing=0.002, steps_max=300):
    ion = IonSpecies("proton")
    specs = workloads.serving_stream(n_jobs=n_jobs, n_min=200, n_max=3000, steps_min=40, steps_max=steps_max,
                                     n_maps=len(fields))
    jobs = []
    for s in specs:
        e, b = fields[s.map_index]
        jobs.append(TrackingJob(s.job_id, ion.q_over_m, s.algorithm, s.r0, s.v0, e, b, s.nsteps, 1e-11,
                                rec_every=50, precision="mixed" if s.job_id % 2 else "fp64",
                                arrival=spacing * s.job_id))
    return ion, jobs


def _check_alone(ion, jobs):
    for job in jobs:
        rh, vh, _ = PusherGPU(ion, job.algorithm, precision=job.precision).track_batch(
            job.r0, job.v0, job.efield, job.bfield, job.nsteps, job.dt, job.rec_every, rf=job.rf)
        np.testing.assert_array_equal(job.r_hist, rh, err_msg=f"job {job.job_id} r")
        np.testing.assert_array_equal(job.v_hist, vh, err_msg=f"job {job.job_id} v")


def test_serving_results_same_alone_and_in_mix(cuda):
    fields = _map_fields()
    ion, jobs = _jobs(fields)
    # equal step windows (no small-bunch boost): every job runs several ticks,
    # so unchanged job sets are captured and replayed
    server = TrackingServer(chunk=32, use_graphs=True, capture_after=1, small_bunch=0)
    rep = server.run(jobs, realtime=False)
    assert rep["jobs"] == len(jobs)
    assert rep["graph_replays"] > 0 and rep["rebuilds"] >= 2
    # jobs overlapped on the device: some job was admitted before an earlier one finished
    admits = sorted((j.t_admit, j.t_done) for j in jobs)
    assert any(admits[i + 1][0] < admits[i][1] for i in range(len(admits) - 1))
    _check_alone(ion, jobs)


def test_serving_budget_queues_jobs(cuda):
    fields = _map_fields()
    ion, jobs = _jobs(fields, n_jobs=6, spacing=0.0)
    budget = 1.5 * max(j.device_bytes() for j in jobs)
    server = TrackingServer(chunk=64, use_graphs=False, budget_bytes=budget)
    rep = server.run(jobs, realtime=False)
    assert rep["jobs"] == len(jobs)
    assert server.used_bytes == 0
    _check_alone(ion, jobs)


def test_serving_realtime_stream_with_graphs(cuda):
    # jobs keep arriving while earlier ones retire: result copies run on the
    # worker thread while later ticks are captured and replayed
    fields = _map_fields()
    # up to 1500 steps: the bunches leave their maps, so field-free runs are
    # split by the 16-step ticks here and by whole-track launches alone
    ion, jobs = _jobs(fields, n_jobs=24, spacing=0.004, steps_max=1500)
    server = TrackingServer(chunk=16, use_graphs=True, capture_after=1)
    rep = server.run(jobs, realtime=True)
    assert rep["jobs"] == len(jobs)
    assert server.used_bytes == 0
    assert rep["p99_latency_s"] is not None and rep["p99_latency_s"] >= rep["p50_latency_s"] > 0
    _check_alone(ion, jobs)


def test_serving_per_job_windows(cuda):
    """Small bunches take longer step windows per tick (tick_steps): they
    finish in fewer ticks than the others and their results are still those
    of the job run alone, bit for bit."""
    fields = _map_fields()
    ion, jobs = _jobs(fields, n_jobs=8, spacing=0.0)
    # half of them with an RF-modulated E: their windows (up to 256 steps) are
    # longer than the tick's RF table (33 entries), so they form the factor
    # without it -- the same values
    rng = np.random.default_rng(9)
    for j in jobs[::2]:
        j.rf = RFModulation(1e8, rng.uniform(0.0, 2 * np.pi, j.n))
    server = TrackingServer(chunk=32, use_graphs=False, small_bunch=1 << 20, max_boost=8)
    windows = {j.job_id: server._tick_steps(j) for j in jobs}
    assert all(w > 32 for w in windows.values())
    rep = server.run(jobs, realtime=False)
    assert rep["jobs"] == len(jobs)
    longest = max(j.nsteps for j in jobs)
    assert rep["ticks"] < -(-longest // 32)          # fewer ticks than equal 32-step windows need
    _check_alone(ion, jobs)

