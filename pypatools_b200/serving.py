"""Continuous-batching tracking server on one GPU.

Jobs (one ``track_batch`` each: a bunch, an algorithm, a precision form, a
field map, a step count) arrive over time.  The loop

* admits waiting jobs, in arrival order, while their device memory (state +
  snapshot histories + RF phases) fits the HBM budget, and uploads them on an
  upload stream while the current tick runs;
* keeps every admitted job's particle state on the device between ticks and
  keeps field maps resident (cached by field object and form);
* advances all admitted jobs together, ``chunk`` steps per tick, through
  ``ppt_jobs_tick`` -- one persistent kernel per (form, algorithm, RF, map
  layout) class, the classes on concurrent streams, whose blocks take (job,
  128-particle block) items from a device work queue, then a step-counter
  kernel.  With ``use_graphs``, once a job set has run ``capture_after`` ticks
  unchanged, its tick is captured in a CUDA graph and replayed until the set
  changes;
* retires jobs whose done flag is set: their histories are copied to the host
  while the next tick runs; a job's latency ends when its results are on the
  host.

Jobs that arrive while others are on the GPU join at the next tick boundary
(continuous batching); each job's arithmetic is the single-job kernels' per
particle, so its result is the same alone and in the mix.
"""
import collections
import concurrent.futures
import ctypes
import time

import numpy as np

from . import _lib
from .device_fields import FieldCache
from .pusher import DeviceTracker, HostStager, _torch, host_array


class TrackingJob:
    """One tracking request: the arguments of ``Pusher.track_batch``."""

    def __init__(self, job_id, q_over_m, algorithm, r0, v0, efield, bfield, nsteps, dt, rec_every=None,
                 precision="mixed", arrival=0.0, rf=None, t0=0.0):
        self.job_id = job_id
        self.q_over_m = float(q_over_m)
        self.algorithm = algorithm
        self.precision = precision
        self.r0 = np.ascontiguousarray(r0, dtype=np.float64)
        self.v0 = np.ascontiguousarray(v0, dtype=np.float64)
        if self.r0.ndim != 2 or self.r0.shape[1] != 3 or self.v0.shape != self.r0.shape:
            raise ValueError(f"r0 and v0 must both be (M, 3), got {self.r0.shape} and {self.v0.shape}")
        if int(nsteps) < 0 or (rec_every is not None and int(rec_every) < 1):
            raise ValueError("nsteps must be >= 0 and rec_every >= 1")
        self.n = self.r0.shape[0]
        self.efield, self.bfield = efield, bfield
        self.nsteps = int(nsteps)
        self.dt = float(dt)
        self.rec_every = int(rec_every or max(self.nsteps, 1))
        self.arrival = float(arrival)
        self.rf = rf
        self.t0 = float(t0)
        self.n_rec = self.nsteps // self.rec_every + 1
        self.reset()

    def reset(self):
        """Forget the results of a previous run (the same job can be served again)."""
        self.t_admit = self.t_done = None
        self.r_hist = self.v_hist = None
        self.steps_done = 0
        self._tracker = None
        self._fields = None

    def device_bytes(self):
        state = 60 * self.n                      # mixed (12 B cells + 48 B floats); float64 48 B
        hist = 2 * self.n_rec * self.n * 24
        phase = 8 * self.n if self.rf is not None else 0
        return state + hist + phase + 4096

    @property
    def latency(self):
        return None if self.t_done is None else self.t_done - self.arrival


class TrackingServer:
    def __init__(self, device=None, budget_bytes=120e9, chunk=500, use_graphs=False, capture_after=16,
                 small_bunch=65536, max_boost=8):
        """``use_graphs``, ``capture_after``: capture a job set's tick as a
        CUDA graph once the set has run ``capture_after`` ticks unchanged.  Off
        by default: issuing a tick's ~20 launches directly costs 0.05 ms of
        host time, so a replay saves little, while a capture stalls the loop
        (0.7 ms per capture after one unchanged tick, 20-33 ms per capture of
        the larger job sets after 16): on the 2000-job serving stream, whose
        job set changes every 4 ticks on average, capturing after one unchanged
        tick raised p99 latency from 0.41 to 0.64 s.

        ``small_bunch``, ``max_boost``: a job of n < small_bunch particles
        advances chunk * small_bunch / n steps per tick (at most max_boost
        chunks), the rest ``chunk``.  A tick lasts as long as its largest
        jobs' work, so with equal step windows a small bunch with many steps
        waits through as many long ticks as a large one; its blocks are few,
        so a longer window costs the tick little.  A job's results do not
        depend on its windows (tracks are split-invariant bit for bit)."""
        torch = _torch()
        self.torch = torch
        self.lib = _lib.load()
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.budget = float(budget_bytes)
        self.chunk = int(chunk)
        self.use_graphs = use_graphs
        self.capture_after = max(1, int(capture_after))
        self.small_bunch = int(small_bunch)
        self.max_boost = max(1, int(max_boost))
        self.fields = FieldCache(capacity=16)
        self.compute = torch.cuda.Stream(device=self.device)
        self.upload = torch.cuda.Stream(device=self.device)
        self.active = []
        self.used_bytes = 0
        self._handle = None
        self._scratch = None
        self._graph = None
        self._h_cap = 0
        self.ticks = 0
        self.rebuilds = 0
        self.graph_captures = 0
        self.graph_replays = 0
        self._pool = concurrent.futures.ThreadPoolExecutor(max_workers=2)

    # -- admission -----------------------------------------------------------
    def _admit(self, job, now):
        """Allocate the job's device state and upload it on the upload stream."""
        torch = self.torch
        with torch.cuda.device(self.device), torch.cuda.stream(self.upload):
            df = self.fields.get(job.efield, job.bfield, job.precision, self.device)
            rf_omega, rf_phase = 0.0, None
            if job.rf is not None:
                rf_omega = job.rf.omega
                rf_phase = torch.from_numpy(np.array(np.broadcast_to(np.asarray(job.rf.phase, dtype=np.float64),
                                                                     (job.n,))))
            tr = DeviceTracker(job.algorithm, job.q_over_m, df, job.n, job.nsteps, job.dt, job.rec_every,
                               job.precision, rf_omega=rf_omega, rf_phase=rf_phase, t0=job.t0, record=True,
                               device=self.device)
            # through pinned host blocks (torch's caching host allocator keeps
            # each block until its copy is done): a copy from pageable memory
            # holds the host thread for the whole transfer
            r = torch.from_numpy(job.r0).pin_memory().to(self.device, non_blocking=True)
            v = torch.from_numpy(job.v0).pin_memory().to(self.device, non_blocking=True)
            tr.load(r, v, stream=self.upload)
        job._tracker, job._fields = tr, df
        job.t_admit = now
        self.used_bytes += job.device_bytes()

    def _desc(self, job):
        tr = job._tracker
        d = _lib.JobDesc()
        d.state = tr.state
        d.fields = tr.dfields.fields
        d.nsteps_total = tr.nsteps_total
        d.rec_every = tr.rec_every
        d.dt = tr.dt
        d.q_over_m = tr.q_over_m
        d.t0 = tr.t0
        d.rf_omega = tr.rf_omega
        d.rf_phase = tr.rf_phase.data_ptr() if tr.rf_phase is not None else None
        d.r_hist = tr.r_hist.data_ptr()
        d.v_hist = tr.v_hist.data_ptr()
        d.status = tr.status.data_ptr()
        d.steps_done = job.steps_done
        d.tick_steps = self._tick_steps(job)
        return d

    def _tick_steps(self, job):
        if job.n >= self.small_bunch:
            return 0
        boost = min(float(self.max_boost), self.small_bunch / max(job.n, 1))
        return int(self.chunk * boost)

    # -- job table and graph -----------------------------------------------------
    def _rebuild(self):
        torch = self.torch
        self._release_table()
        n = len(self.active)
        if n == 0:
            return
        # the new jobs' uploads (upload stream) must land before their first tick
        ev = torch.cuda.Event()
        ev.record(self.upload)
        self.compute.wait_event(ev)
        descs = (_lib.JobDesc * n)(*[self._desc(j) for j in self.active])
        nbytes = self.lib.ppt_jobs_scratch_bytes(n)
        if self._scratch is None or self._scratch.numel() < nbytes:
            self.compute.synchronize()
            self._scratch = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        handle = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.check(self.lib.ppt_jobs_create(descs, n, self._scratch.data_ptr(), handle,
                                                self.compute.cuda_stream))
        self._handle = handle.value
        steps, done = ctypes.c_void_p(), ctypes.c_void_p()
        _lib.check(self.lib.ppt_jobs_progress(self._handle, steps, done))
        # the counters live in the scratch tensor: read them through views of it
        base = self._scratch.data_ptr()
        so, do = steps.value - base, done.value - base
        self._d_steps = self._scratch[so:so + 8 * n].view(torch.int64)
        self._d_done = self._scratch[do:do + 4 * n].view(torch.int32)
        if self._h_cap < n:
            # pinned progress buffers, grown (never per table: a pinned
            # allocation costs more host time than a tick)
            self._h_cap = max(n, 2 * self._h_cap)
            self._h_steps_buf = torch.empty(self._h_cap, dtype=torch.int64, pin_memory=True)
            self._h_done_buf = torch.empty(self._h_cap, dtype=torch.int32, pin_memory=True)
        self._h_steps = self._h_steps_buf[:n]
        self._h_done = self._h_done_buf[:n]
        self.rebuilds += 1

    def _capture(self):
        """Capture the tick of the current (unchanged) job set in a CUDA graph."""
        torch = self.torch
        self.compute.synchronize()
        g = torch.cuda.CUDAGraph()
        cap = torch.cuda.Stream(device=self.device)
        with torch.cuda.device(self.device), torch.cuda.stream(cap):
            g.capture_begin()
            _lib.check(self.lib.ppt_jobs_tick(self._handle, self.chunk, cap.cuda_stream))
            g.capture_end()
        self._graph = g
        self.graph_captures += 1

    def _release_table(self):
        self._graph = None
        if self._handle is not None:
            self.lib.ppt_jobs_destroy(self._handle)
            self._handle = None

    def _tick(self):
        torch = self.torch
        with torch.cuda.device(self.device), torch.cuda.stream(self.compute):
            if self._graph is not None:
                self._graph.replay()
                self.graph_replays += 1
            else:
                _lib.check(self.lib.ppt_jobs_tick(self._handle, self.chunk, self.compute.cuda_stream))
            self._h_steps.copy_(self._d_steps, non_blocking=True)
            self._h_done.copy_(self._d_done, non_blocking=True)
        self.ticks += 1

    # -- retirement ------------------------------------------------------------
    def _collect(self, job, t_base):
        """Start copying a finished job's histories to the host on a worker
        thread, so the loop keeps issuing ticks meanwhile.  The copies go
        through the device's pinned ring (HostStager): a device-to-pageable
        copy runs at a few GB/s, the ring at the link's rate.  The job's last
        tick has completed (the loop synchronised on it), so the copies need
        no event."""
        tr = job._tracker
        stager = HostStager.for_device(self.device)

        def work():
            r = host_array(tuple(tr.r_hist.shape))
            v = host_array(tuple(tr.v_hist.shape))
            stager.copy(tr.r_hist, r)
            stager.copy(tr.v_hist, v)
            stager.finish()
            return r, v, time.perf_counter() - t_base

        return self._pool.submit(work)

    def _finish(self, collecting, finished, block=False):
        """Jobs whose results reached the host: record them, free their memory."""
        still = []
        for job, fut in collecting:
            if block or fut.done():
                job.r_hist, job.v_hist, job.t_done = fut.result()
                self.used_bytes -= job.device_bytes()
                job._tracker = None
                finished.append(job)
            else:
                still.append((job, fut))
        return still

    # -- main loop -------------------------------------------------------------
    def run(self, jobs, realtime=True):
        """Serve ``jobs`` (arrival times in seconds from the start).  With
        realtime=False an idle server jumps to the next arrival instead of
        sleeping.  Returns a report dict; each job gets t_admit, t_done,
        r_hist, v_hist."""
        torch = self.torch
        base = (self.ticks, self.rebuilds, self.graph_captures, self.graph_replays)
        for j in jobs:
            j.reset()
        pending = collections.deque(sorted(jobs, key=lambda j: j.arrival))
        finished, retiring, joining, collecting = [], [], [], []
        t_start = time.perf_counter()
        clock_offset = 0.0              # realtime=False: skipped idle time
        host = collections.Counter()
        gpu_tick_ms = 0.0
        stable = 0                      # ticks the current job set has run unchanged
        while pending or self.active or joining or retiring or collecting:
            t0 = time.perf_counter()
            # 1) enqueue this tick for the current job set
            ticked = False
            if self.active:
                # capture only with no result copy in flight: no other thread syncs on the device then
                if self.use_graphs and self._graph is None and stable >= self.capture_after and not collecting:
                    self._capture()
                ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                ev0.record(self.compute)
                self._tick()
                ev1.record(self.compute)
                ticked = True
            t1 = time.perf_counter()
            host["issue"] += t1 - t0
            # 2) while it runs: results of jobs finished last tick, then arrivals
            collecting += [(job, self._collect(job, t_start - clock_offset)) for job in retiring]
            retiring = []
            # with nothing to run, wait for the copies: they free the memory the next arrivals need
            collecting = self._finish(collecting, finished, block=not self.active and not joining)
            t2 = time.perf_counter()
            host["collect"] += t2 - t1
            now = t2 - t_start + clock_offset
            if not realtime and not self.active and not joining and pending and pending[0].arrival > now:
                clock_offset += pending[0].arrival - now
                now = pending[0].arrival
            while pending and pending[0].arrival <= now:
                job = pending[0]
                if self.used_bytes + job.device_bytes() > self.budget:
                    if not self.active and not joining and not collecting:
                        raise MemoryError(f"job {job.job_id} needs {job.device_bytes()} B, budget {self.budget}")
                    break
                pending.popleft()
                self._admit(job, now)
                joining.append(job)
            t3 = time.perf_counter()
            host["admit"] += t3 - t2
            # 3) end of the tick: progress, finished jobs
            changed = bool(joining)
            if ticked:
                self.compute.synchronize()
                gpu_tick_ms += ev0.elapsed_time(ev1)
                steps = self._h_steps.numpy()
                done = self._h_done.numpy()
                keep = []
                for i, job in enumerate(self.active):
                    job.steps_done = int(steps[i])
                    (retiring if done[i] else keep).append(job)
                if len(keep) != len(self.active):
                    changed = True
                self.active = keep
            t4 = time.perf_counter()
            host["wait"] += t4 - t3
            # 4) the next tick's job table
            if changed:
                self.active += joining
                joining = []
                self._rebuild() if self.active else self._release_table()
                stable = 0
            elif ticked:
                stable += 1
            host["rebuild"] += time.perf_counter() - t4
            if realtime and not self.active and not joining and not retiring and not collecting and pending:
                time.sleep(max(0.0, pending[0].arrival - (time.perf_counter() - t_start)))
        self._release_table()
        wall = time.perf_counter() - t_start
        lat = np.array([j.latency for j in finished])
        total_ps = sum(j.n * j.nsteps for j in finished)
        return {"jobs": len(finished), "wall_s": wall, "particle_steps": total_ps,
                "particle_steps_per_s": total_ps / wall if wall > 0 else 0.0,
                "p50_latency_s": float(np.percentile(lat, 50)) if lat.size else None,
                "p99_latency_s": float(np.percentile(lat, 99)) if lat.size else None,
                "max_latency_s": float(lat.max()) if lat.size else None,
                "ticks": self.ticks - base[0], "rebuilds": self.rebuilds - base[1],
                "graph_captures": self.graph_captures - base[2], "graph_replays": self.graph_replays - base[3],
                "gpu_tick_s": gpu_tick_ms / 1e3,
                "gpu_busy_fraction": gpu_tick_ms / 1e3 / wall if wall > 0 else 0.0,
                "host_s": {k: round(v, 4) for k, v in host.items()}}
