"""GPU drop-in for the reference's ``Pusher`` (src/PyPATools/pusher.py:430-1037).

``PusherGPU`` keeps the reference's constructor, method names, signatures,
return shapes and error messages:

    Pusher(ion, algorithm='boris', use_numba=True, electrode_assembly=None)
    push(r(3,), v(3,), efield, bfield, dt)                      -> (r, v)
    track(r0(3,), v0(3,), efield, bfield, nsteps, dt, rec_every_n_steps=1)
                                                                -> (r_hist(n_rec,3), v_hist)
    push_batch(r(M,3), v(M,3), efield, bfield, dt)              -> (r, v)
    track_batch(r0(M,3), v0(M,3), efield, bfield, nsteps, dt, rec_every_n_steps=1, verbose=False)
                                                                -> (r_hist(n_rec,M,3), v_hist, active(M,))
    change_algorithm(name), ALGORITHMS, __repr__

and adds keyword-only options: ``precision`` ('fp64' = the reference method
in float64, the drop-in; 'mixed' = the mixed-precision form), ``device``,
``snapshot`` ('host' numpy arrays like the reference, or 'device' torch
tensors), ``steps_per_launch``, ``sort_every`` (cell re-sort interval; 'auto' = every 300
steps for bunches of 65536 or more, none below) and,
on ``track_batch``, ``rf`` (an ``RFModulation`` multiplying E by
cos(2 pi f t + phi_i)) and ``t0``.  ``electrode_assembly`` takes an
``electrodes.ElectrodeSurface`` (or any object with ``vertices`` and
``triangles``): particles whose step meets it stop, as in the reference.

All work runs in libppt.so kernels; there is no CPU fallback.
"""
import math
import mmap
import warnings

import numpy as np

from . import _lib
from .device_fields import FieldCache

REFERENCE_ALGORITHMS = ["leapfrog", "boris", "rk4", "yoshida", "vay_rel", "rk4_rel", "yoshida_rel"]
EXTRA_ALGORITHMS = ["boris_rel", "vay"]
MIXED_ALGORITHMS = ("leapfrog", "boris", "rk4", "vay_rel", "rk4_rel", "boris_rel", "vay")


class RFModulation:
    """Time dependence of E: E(x, t) = E(x) cos(2 pi frequency t + phase_i).

    ``phase`` is a scalar or one value per particle [rad]."""

    def __init__(self, frequency, phase=0.0):
        self.frequency = float(frequency)
        self.phase = phase

    @property
    def omega(self):
        return 2.0 * math.pi * self.frequency


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("PusherGPU needs a CUDA device (there is no CPU fallback)")
    return torch


def default_steps_per_launch(n, nsteps):
    """Steps per kernel launch: whole tracks for small bunches, about 4e9
    particle-steps per launch for large ones (launches of roughly a second or
    less, so the stream stays responsive)."""
    if nsteps <= 0:
        return 1
    return int(max(1, min(nsteps, 2 ** 31 - 1, math.ceil(4e9 / max(n, 1)))))


def check_rows(t, n, device, name):
    """``t`` as the state load / store kernels read and write it: a
    contiguous (n, 3) float64 tensor on ``device`` (a CUDA device with its
    index).  Anything else is refused before a launch: the kernels address n
    rows of 24 B from its data pointer."""
    import torch
    if not torch.is_tensor(t):
        raise TypeError(f"{name} must be a torch tensor, got {type(t).__name__}")
    if t.dtype != torch.float64 or tuple(t.shape) != (n, 3):
        raise ValueError(f"{name} must be a ({n}, 3) float64 tensor, got {tuple(t.shape)} {t.dtype}")
    if t.device != device or not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous on {device} (got {t.device}, "
                         f"{'contiguous' if t.is_contiguous() else 'strided'})")
    return t


class DeviceTracker:
    """Device-resident state of one bunch: the building block of
    ``track_batch``, the serving loop and the benchmark.

    State (structure of arrays), snapshot histories, the slot -> row order
    after cell sorts, the RF phases and the device status word all live in
    torch CUDA tensors owned by this object."""

    def __init__(self, algorithm, q_over_m, dfields, n, nsteps_total, dt, rec_every=1, precision="fp64",
                 rf_omega=0.0, rf_phase=None, t0=0.0, record=True, stagger=True, counters=False,
                 device=None, surface=None, dt_rows=None):
        torch = _torch()
        self.torch = torch
        if algorithm not in _lib.ALG_IDS:
            raise ValueError(f"unknown algorithm {algorithm!r}")
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        if precision == "mixed" and algorithm not in MIXED_ALGORITHMS:
            raise NotImplementedError(f"the mixed form covers {MIXED_ALGORITHMS}; use precision='fp64'")
        if rec_every < 1:
            raise ValueError("rec_every_n_steps must be >= 1")
        self.lib = _lib.load()
        self.device = torch.device(device) if device is not None else dfields.device
        self.algorithm = algorithm
        self.precision = precision
        self.q_over_m = float(q_over_m)
        self.dfields = dfields
        self.n = int(n)
        self.nsteps_total = int(nsteps_total)
        self.dt = float(dt)
        self.rec_every = int(rec_every)
        self.n_rec = self.nsteps_total // self.rec_every + 1
        self.t0 = float(t0)
        self.stagger = stagger
        self.step = 0
        dev = self.device
        n = self.n
        if precision == "fp64":
            self.f64 = torch.empty(6 * n, dtype=torch.float64, device=dev)
            self.i32 = self.f32 = None
        else:
            self.f64 = None
            self.i32 = torch.empty(3 * n, dtype=torch.int32, device=dev)
            self.f32 = torch.empty(12 * n, dtype=torch.float32, device=dev)
        self.state = _lib.State(_lib.PREC_F64 if precision == "fp64" else _lib.PREC_MIXED,
                                _lib.ALG_IDS[algorithm], n,
                                self.f64.data_ptr() if self.f64 is not None else None,
                                self.i32.data_ptr() if self.i32 is not None else None,
                                self.f32.data_ptr() if self.f32 is not None else None)
        # an electrode surface (float64 form): particles whose step segment
        # meets it stop; active[row] says which are still tracked
        self.surface = None
        self.active = None
        if surface is not None:
            if precision != "fp64" and algorithm != "boris":
                raise NotImplementedError("electrode surfaces run in the float64 form and in the mixed form's "
                                          "boris; use precision='fp64'")
            self.surface = surface.handle(dev)
            self.active = torch.ones(n, dtype=torch.uint8, device=dev)
        if record:
            # stopped particles leave their later rows unwritten: NaN, as the
            # reference's histories start (pusher.py:947-948)
            make = torch.full if surface is not None else torch.empty
            args = (float("nan"),) if surface is not None else ()
            self.r_hist = make((self.n_rec, n, 3), *args, dtype=torch.float64, device=dev)
            self.v_hist = make((self.n_rec, n, 3), *args, dtype=torch.float64, device=dev)
        else:
            self.r_hist = self.v_hist = None
        self.rf_omega = float(rf_omega)
        if rf_phase is not None:
            ph = torch.as_tensor(rf_phase, dtype=torch.float64)
            if ph.ndim == 0:
                ph = ph.expand(n)
            if tuple(ph.shape) != (n,):
                raise ValueError(f"rf_phase must be a scalar or ({n},), got {tuple(ph.shape)}")
            self.rf_phase = ph.to(dev).contiguous().clone()
        else:
            self.rf_phase = None
        # one time step per particle (row order): the float64 RK4 pushers only,
        # as in the reference's batch RK4 step (pusher.py:815-816)
        self.dt_rows = None
        if dt_rows is not None:
            if precision != "fp64" or algorithm not in ("rk4", "rk4_rel"):
                raise NotImplementedError("a per-particle dt runs in the float64 form of rk4 and rk4_rel")
            d = torch.as_tensor(dt_rows, dtype=torch.float64)
            if tuple(d.shape) != (n,):
                raise ValueError(f"dt must be a scalar or ({n},), got {tuple(d.shape)}")
            self.dt_rows = d.to(dev).contiguous().clone()
        self.order = None
        self.row_order = False   # order is the identity (restore_order): the kernels need not read it
        self.sort_scratch = None
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        self.counters = torch.zeros(2, dtype=torch.int64, device=dev) if counters else None
        self.launches = 0

    def _stream(self, stream):
        return _lib.stream_handle(stream)

    def load(self, r, v, stream=None):
        """r, v: (n,3) float64 CUDA tensors, loaded in row order."""
        dev = self.status.device
        check_rows(r, self.n, dev, "r")
        check_rows(v, self.n, dev, "v")
        _lib.check(self.lib.ppt_state_load(self.state, self.dfields.fields, r.data_ptr(), v.data_ptr(),
                                           self._stream(stream)))
        if self.rf_phase is not None and self.order is not None and not self.row_order:
            # the RF phases were permuted with the old state: back to rows
            with self.torch.cuda.stream(stream if stream is not None else self.torch.cuda.current_stream()):
                self.rf_phase.index_copy_(0, self.order, self.rf_phase.clone())
        self.order = None           # slot s holds row s again
        self.row_order = False
        self.launches += 1

    def advance(self, k, stream=None):
        k = int(k)
        if self.step + k > self.nsteps_total:
            raise ValueError("advance past nsteps_total")
        flags = 0
        if self.stagger:
            if self.step == 0:
                flags |= _lib.TRACK_INIT
            if self.step + k == self.nsteps_total:
                flags |= _lib.TRACK_FINAL
        a = _lib.TrackArgs()
        a.step0 = self.step
        a.nsteps = k
        a.nsteps_total = self.nsteps_total
        a.rec_every = self.rec_every
        a.flags = flags
        a.dt = self.dt
        a.q_over_m = self.q_over_m
        a.t0 = self.t0
        a.rf_omega = self.rf_omega
        a.rf_phase = self.rf_phase.data_ptr() if self.rf_phase is not None else None
        a.r_hist = self.r_hist.data_ptr() if self.r_hist is not None else None
        a.v_hist = self.v_hist.data_ptr() if self.v_hist is not None else None
        a.order = self._order_ptr()
        a.status = self.status.data_ptr()
        a.counters = self.counters.data_ptr() if self.counters is not None else None
        if self.surface is not None:
            a.surface = self.surface
            a.active = self.active.data_ptr()
        if self.dt_rows is not None:
            a.dt_rows = self.dt_rows.data_ptr()
        _lib.check(self.lib.ppt_track(self.state, self.dfields.fields, a, self._stream(stream)))
        if k > 0 or flags:
            self.launches += 1
        self.step += k

    def run(self, nsteps, chunk, sort_every=0, long_chunk=None, after_launch=None, launch_events=None,
            stream=None, in_flight=2, free_chunk=None):
        """Advance ``nsteps`` steps in launches of at most ``chunk`` steps.

        With ``sort_every`` > 0 and maps present the schedule follows the
        bunch: while the maps are populated, every launch of ``sort_every``
        steps starts with a cell sort; once a finished launch spent less than
        1/16 of its particle-steps inside a map, one more sort (it groups the
        stragglers still inside, see ``ppt_cell_sort``) and then launches of
        ``long_chunk`` steps without sorts, which read and write the state
        less often; the sorted schedule returns when the in-map share rises
        again.  The share comes from the device counters, copied to pinned
        memory after each launch and read with a lag: at most ``in_flight``
        launches are queued ahead, so the GPU never waits on the host.
        Once a finished launch met no map at all, the particles go back to
        row order (``restore_order``) for the snapshot rows' sake, until a
        map holds particles again; launches in row order with no map met take
        ``free_chunk`` steps (default 10 ``long_chunk``): their field-free runs
        cost little, so the state read and written per launch is what a
        longer launch saves, while the counters still come back often enough
        to notice a bunch that meets a map again.
        ``after_launch(steps_done)`` runs after each launch is enqueued;
        ``launch_events`` (a list) receives (start event, end event, first
        step, steps) for each track launch."""
        torch = self.torch
        nsteps = int(nsteps)
        chunk = max(1, int(chunk))
        adaptive = sort_every > 0 and self.dfields.has_maps and self.n > 0
        long_chunk = max(chunk, int(long_chunk or 10 * max(sort_every, 1)))
        free_chunk = max(long_chunk, int(free_chunk or 10 * long_chunk))
        st = torch.cuda.current_stream(self.device) if stream is None else stream
        if adaptive and self.counters is None:
            self.counters = torch.zeros(2, dtype=torch.int64, device=self.device)
        pending = []            # (event, pinned counters copy, steps in the launch)
        last_hits = None
        dense = True            # the maps hold a good share of the particles
        sorted_sparse = False   # the grouping sort after the bunch left has been made
        empty = False           # the newest finished launch met no map
        done = 0
        if nsteps == 0:
            self.advance(0, stream)
            return
        while done < nsteps:
            if adaptive:
                # newest in-map share from the launches that have finished
                while pending and (len(pending) > in_flight or pending[0][0].query()):
                    ev, host, k_done = pending.pop(0)
                    ev.synchronize()
                    hits = int(host[0])
                    if last_hits is not None:
                        frac = (hits - last_hits) / max(1, self.n * k_done)
                        if frac * 16 >= 1:
                            dense, sorted_sparse = True, False
                        else:
                            dense = False
                        empty = hits == last_hits
                    last_hits = hits
                if dense or not sorted_sparse:
                    if (self.step % sort_every == 0) or not dense:
                        self.sort(stream)
                    sorted_sparse = not dense
                elif empty and not self.row_order:
                    self.restore_order(stream)
                if dense:
                    k = min(sort_every, chunk, nsteps - done)
                else:
                    k = min(free_chunk if (empty and self.row_order) else long_chunk, nsteps - done)
                if dense:
                    k = min(k, sort_every - self.step % sort_every)
            else:
                k = min(chunk, nsteps - done)
            if launch_events is not None:
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                step0 = self.step
                a.record(st)
                self.advance(k, stream)
                b.record(st)
                launch_events.append((a, b, step0, k))
            else:
                self.advance(k, stream)
            done += k
            if adaptive:
                host = torch.empty(2, dtype=torch.int64, pin_memory=True)
                with torch.cuda.stream(st):
                    host.copy_(self.counters, non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(st)
                pending.append((ev, host, k))
            if after_launch is not None:
                after_launch(done)

    def _order_ptr(self):
        return None if self.order is None or self.row_order else self.order.data_ptr()

    def _sort_scratch(self):
        if self.order is None:
            self.order = self.torch.arange(self.n, dtype=self.torch.int64, device=self.device)
        if self.sort_scratch is None:
            nbytes = self.lib.ppt_cell_sort_scratch_bytes(self.n)
            self.sort_scratch = self.torch.empty(nbytes, dtype=self.torch.uint8, device=self.device)
        return self.sort_scratch

    def restore_order(self, stream=None):
        """Put the particles back in row order (``ppt_restore_order``); the
        order array becomes the identity and the kernels stop reading it."""
        if self.n == 0 or self.order is None or self.row_order:
            return
        scratch = self._sort_scratch()
        _lib.check(self.lib.ppt_restore_order(self.state, self.order.data_ptr(),
                                              self.rf_phase.data_ptr() if self.rf_phase is not None else None,
                                              scratch.data_ptr(), self._stream(stream)))
        self.row_order = True
        # inverse, gather and iota kernels (the fill and copy-backs are memset / memcpy calls)
        self.launches += 3

    def sort(self, stream=None):
        """Reorder particles by cell (gather locality)."""
        if not self.dfields.has_maps or self.n == 0:
            return
        scratch = self._sort_scratch()
        self.row_order = False
        _lib.check(self.lib.ppt_cell_sort(self.state, self.dfields.fields, self.order.data_ptr(),
                                          self.rf_phase.data_ptr() if self.rf_phase is not None else None,
                                          scratch.data_ptr(), self._stream(stream)))
        # keys, tile scan, top scan, scan add, scatter, then one copy-back per
        # permuted array (state block(s), order, RF phase)
        self.launches += 5 + (1 if self.precision == "fp64" else 2) + 1 + (1 if self.rf_phase is not None else 0)

    def store(self, r, v, stream=None):
        """Write the current state as (n,3) float64 r, v in row order."""
        for t, name in ((r, "r"), (v, "v")):
            if t is not None:
                check_rows(t, self.n, self.status.device, name)
        _lib.check(self.lib.ppt_state_store(self.state, self.dfields.fields, self._order_ptr(),
                                            r.data_ptr() if r is not None else None,
                                            v.data_ptr() if v is not None else None, self._stream(stream)))
        self.launches += 1

    def device_status(self):
        return int(self.status.item())

    def counter_values(self):
        if self.counters is None:
            return None
        c = self.counters.cpu().numpy()
        return {"map_hits": int(c[0]), "particle_steps": int(c[1])}


class HostResultPool:
    """Anonymous host mappings for results the GPU fills (``host_array``),
    recycled once the caller drops the arrays built on them.

    A fresh mapping costs its first touch: the kernel zeroes every page as
    the results land (about 50 GB/s with 24 threads on a B200 host even with
    transparent huge pages, against 145 GB/s for a copy into touched pages),
    which for the 19.7 GB histories of a 1e7-particle track is slower than
    the PCIe link.  When every array over a mapping has been released, the
    mapping goes back to this pool, still touched, and the next request of
    the same size takes it; the pool keeps at most ``limit`` bytes of free
    mappings (``PPT_HOST_POOL_BYTES``, default 32 GiB; 0 disables it) and
    unmaps the rest.  The results are always fully written before they are
    returned, so a recycled mapping's earlier contents are never visible."""

    def __init__(self, limit):
        import threading
        self.limit = int(limit)
        self.free = {}          # nbytes -> [mmap, ...]
        self.free_bytes = 0
        self.lock = threading.RLock()   # a collection inside take() may call give()

    def take(self, nbytes):
        with self.lock:
            maps = self.free.get(nbytes)
            if maps:
                self.free_bytes -= nbytes
                return maps.pop()
        m = mmap.mmap(-1, nbytes, flags=mmap.MAP_PRIVATE | mmap.MAP_ANONYMOUS)
        try:
            m.madvise(mmap.MADV_HUGEPAGE)
        except (OSError, AttributeError):
            pass        # transparent huge pages off: plain pages, still correct
        return m

    def give(self, m):
        nbytes = len(m)
        with self.lock:
            if self.free_bytes + nbytes <= self.limit:
                self.free.setdefault(nbytes, []).append(m)
                self.free_bytes += nbytes
        # over the limit: dropped here and unmapped with its last reference
        # (the array's buffer export on it is released after this callback)

    def clear(self):
        """Drop every free mapping (unmapped as their references go)."""
        with self.lock:
            self.free, self.free_bytes = {}, 0


def _pool_limit():
    import os
    try:
        return int(float(os.environ.get("PPT_HOST_POOL_BYTES", 32 << 30)))
    except ValueError:
        return 32 << 30


HOST_POOL = HostResultPool(_pool_limit())


def host_array(shape, dtype=np.float64):
    """A numpy array for results the GPU fills, backed (from 64 MiB up) by an
    anonymous mapping advised for transparent huge pages, taken from
    ``HOST_POOL``: writing tens of GB into fresh 4 KiB pages is bound by page
    faults (27 GB/s measured with 24 threads on a B200 host), with huge pages
    by their zeroing (50 GB/s), and into a recycled mapping by the copy
    alone.  The mapping returns to the pool when the array and every view of
    it are gone."""
    import weakref
    nbytes = int(np.prod(shape)) * np.dtype(dtype).itemsize
    if nbytes < (64 << 20) or not hasattr(mmap, "MADV_HUGEPAGE"):
        return np.empty(shape, dtype)
    m = HOST_POOL.take(nbytes)
    base = np.frombuffer(m, dtype=dtype)
    # views of the result keep `base` alive; once it is collected its buffer
    # export on m is released and m can serve the next request
    weakref.finalize(base, HOST_POOL.give, m)
    return base.reshape(shape)


class HostStager:
    """Host <-> device copies through a ring of pinned buffers.

    Device -> numpy: each piece (``chunk`` bytes at most) goes device -> pinned
    buffer on a copy stream (PCIe at ~50 GB/s on B200 hosts), then a worker
    thread copies it into the destination numpy array (numpy releases the GIL
    for the copy); the ring keeps ``slots`` pieces in flight.  The
    destinations of ``track_batch`` are fresh huge-page-advised arrays
    (``host_array``), whose first touch keeps up with the link; with 4 KiB
    pages it ran at half of it.  Pinning the destination instead costs about a
    second per 1.5 GB whenever the caller still holds earlier results, and a
    device copy into pageable memory runs at ~2 GB/s.  numpy -> device
    (``upload``): worker threads copy the pieces into the pinned buffers and
    enqueue their host-to-device copies."""

    _by_device = {}

    def __init__(self, device, chunk=32 << 20, slots=24):
        import threading
        from concurrent.futures import ThreadPoolExecutor
        torch = _torch()
        self.torch = torch
        self.device = device
        self.chunk = int(chunk)
        self.buffers = [torch.empty(self.chunk, dtype=torch.uint8, pin_memory=True) for _ in range(slots)]
        self.views = [b.numpy() for b in self.buffers]
        self.events = [torch.cuda.Event() for _ in range(slots)]
        self.pending = [None] * slots
        self.next = 0
        self.stream = torch.cuda.Stream(device=device)
        self.pool = ThreadPoolExecutor(max_workers=slots)
        self.lock = threading.Lock()

    @classmethod
    def for_device(cls, device):
        import torch
        key = torch.device(device).index if torch.device(device).index is not None else torch.cuda.current_device()
        st = cls._by_device.get(key)
        if st is None:
            st = cls._by_device[key] = cls(torch.device("cuda", key))
        return st

    def copy(self, src, dst, after=None):
        """Queue the copy of the contiguous device tensor ``src`` into the
        contiguous numpy array ``dst`` (same bytes), after event ``after``.
        The caller keeps ``src`` alive (and unchanged) until ``finish()``
        returns: the copy stream reads it after this call returns."""
        with self.lock:
            self._copy(src, dst, after)

    def _copy(self, src, dst, after):
        torch = self.torch
        sb = src.reshape(-1).view(torch.uint8)
        db = dst.reshape(-1).view(np.uint8)
        if after is not None:
            self.stream.wait_event(after)
        for a in range(0, db.size, self.chunk):
            b = min(a + self.chunk, db.size)
            k = self.next
            self.next = (k + 1) % len(self.buffers)
            if self.pending[k] is not None:
                self.pending[k].result()          # the slot's previous piece is in its numpy array
            with torch.cuda.stream(self.stream):
                self.buffers[k][:b - a].copy_(sb[a:b], non_blocking=True)
                self.events[k].record(self.stream)
            self.pending[k] = self.pool.submit(self._land, k, db, a, b)

    def _land(self, k, db, a, b):
        self.events[k].synchronize()
        np.copyto(db[a:b], self.views[k][:b - a])

    def upload(self, src, dst):
        """Copy the contiguous numpy array ``src`` into the contiguous device
        tensor ``dst`` (same bytes) through the ring: worker threads copy the
        pieces into the pinned buffers and enqueue each piece's host-to-device
        copy on the copy stream.  Returns an event recorded after the last
        piece; the caller's stream waits on it before reading ``dst``."""
        torch = self.torch
        sb = src.reshape(-1).view(np.uint8)
        db = dst.reshape(-1).view(torch.uint8)
        with self.lock:
            staged = []
            for a in range(0, sb.size, self.chunk):
                b = min(a + self.chunk, sb.size)
                k = self.next
                self.next = (k + 1) % len(self.buffers)
                if self.pending[k] is not None:
                    self.pending[k].result()      # the slot's previous piece has landed or left
                self.events[k].synchronize()      # and its last copy is done
                self.pending[k] = self.pool.submit(self._stage, k, sb, db, a, b)
                staged.append(self.pending[k])
            for f in staged:
                f.result()
            ev = torch.cuda.Event()
            ev.record(self.stream)
        return ev

    def _stage(self, k, sb, db, a, b):
        torch = self.torch
        np.copyto(self.views[k][:b - a], sb[a:b])
        with torch.cuda.device(self.device), torch.cuda.stream(self.stream):
            db[a:b].copy_(self.buffers[k][:b - a], non_blocking=True)
            self.events[k].record(self.stream)

    def finish(self):
        with self.lock:
            for k, f in enumerate(self.pending):
                if f is not None:
                    f.result()
                    self.pending[k] = None


class PusherGPU:
    """Batch and single-particle tracking on the GPU with the reference's API."""

    ALGORITHMS = list(REFERENCE_ALGORITHMS)
    EXTRA_ALGORITHMS = list(EXTRA_ALGORITHMS)

    def __init__(self, ion, algorithm="boris", use_numba=True, electrode_assembly=None, *, precision="fp64",
                 device=None, snapshot="host", steps_per_launch=None, sort_every="auto"):
        self.ion = ion
        self.q_over_m = ion.q_over_m
        algorithm = algorithm.lower()
        if algorithm not in self.ALGORITHMS + self.EXTRA_ALGORITHMS:
            raise ValueError(f"Unknown algorithm '{algorithm}'. Must be one of {self.ALGORITHMS}")
        # pusher.py:482-489: leapfrog with a >100 keV ion object switches to vay_rel
        if algorithm == "leapfrog" and hasattr(ion, "energy_mev") and ion.energy_mev > 0.1:
            warnings.warn("Leapfrog is non-relativistic. Using 'vay_rel' instead for better relativistic "
                          "accuracy.", UserWarning)
            algorithm = "vay_rel"
        self.surface = None
        if electrode_assembly is not None:
            from .electrodes import ElectrodeSurface
            self.surface = ElectrodeSurface.from_assembly(electrode_assembly)
            if precision != "fp64" and algorithm != "boris":
                raise NotImplementedError("electrode surfaces run in the float64 form and in the mixed form's "
                                          "boris; use precision='fp64'")
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        if snapshot not in ("host", "device"):
            raise ValueError("snapshot must be 'host' or 'device'")
        self.algorithm = algorithm
        self.use_numba = use_numba
        self.relativistic = algorithm.endswith("_rel")
        self.elec_assy = electrode_assembly
        self.precision = precision
        self.device = device
        self.snapshot = snapshot
        self.steps_per_launch = steps_per_launch
        if sort_every != "auto":
            sort_every = int(sort_every)
        self.sort_every = sort_every
        self._fields = FieldCache(capacity=4)
        self.last_tracker = None

    # -- helpers -----------------------------------------------------------
    # 'auto' cell-sort interval: bunches this large re-sort every AUTO_SORT_STEPS
    # steps while they are in a map (sorting never changes a result, it only
    # makes the corner gathers of a warp hit the same records); smaller bunches
    # are not sorted, a sort costing more than it saves there.
    AUTO_SORT_MIN_PARTICLES = 65536
    AUTO_SORT_STEPS = 300

    def _sort_interval(self, m):
        if self.sort_every == "auto":
            return self.AUTO_SORT_STEPS if m >= self.AUTO_SORT_MIN_PARTICLES else 0
        return self.sort_every

    def _device_fields(self, efield, bfield):
        _torch()
        return self._fields.get(efield, bfield, self.precision, self.device)

    @staticmethod
    def _as_rows(a, name):
        a = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
        if a.ndim != 2 or a.shape[1] != 3:
            raise ValueError(f"{name} must have shape (M, 3), got {a.shape}")
        return a

    def _time_step(self, dt, m):
        """(scalar dt, per-particle dt or None).  The reference's batch RK4
        step takes an array dt, one value per particle (pusher.py:815-816);
        its other pushers take a float."""
        if np.isscalar(dt) or np.ndim(dt) == 0:
            return float(dt), None
        if self.algorithm not in ("rk4", "rk4_rel") or self.precision != "fp64":
            raise TypeError("dt must be a scalar (an array dt is taken by the float64 rk4 and rk4_rel only)")
        d = np.ascontiguousarray(np.asarray(dt, dtype=np.float64))
        if d.shape != (m,):
            raise ValueError(f"dt must be a scalar or have shape ({m},), got {d.shape}")
        return (float(d[0]) if m else 0.0), d

    def _upload(self, a, device):
        torch = _torch()
        t = torch.from_numpy(a)
        if device.type == "cuda":
            t = t.pin_memory()
        return t.to(device, non_blocking=True)

    # -- batch API -----------------------------------------------------------
    def push_batch(self, r_array, v_array, efield, bfield, dt):
        """One step for M particles (pusher.py:699-801): no half-step
        staggering, exactly the reference's push_batch.  ``dt`` may be an (M,)
        array for rk4 / rk4_rel in the float64 form, as in the reference."""
        r = self._as_rows(r_array, "r_array")
        v = self._as_rows(v_array, "v_array")
        if r.shape != v.shape:
            raise ValueError("r_array and v_array must have the same shape")
        m = r.shape[0]
        dt, dt_rows = self._time_step(dt, m)
        if m == 0:
            return r.copy(), v.copy()
        torch = _torch()
        df = self._device_fields(efield, bfield)
        tr = DeviceTracker(self.algorithm, self.q_over_m, df, m, 1, dt, 1, self.precision, record=False,
                           stagger=False, device=self.device, dt_rows=dt_rows)
        d_r, d_v = self._upload(r, df.device), self._upload(v, df.device)
        with torch.cuda.device(df.device):
            tr.load(d_r, d_v)
            tr.advance(1)
            tr.store(d_r, d_v)
        return d_r.cpu().numpy(), d_v.cpu().numpy()

    def track_batch(self, r0_array, v0_array, efield, bfield, nsteps, dt, rec_every_n_steps=1, verbose=False,
                    *, rf=None, t0=0.0, _collide=True):
        """Track M particles (pusher.py:894-1012).  Returns
        (r_hist (n_rec, M, 3), v_hist, active (M,)) with
        n_rec = nsteps // rec_every_n_steps + 1.  With an electrode assembly,
        a particle whose step meets it stops after that step (its later rows
        stay NaN, no closing half step) and is False in ``active``.  ``dt``
        may be an (M,) array for rk4 / rk4_rel in the float64 form, as in
        the reference."""
        nsteps = int(nsteps)
        rec = int(rec_every_n_steps)
        if nsteps < 0:
            raise ValueError("nsteps must be >= 0")
        if rec < 1:
            raise ValueError("rec_every_n_steps must be >= 1")
        r0 = self._as_rows(r0_array, "r0_array")
        v0 = self._as_rows(v0_array, "v0_array")
        if r0.shape != v0.shape:
            raise ValueError("r0_array and v0_array must have the same shape")
        m = r0.shape[0]
        dt, dt_rows = self._time_step(dt, m)
        n_rec = nsteps // rec + 1
        torch = _torch()
        if m == 0:
            empty = np.full((n_rec, 0, 3), np.nan)
            if self.snapshot == "device":
                return (torch.from_numpy(empty).cuda(), torch.from_numpy(empty.copy()).cuda(),
                        np.ones(0, dtype=bool))
            return empty, empty.copy(), np.ones(0, dtype=bool)
        df = self._device_fields(efield, bfield)
        stager = HostStager.for_device(df.device)
        uploads = []

        def upload(a):
            t = torch.empty(a.shape, dtype=torch.float64, device=df.device)
            uploads.append(stager.upload(np.ascontiguousarray(a, dtype=np.float64), t))
            return t

        rf_omega, rf_phase = 0.0, None
        if rf is not None:
            rf_omega = rf.omega
            rf_phase = upload(np.broadcast_to(np.asarray(rf.phase, dtype=np.float64), (m,)))
        d_r0, d_v0 = upload(r0), upload(v0)
        with torch.cuda.device(df.device):
            for ev in uploads:                 # the tracker reads them on this stream
                torch.cuda.current_stream().wait_event(ev)
        surface = self.surface if _collide else None
        tr = DeviceTracker(self.algorithm, self.q_over_m, df, m, nsteps, dt, rec, self.precision,
                           rf_omega=rf_omega, rf_phase=rf_phase, t0=t0, record=True, device=self.device,
                           surface=surface, dt_rows=dt_rows)
        self.last_tracker = tr
        chunk = self.steps_per_launch or default_steps_per_launch(m, nsteps)
        sort_every = self._sort_interval(m)
        if sort_every > 0:
            chunk = min(chunk, sort_every)
        to_host = self.snapshot == "host"
        with torch.cuda.device(df.device):
            if to_host:
                # Snapshot rows stream to the numpy results while later
                # launches run: finished rows go through a small ring of
                # pinned buffers (HostStager) instead of pinning the whole
                # histories, which costs seconds per call for large bunches.
                h_r = host_array((n_rec, m, 3))
                h_v = host_array((n_rec, m, 3))
                compute = torch.cuda.current_stream()
                copied = 0

                def drain(upto):
                    nonlocal copied
                    if upto <= copied:
                        return
                    ev = torch.cuda.Event()
                    ev.record(compute)
                    stager.copy(tr.r_hist[copied:upto], h_r[copied:upto], ev)
                    stager.copy(tr.v_hist[copied:upto], h_v[copied:upto], ev)
                    copied = upto
            tr.load(d_r0, d_v0)

            def after_launch(done):
                if verbose:
                    print(f"Step {done}/{nsteps} ({100 * done / nsteps:.0f}%)")
                if to_host and done < nsteps:
                    # records 0 .. done // rec are final; the last one waits for
                    # the closing half step of the Boris family
                    drain(min(done // rec + 1, n_rec - 1))

            tr.run(nsteps, chunk, sort_every=sort_every, after_launch=after_launch)
            if to_host:
                drain(n_rec)
                stager.finish()
            status = tr.device_status()
        if status & _lib.STATUS_NONFINITE:
            warnings.warn("non-finite particle state encountered during tracking", RuntimeWarning)
        if status & _lib.STATUS_RANGE:
            warnings.warn("mixed form: a particle went 2^24 cells or more from the map; its position is no "
                          "longer exact (use precision='fp64' for such tracks)", RuntimeWarning)
        if verbose:
            print(f"Tracking complete: {nsteps} steps, {m} particles")
        active = np.ones(m, dtype=bool) if tr.active is None else tr.active.cpu().numpy().astype(bool)
        if not to_host:
            return tr.r_hist, tr.v_hist, active
        return h_r, h_v, active

    # -- single-particle API -------------------------------------------------
    def push(self, r, v, efield, bfield, dt):
        """One step of one particle (pusher.py:508-565)."""
        rn, vn = self.push_batch(np.asarray(r, dtype=np.float64).reshape(1, 3),
                                 np.asarray(v, dtype=np.float64).reshape(1, 3), efield, bfield, dt)
        return rn[0], vn[0]

    def track(self, r0, v0, efield, bfield, nsteps, dt, rec_every_n_steps=1):
        """Track one particle (pusher.py:620-693): (n_rec, 3) histories."""
        snap = self.snapshot
        self.snapshot = "host"
        try:
            # the reference's single-particle track makes no collision test
            rh, vh, _ = self.track_batch(np.asarray(r0, dtype=np.float64).reshape(1, 3),
                                         np.asarray(v0, dtype=np.float64).reshape(1, 3), efield, bfield,
                                         nsteps, dt, rec_every_n_steps, _collide=False)
        finally:
            self.snapshot = snap
        return rh[:, 0, :], vh[:, 0, :]

    # -- utilities -------------------------------------------------------------
    def change_algorithm(self, algorithm):
        algorithm = algorithm.lower()
        if algorithm not in self.ALGORITHMS + self.EXTRA_ALGORITHMS:
            raise ValueError(f"Unknown algorithm '{algorithm}'. Must be one of {self.ALGORITHMS}")
        # as the reference (pusher.py:1033), the electrode assembly is not carried over
        self.__init__(self.ion, algorithm=algorithm, use_numba=self.use_numba, precision=self.precision,
                      device=self.device, snapshot=self.snapshot, steps_per_launch=self.steps_per_launch,
                      sort_every=self.sort_every)

    def __repr__(self):
        return (f"PusherGPU(ion={getattr(self.ion, 'name', '?')}, algorithm='{self.algorithm}', "
                f"relativistic={self.relativistic}, precision={self.precision})")


# The reference's class name, so scripts can switch with one import.
Pusher = PusherGPU
