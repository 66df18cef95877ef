"""Serving loop: continuous batching of leapfrog sessions on one GPU.

Sessions are N-body systems integrated with kick-drift-kick leapfrog. They
arrive at any time, wait in a queue, and are admitted when the HBM budget and
the latency target allow. A lane owns an engine context, a CUDA stream and, in
threaded mode, a host thread, and advances its sessions one step per tick: the
half kicks and drifts of all its sessions are one elementwise pass over their
concatenated state, and their force evaluations are batched into ONE forest
build + evaluation (fmmx_build_ensemble_device) -- one tree per session, no
interaction across sessions, each session's result bitwise the one it gets
alone. A session joins a lane by riding along in the lane's next forest
evaluation with a zero time step (that evaluation gives its initial forces, so
joining costs the others no extra pass), steps from the tick after, and leaves
(freeing its memory) at the end of the tick that finishes it.

Host<->device traffic stays off the step path and on the thread that issues
every other CUDA call: submitting a session only queues it. After a tick's
launches, while the device runs that tick, the first lane's thread moves
queued bodies to the device and finished sessions' final states to the host
in slices of a few MB (`Server.pump`, bounded by half the tick's expected
device time), through page-locked buffers allocated once (`PinnedRing`) on a
copy stream. Copies issued from other host threads at the same time as a
lane's launches (pageable or pinned) held those launches up for tens to
hundreds of milliseconds on the B200 boxes measured.

Latency: a session's step latency is the wall-clock interval between the ends
of its consecutive steps; every step should take at most `latency_slo` times
the step latency of the same session run alone. At start-up the server
calibrates, for Plummer and uniform-cube systems of 1e3 .. 1e6 bodies, the
isolated step latency and the extra latency of a second system of the same
size in the same forest. A session is admitted only if the batch's latency
predicted with it -- the batch's last measured step latency plus the session's
calibrated extra latency (the larger of the two system types) -- stays within
`headroom` times the isolated latency (the smaller of the two types) of the
batch's smallest session, and only while the lane's recent steps stay within
that bound (feedback against prediction error). A tick in which sessions join
a running batch is a step interval of the sessions already stepping, so it
measures the prediction: its ratio to the prediction (kept >= 1, decaying as
sessions finish) scales later predictions, and if it took longer than
`headroom` times the isolated latency of the batch's smallest session, the
sessions that joined in it -- which have not stepped yet, so nothing of theirs
changes -- go back to the front of the queue and wait for a session of the
lane to finish before they are tried again. A running batch in which a session
has already had a step over `latency_slo` times its isolated latency takes no
more joins (its p99 allows one such step in a hundred). Sessions that start
together in an empty lane are bounded by the model alone (their joining tick, with the
one-time costs of joining, is no session's step). Only the first session of an
empty lane may join before the background copies have put its bodies on the
device. The queue is scanned in arrival
order and sessions that fit may overtake ones that do not, except a session
that has waited longer than `max_bypass_s`: nobody overtakes it, save the
sessions that start together with an older one in an empty lane (their steps
end with that session's, so they keep the waiting one out no longer). Waiting
time is reported apart from the step latency.

By default there is one lane. Several lanes (`lanes`: lower bounds of N) run
concurrently on streams of decreasing priority for increasing N; they share
the GPU block by block, so each lane's ticks stretch by the others' work --
more throughput at low load, weaker latency bounds.

Every session's bodies, velocities and last accelerations stay resident on the
device between its steps. No reference counterpart (the reference has no
serving component).
"""

from __future__ import annotations

import dataclasses
import sys
import threading
import time
from collections import deque

import numpy as np

# Device bytes per body kept resident (pos, vel, acc, pot, mass, dt: 12 FP64) and
# the engine's working memory per body of a forest evaluation (tree, expansions,
# lists) at p=8, leaf 64 with headroom; plus a fixed part per session.
RESIDENT_BYTES_PER_BODY = 96
ENGINE_BYTES_PER_BODY = 640
SESSION_FIXED_BYTES = 1 << 20
STAGED_BYTES_PER_BODY = 56  # pos, vel, mass staged on the device while queued
SMALL_POOL_RESERVE = 256 << 20  # small-block pool reserved per stream (blocks <= 1 MB)
ARENA_PLAN_SHARE = 0.8  # share of the staging arena that background staging may plan

# Size classes (lower bounds of N) of the lanes: one lane by default.
LANE_BOUNDS = (0,)
# Sizes at which the latencies are calibrated.
CALIBRATION_N = (1_000, 3_000, 10_000, 30_000, 100_000, 300_000, 1_000_000)


@dataclasses.dataclass(eq=False)  # sessions compare by identity
class Session:
    sid: int
    mass: np.ndarray
    pos: np.ndarray
    vel: np.ndarray
    steps: int
    dt: float
    arrival: float = 0.0
    # filled by the server (times are perf_counter seconds)
    submitted_at: float | None = None
    admitted_at: float | None = None
    finished_at: float | None = None
    steps_done: int = 0
    primed: bool = False
    last_end: float = 0.0  # end of its last step (or of its joining tick)
    retry_after: int = -1  # after a failed join: the lane's departure count it must wait past
    step_ms: list = dataclasses.field(default_factory=list)
    result_pos: np.ndarray | None = None
    result_vel: np.ndarray | None = None
    staged: tuple | None = dataclasses.field(default=None, repr=False)  # device pos, vel, mass, ready event
    pending: tuple | None = dataclasses.field(default=None, repr=False)  # result copy job, host pos, host vel
    stage_job: object | None = dataclasses.field(default=None, repr=False)  # staging in progress
    planned: bool = False  # counted in the staging budget (queued for staging, staging, or staged)
    slow_steps: int = 0  # steps that took longer than latency_slo times its isolated latency
    stage_region: tuple | None = dataclasses.field(default=None, repr=False)  # (offset, bytes) in the arena

    @property
    def n(self) -> int:
        return len(self.mass)

    def bytes_needed(self) -> int:
        return self.n * (RESIDENT_BYTES_PER_BODY + ENGINE_BYTES_PER_BODY) + SESSION_FIXED_BYTES

    def fresh(self) -> "Session":
        """The same request, not yet served."""
        return dataclasses.replace(self, submitted_at=None, admitted_at=None, finished_at=None, steps_done=0,
                                   primed=False, last_end=0.0, retry_after=-1, step_ms=[], result_pos=None,
                                   result_vel=None, staged=None, pending=None, stage_job=None, planned=False,
                                   stage_region=None, slow_steps=0)


def _interp_loglog(ns, vals, n):
    ln = np.log(np.asarray(ns, dtype=np.float64))
    lv = np.log(np.maximum(np.asarray(vals, dtype=np.float64), 1e-4))
    x = np.log(max(float(n), 1.0))
    if x >= ln[-1] and len(ln) > 1:
        slope = max((lv[-1] - lv[-2]) / (ln[-1] - ln[-2]), 0.0)
        return float(np.exp(lv[-1] + slope * (x - ln[-1])))
    return float(np.exp(np.interp(x, ln, lv)))


class DeviceArena:
    """First-fit allocator over one device buffer allocated at start-up. The
    bodies of queued sessions are staged here, so staging never calls the
    caching allocator, which on a busy device fell back to cudaMalloc (or
    freed cached segments, synchronising the device) and held the lane's
    thread for 100-150 ms. A region given back is reused once the event
    recorded with it (after the last read of the region) has completed."""

    ALIGN = 256

    def __init__(self, torch, dev, nbytes):
        self.size = int(nbytes)
        self.buf = torch.empty(self.size, dtype=torch.uint8, device=dev) if self.size > 0 else None
        self.free = [(0, self.size)] if self.size > 0 else []  # (offset, bytes), by offset
        self.pending = []  # (event, offset, bytes)
        self.lock = threading.Lock()

    def _put(self, off, size):
        fr = self.free
        i = 0
        while i < len(fr) and fr[i][0] < off:
            i += 1
        fr.insert(i, (off, size))
        if i + 1 < len(fr) and fr[i][0] + fr[i][1] == fr[i + 1][0]:  # merge with the next
            fr[i] = (off, fr[i][1] + fr[i + 1][1])
            del fr[i + 1]
        if i > 0 and fr[i - 1][0] + fr[i - 1][1] == fr[i][0]:  # and with the previous
            fr[i - 1] = (fr[i - 1][0], fr[i - 1][1] + fr[i][1])
            del fr[i]

    def alloc(self, nbytes):
        """(offset, bytes) of a free region of at least nbytes, or None."""
        nb = -(-int(nbytes) // self.ALIGN) * self.ALIGN
        with self.lock:
            keep = []
            for ev, off, size in self.pending:
                if ev is None or ev.query():
                    self._put(off, size)
                else:
                    keep.append((ev, off, size))
            self.pending = keep
            for i, (off, size) in enumerate(self.free):
                if size >= nb:
                    if size == nb:
                        del self.free[i]
                    else:
                        self.free[i] = (off + nb, size - nb)
                    return off, nb
        return None

    def release(self, region, event=None):
        with self.lock:
            self.pending.append((event, region[0], region[1]))


class CopyJob:
    """A host<->device copy done in chunks: parts of (host uint8 view, device
    uint8 view), all in one direction."""

    def __init__(self, parts, to_device: bool):
        self.parts = [(h, d) for h, d in parts if h.size > 0]
        self.to_device = to_device
        self.i = 0
        self.off = 0
        self.lock = threading.Lock()

    @property
    def done(self) -> bool:
        return self.i >= len(self.parts)


class PinnedRing:
    """Page-locked host buffers, allocated once, through which copy jobs move
    chunk by chunk on a given stream: host-to-device double-buffered (the host
    fills one buffer while the other's DMA runs), device-to-host one chunk at
    a time."""

    def __init__(self, torch, chunk_bytes=4 << 20):
        self.torch = torch
        self.chunk = int(chunk_bytes)
        self.up = [torch.empty(self.chunk, dtype=torch.uint8, pin_memory=True) for _ in range(2)]
        self.up_np = [b.numpy() for b in self.up]
        self.up_ev = [None, None]
        self.up_next = 0
        self.down = torch.empty(self.chunk, dtype=torch.uint8, pin_memory=True)
        self.down_np = self.down.numpy()
        self.lock = threading.Lock()

    def advance(self, job: CopyJob, stream) -> bool:
        """Move one chunk of `job` on `stream`; True once the job is complete
        (host-to-device: queued on the stream; device-to-host: on the host)."""
        torch = self.torch
        with job.lock, self.lock, torch.cuda.stream(stream):
            if job.done:
                return True
            h, d = job.parts[job.i]
            m = min(self.chunk, h.size - job.off)
            sl = slice(job.off, job.off + m)
            if job.to_device:
                k = self.up_next
                self.up_next ^= 1
                if self.up_ev[k] is not None:
                    self.up_ev[k].synchronize()  # this buffer's previous DMA is done
                np.copyto(self.up_np[k][:m], h[sl])
                d[sl].copy_(self.up[k][:m], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(stream)
                self.up_ev[k] = ev
            else:
                self.down[:m].copy_(d[sl], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(stream)
                ev.synchronize()
                np.copyto(h[sl], self.down_np[:m])
            job.off += m
            if job.off >= h.size:
                job.i += 1
                job.off = 0
            return job.done

    def finish(self, job: CopyJob, stream):
        while not self.advance(job, stream):
            pass


def _u8(a):
    """uint8 view of a contiguous host array or device tensor."""
    if isinstance(a, np.ndarray):
        return a.reshape(-1).view(np.uint8)
    import torch

    return a.reshape(-1).view(torch.uint8)


class LatencyModel:
    """Calibrated step latencies (ms) against N: `iso(n)` the isolated step
    latency, `extra(n)` the added latency of one more system of n bodies in a
    forest. Log-log interpolation, extrapolated with the end slope."""

    def __init__(self, ns, iso_ms, extra_ms):
        self.ns = [int(n) for n in ns]
        self.iso_ms = [float(v) for v in np.maximum.accumulate(np.asarray(iso_ms, dtype=np.float64))]
        self.extra_ms = [max(float(v), 1e-3) for v in np.maximum.accumulate(np.asarray(extra_ms, dtype=np.float64))]

    def iso(self, n) -> float:
        return _interp_loglog(self.ns, self.iso_ms, n)

    def extra(self, n) -> float:
        return _interp_loglog(self.ns, self.extra_ms, n)

    def table(self):
        return [[n, round(a, 3), round(b, 3)] for n, a, b in zip(self.ns, self.iso_ms, self.extra_ms)]


# Fields of a lane's per-tick trace record: perf_counter seconds at the tick's
# start, after admission and joins, after the step's launches, after the device
# finished it, and at the tick's end (departures done); then its device time
# (ms), members, bodies, sessions joined, joins undone and departures; then the
# times inside the launch phase after the first kick and drift, after the
# forest build and after the evaluation.
TICK_FIELDS = ("t_start", "t_joined", "t_launched", "t_synced", "t_end", "device_ms", "members", "bodies",
               "joined", "undone", "left", "t_kick_drift", "t_built", "t_evaluated")


def worst_intervals(trace, k=8, copies=()):
    """The k longest intervals between consecutive tick ends of a lane, each
    split into its host phases: idle gap before the tick, admission and joins,
    launches, wait for the device, departures (ms); with `copies` (a server's
    copy log), the staging and result copy time that overlapped the interval."""
    out = []
    tr = list(trace)
    cp = list(copies)
    for a, b in zip(tr, tr[1:]):
        out.append({"interval_ms": 1e3 * (b[4] - a[4]), "gap_ms": 1e3 * (b[0] - a[4]), "join_ms": 1e3 * (b[1] - b[0]),
                    "launch_ms": 1e3 * (b[2] - b[1]), "sync_ms": 1e3 * (b[3] - b[2]), "leave_ms": 1e3 * (b[4] - b[3]),
                    "device_ms": b[5], "members": b[6], "bodies": b[7], "joined": b[8], "undone": b[9],
                    "left": b[10], "_t": (a[4], b[4]), "kick_drift_ms": 1e3 * (b[11] - b[1]),
                    "build_ms": 1e3 * (b[12] - b[11]), "evaluate_ms": 1e3 * (b[13] - b[12]),
                    "last_kick_ms": 1e3 * (b[2] - b[13])})
    out.sort(key=lambda r: -r["interval_ms"])
    out = out[:k]
    for r in out:
        t0, t1 = r.pop("_t")
        r["copy_overlap_ms"] = 1e3 * sum(max(0.0, min(c[1], t1) - max(c[0], t0)) for c in cp)
        r["copies"] = [[c[2], round(1e3 * (c[0] - t0), 2), round(1e3 * (c[1] - c[0]), 2), round(c[3] / 1e6, 2)]
                       for c in cp if c[1] > t0 and c[0] < t1][:12]
    return [{k2: (round(v, 3) if isinstance(v, float) else v) for k2, v in r.items()} for r in out[:k]]


class Lane:
    """One size class: its own context and stream, continuous batching."""

    def __init__(self, server: "Server", lo: int, priority: int = 0, preemptible: bool = False):
        torch = server.torch
        self.srv = server
        self.lo = lo
        self.priority = priority
        self.stream = torch.cuda.Stream(device=server.device, priority=priority)
        self.fmm = server.fx.Fmm(None, None, server.p, 0.0, server.n_leaf, mac="theta", theta=server.theta,
                                 softening=server.softening, precision=server.precision, device=server.device,
                                 stream=self.stream.cuda_stream, preemptible=preemptible)
        self.queue: deque[Session] = deque()
        self.members: list[Session] = []  # primed (stepping) and joining sessions, in row order
        self.state = None  # pos, vel, acc, pot, mass of the members (device)
        self.dts = None  # per-row time step of the members; 0 for rows joining this tick
        self.tick_ms: list[float] = []  # device time of each tick
        self.last_interval_ms = None  # wall interval of the last tick that stepped sessions
        self.predicted_ms = None  # predicted interval after the last admission, until measured
        self.corr = 1.0  # >= 1: measured over predicted latency of recent joining ticks
        self.recent_ratio: deque[float] = deque(maxlen=8)
        self.bodies_stepped = 0
        self.departures = 0  # sessions finished in this lane
        self.evictions = 0  # joins undone because the joining tick broke the bound
        self.t_built = 0.0
        self.forest_dirty = True  # the members changed since the forest was built
        self.ticks_on_tree = 0  # ticks stepped on the current forest's tree and lists
        # one record per tick (TickRecord fields), for latency analysis
        self.trace: deque[tuple] = deque(maxlen=1 << 17)

    # ---------------------------------------------------------------- helpers
    @staticmethod
    def offsets(sessions):
        return np.concatenate([[0], np.cumsum([s.n for s in sessions])]).astype(np.uint64)

    @property
    def stepping(self):
        return [s for s in self.members if s.primed]

    def bodies(self):
        return sum(s.n for s in self.members)

    # ---------------------------------------------------------------- admission
    def admit(self, now):
        srv = self.srv
        model = srv.model
        new = []
        if not srv.gate_open(self):
            return new
        if model is not None and any(m.slow_steps for m in self.members):
            # a join stretches the tick it happens in; a session's p99 step
            # latency allows one such step in a hundred, so a batch one of
            # whose sessions already had a slow step takes no more joins
            return new
        # predicted step latency of the batch as it stands, and its smallest member
        tau = self.predicted_ms if self.predicted_ms is not None else self.last_interval_ms
        nmin = min((s.n for s in self.members), default=None)
        was_empty = not self.members
        for s in list(self.queue)[: srv.scan]:
            pred = None
            fits = s.retry_after < self.departures
            if fits and (new or self.members) and s.staged is None:
                # only the first session of an empty lane joins before its
                # bodies are on the device: a copy inside a tick would stretch
                # every member's step
                fits = False
            if fits and model is not None and nmin is not None:
                pred = (tau if tau is not None else model.iso(nmin)) + model.extra(s.n)
                fits = pred * self.corr <= srv.headroom * model.iso(min(nmin, s.n))
            if fits and srv.reserve(s.bytes_needed()):
                self.queue.remove(s)
                s.admitted_at = now
                new.append(s)
                if model is not None:
                    tau = model.iso(s.n) if pred is None else pred
                nmin = s.n if nmin is None else min(nmin, s.n)
                continue
            if model is None or (s.submitted_at is not None and now - s.submitted_at > srv.max_bypass_s):
                if model is not None and was_empty and new:
                    # the lane was empty and the oldest session has just been
                    # admitted: sessions that fit beside it start with it (the
                    # batch ends no later for them), and the one that does not
                    # fit heads the next batch
                    continue
                break  # first come, first served from this session on
        if new and model is not None:
            self.predicted_ms = tau
        return new

    def join(self, new):
        """Append the new sessions' rows with a zero time step."""
        if not new:
            return
        torch = self.srv.torch
        for s in new:
            if s.staged is None:
                self.srv.stage_now(s)
            self.stream.wait_event(s.staged[3])
        pos = torch.cat([s.staged[0] for s in new])
        vel = torch.cat([s.staged[1] for s in new])
        mass = torch.cat([s.staged[2] for s in new])
        done = torch.cuda.Event()
        done.record(self.stream)  # after the copies out of the staged buffers
        for s in new:
            if s.stage_region is not None:
                self.srv.arena.release(s.stage_region, done)
                s.stage_region = None
            else:
                for t in s.staged[:3]:
                    t.record_stream(self.stream)
            s.staged = None
        self.srv.unstage(sum(s.n for s in new))
        acc = torch.zeros_like(pos)
        pot = torch.zeros_like(mass)
        rows = [pos, vel, acc, pot, mass]
        self.state = rows if self.state is None else [torch.cat([a, b]) for a, b in zip(self.state, rows)]
        self.members.extend(new)
        self.forest_dirty = True
        self._set_dts()

    def _set_dts(self):
        torch = self.srv.torch
        if not self.members:
            self.dts = None
            return
        d = np.concatenate([np.full(s.n, s.dt if s.primed else 0.0) for s in self.members])
        self.dts = torch.from_numpy(d).to(self.srv.dev)[:, None]

    def evict(self, sessions):
        """Undo the join of sessions that have not stepped: drop their rows and
        put them back at the front of the queue until a session finishes."""
        torch = self.srv.torch
        out = set(id(s) for s in sessions)
        keep, rows = [], []
        off = self.offsets(self.members)
        for i, s in enumerate(self.members):
            if id(s) not in out:
                keep.append(s)
                rows.append(torch.arange(int(off[i]), int(off[i + 1]), device=self.srv.dev))
        idx = torch.cat(rows)
        self.state = [t.index_select(0, idx) for t in self.state]
        self.members = keep
        for s in reversed(sessions):
            s.admitted_at = None
            s.retry_after = self.departures
            s.planned = False  # its device copy went into the lane's rows: staged again before a retry
            self.srv.release(s.bytes_needed())
            self.queue.appendleft(s)
        self.evictions += len(sessions)
        self.predicted_ms = None
        self.forest_dirty = True
        self._set_dts()

    def leave(self, now):
        torch = self.srv.torch
        keep, rows, out = [], [], []
        off = self.offsets(self.members)
        pos, vel = self.state[0], self.state[1]
        for i, s in enumerate(self.members):
            a, b = int(off[i]), int(off[i + 1])
            if s.steps_done >= s.steps:
                out.append((s, pos[a:b].clone(), vel[a:b].clone()))
            else:
                keep.append(s)
                rows.append(torch.arange(a, b, device=self.srv.dev))
        self.departures += len(out)
        for _ in out:  # the learned under-prediction of joins fades as sessions finish
            self.corr = max(1.0, 0.9 * self.corr)
        for s, p, v in out:
            ev = torch.cuda.Event()
            ev.record(self.stream)
            self.srv.copy_stream.wait_event(ev)  # the copies read what this tick wrote
            hp, hv = np.empty((s.n, 3)), np.empty((s.n, 3))
            s.pending = (CopyJob([(_u8(hp), _u8(p)), (_u8(hv), _u8(v))], to_device=False), hp, hv)
            s.finished_at = now
            self.srv.release(s.bytes_needed())
            self.srv.finished(s)
        changed = bool(out)
        self.members = keep
        if not keep:
            self.state = None
            self.dts = None
            self.recent_ratio.clear()
            self.last_interval_ms = None
            self.predicted_ms = None
            return changed
        if changed:
            idx = torch.cat(rows)
            self.state = [t.index_select(0, idx) for t in self.state]
            self.forest_dirty = True
        return changed

    # ---------------------------------------------------------------- one tick
    def tick(self) -> float:
        torch = self.srv.torch
        t_start = time.perf_counter()
        with torch.cuda.stream(self.stream):
            new = self.admit(time.perf_counter())
            self.join(new)
            if not self.members:
                return 0.0
            t_joined = time.perf_counter()
            stepping = self.stepping
            pos, vel, acc, pot, mass = self.state
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(self.stream)
            # one engine call: kick and drift with per-row time steps (0 for
            # joining rows), the forest build -- over the new members when they
            # changed, else every refresh_every ticks, in between the tree and
            # lists are reused -- the evaluation and the closing kick
            rebuild = self.forest_dirty or self.ticks_on_tree + 1 >= self.srv.refresh_every
            offsets = self.offsets(self.members) if self.forest_dirty else None
            t_kd = time.perf_counter()
            self.fmm.kdk_step_device(pos.data_ptr(), vel.data_ptr(), mass.data_ptr(), acc.data_ptr(),
                                     pot.data_ptr(), self.dts.data_ptr(), offsets, rebuild)
            self.t_built = t_kd
            self.forest_dirty = False
            self.ticks_on_tree = 0 if rebuild else self.ticks_on_tree + 1
            t_ev = time.perf_counter()
            t_launched = time.perf_counter()
            e1.record(self.stream)
            if self.srv.lanes[0] is self:
                # copies in the shadow of this tick's device time
                expect = self.tick_ms[-1] if self.tick_ms else 1.0
                self.srv.pump(0.5e-3 * expect)
            e1.synchronize()
            t_end = time.perf_counter()
            ms = e0.elapsed_time(e1)
            n_members, n_bodies, ev0, dep0 = len(self.members), self.bodies(), self.evictions, self.departures
            self.tick_ms.append(ms)
            for s in stepping:
                s.steps_done += 1
                s.step_ms.append(1e3 * (t_end - s.last_end))
                s.last_end = t_end
                self.bodies_stepped += s.n
                if self.srv.model is not None and self.srv.latency_slo is not None and \
                        s.step_ms[-1] > self.srv.latency_slo * self.srv.model.iso(s.n):
                    s.slow_steps += 1
            predicted = self.predicted_ms
            if stepping:
                self.last_interval_ms = max(s.step_ms[-1] for s in stepping)
                self.predicted_ms = None
                if self.srv.model is not None:
                    self.recent_ratio.append(max(s.step_ms[-1] / self.srv.model.iso(s.n) for s in stepping))
            joined = [s for s in self.members if not s.primed]
            model = self.srv.model
            if predicted and stepping and not joined and model is not None:
                # the first step of a batch started in an empty lane: learn
                # from its prediction as from a join
                self.corr = min(4.0, max(1.0, 0.9 * self.corr, self.last_interval_ms / predicted))
            if joined and model is not None and stepping:
                # a join into a running batch: this tick is a step interval of
                # the sessions already stepping. Learn how far the model
                # under-predicts joins (decaying toward 1), and undo the join
                # if the tick broke the bound. (A batch started in an empty
                # lane is bounded by the model alone: its joining tick, with
                # the one-time costs of joining, is no session's step.)
                if predicted:
                    seen = 1e3 * (t_end - t_start) / predicted
                    self.corr = min(4.0, max(1.0, 0.9 * self.corr, seen))
                ratio = 1e3 * (t_end - t_start) / model.iso(min(s.n for s in self.members))
                undo = joined
                if ratio > self.srv.headroom and undo:
                    self.evict(undo)
                    joined = [s for s in joined if s not in undo]
            for s in joined:
                s.primed = True
                s.last_end = t_end
            changed = self.leave(time.perf_counter())
            if joined or changed:
                self._set_dts()
            self.trace.append((t_start, t_joined, t_launched, t_end, time.perf_counter(), ms, n_members, n_bodies,
                               len(new), self.evictions - ev0, self.departures - dep0, t_kd, self.t_built, t_ev))
            return ms


class Server:
    """Front end: HBM and latency admission, routing to lanes, synchronous or
    threaded driving.

    latency_slo: target ratio of a step's latency to the session's isolated
    step latency; None turns latency admission off (first come, first served
    under the HBM budget only).
    headroom: the bound used for admission decisions (below latency_slo, to
    leave room for prediction error).
    stage_limit_bytes: device bytes of queued sessions' bodies staged ahead of
    their admission (sessions beyond it are staged when they join); the
    staging arena, allocated at start-up, holds stage_limit_bytes /
    ARENA_PLAN_SHARE.
    lane_reserve_bytes: allocator pool reserved on each lane's stream.
    refresh_every: a lane's forest is rebuilt whenever its members change and
    otherwise every refresh_every ticks; in between the tree and interaction
    lists are reused (1, the default: every tick, which keeps each session's
    result bitwise the one it gets alone; above 1 a session's rebuild times
    depend on its neighbours' arrivals and departures).
    """

    def __init__(self, *, p=8, theta=0.5, softening=1e-3, n_leaf=64, precision="mixed", budget_bytes=160e9,
                 lanes=LANE_BOUNDS, device=0, latency_slo=None, headroom=None, model=None, max_bypass_s=2.0,
                 scan=256, stage_limit_bytes=8e9, lane_reserve_bytes=2e9, refresh_every=1):
        import torch

        import fmms_b200 as fx

        self.torch = torch
        self.fx = fx
        self.device = device
        self.dev = f"cuda:{device}"
        torch.cuda.set_device(device)
        self.p, self.theta, self.softening, self.n_leaf, self.precision = p, theta, softening, n_leaf, precision
        self.refresh_every = max(1, int(refresh_every))
        self.budget = float(budget_bytes)
        self.used = 0.0
        self.staged_bytes = 0.0
        self.stage_limit = float(stage_limit_bytes)
        self.lock = threading.Lock()
        self.latency_slo = latency_slo
        self.headroom = headroom if headroom is not None else (0.8 * latency_slo if latency_slo else None)
        self.max_bypass_s = max_bypass_s
        self.scan = scan
        self.copy_stream = torch.cuda.Stream(device=device)
        self.ring = PinnedRing(torch)
        self.copy_lock = threading.RLock()  # one copy activity at a time (several lanes may join)
        self.to_stage: deque[Session] = deque()  # submitted, not staged, within the staging limit
        self.staging: Session | None = None  # the session being staged
        self.results: deque[Session] = deque()  # finished, final state still to copy
        # (start, end, kind, bytes) of every staging and result copy, perf_counter seconds
        self.copy_log: deque[tuple] = deque(maxlen=1 << 16)
        bounds = tuple(sorted(lanes))
        try:
            least, greatest = torch.cuda.Stream.priority_range()
        except Exception:  # noqa: BLE001 - no priorities: every lane at the default
            least, greatest = 0, 0
        self.lanes = []
        for i, lo in enumerate(bounds):
            prio = max(greatest, least - (len(bounds) - 1 - i)) if greatest < least else least
            # with several lanes, short M2L blocks let the higher-priority lanes in
            self.lanes.append(Lane(self, lo, prio, preemptible=len(bounds) > 1))
        # Staged bodies live in the arena. The lanes' own allocations (joins,
        # kicks, departures) come from the caching allocator's pools, one per
        # stream and size class (blocks up to 1 MB are carved from 2 MB
        # segments, larger ones from their own): reserve both up front
        # (allocate and free once), so that they do not reach cudaMalloc,
        # which was seen to take ~90 ms at times on a busy device, even for a
        # 2 MB segment.
        # staging ahead fills the arena up to ARENA_PLAN_SHARE of it: the rest
        # is for sessions that join before their background copy began
        self.arena = DeviceArena(torch, self.dev, self.stage_limit / ARENA_PLAN_SHARE)
        for st, nbytes in [(ln.stream, lane_reserve_bytes) for ln in self.lanes]:
            if nbytes > 0:
                with torch.cuda.stream(st):
                    blk = torch.empty(int(nbytes), dtype=torch.uint8, device=self.dev)
                    small = [torch.empty(1 << 20, dtype=torch.uint8, device=self.dev)
                             for _ in range(int(min(nbytes, SMALL_POOL_RESERVE)) >> 20)]
                    del blk, small
        self.done: list[Session] = []
        self.outstanding = 0
        self._threads = []
        self._stop = threading.Event()
        self._switch = None
        self.error: BaseException | None = None  # first exception of a lane thread
        self.model = None
        if latency_slo is not None:
            self.model = model if model is not None else self.calibrate()

    # -------------------------------------------------------------- calibration
    def _run_batch(self, sessions):
        """Run sessions to completion as one batch in the lane of the first
        (synchronously); the median step latency without the first two steps
        (which may grow the lane's buffers)."""
        ln = self.lane_for(sessions[0])
        assert not ln.members and not ln.queue
        for s in sessions:
            self.submit(s, lane=ln)
        while ln.members or ln.queue:
            ln.tick()
        self.collect(sessions)
        for s in sessions:
            self.done.remove(s)
        return float(np.median(sessions[0].step_ms[2:]))

    def calibrate(self, ns=CALIBRATION_N, steps=5) -> LatencyModel:
        """Isolated step latency and the extra latency of a second system of
        the same size, for Plummer and uniform-cube systems of each size."""
        iso, extra = [], []
        for i, n in enumerate(ns):
            iso_t, ext_t = [], []
            for kind in ("plummer", "uniform"):
                pair = []
                for j in range(2):
                    seed = 90_000 + 10 * i + j
                    if kind == "plummer":
                        mass, pos, vel = self.fx.gen_plummer_ic(int(n), 1.0, 1.0, 20.0, seed)
                    else:
                        mass, pos = self.fx.gen_uniform_lognormal(int(n), 0.5, seed)
                        vel = np.zeros_like(pos)
                    pair.append(Session(sid=-1, mass=mass, pos=pos, vel=vel, steps=steps, dt=1e-3))
                one = self._run_batch([pair[0]])
                two = self._run_batch([pair[0].fresh(), pair[1]])
                iso_t.append(one)
                ext_t.append(two - one)
            iso.append(min(iso_t))
            extra.append(max(ext_t))
        for ln in self.lanes:
            ln.tick_ms.clear()
            ln.trace.clear()
            ln.bodies_stepped = 0
        return LatencyModel(ns, iso, extra)

    # -------------------------------------------------------------- memory
    def reserve(self, nbytes) -> bool:
        with self.lock:
            if self.used + nbytes > self.budget:
                return False
            self.used += nbytes
            return True

    def release(self, nbytes):
        with self.lock:
            self.used -= nbytes

    def mem_used(self) -> float:
        return self.used

    def _start_staging(self, s: Session, wait: bool = False) -> bool:
        """Place the session's device buffers (in the arena; with wait, from
        the caching allocator when the arena has no room) and prepare the
        copy; False if there is no room now."""
        torch = self.torch
        t0 = time.perf_counter()
        n = s.n
        region = self.arena.alloc(STAGED_BYTES_PER_BODY * n)
        if region is not None:
            seg = self.arena.buf[region[0]:region[0] + STAGED_BYTES_PER_BODY * n]
            dev = [seg[:24 * n].view(torch.float64).view(n, 3), seg[24 * n:48 * n].view(torch.float64).view(n, 3),
                   seg[48 * n:56 * n].view(torch.float64)]
            s.stage_region = region
        elif wait:
            with torch.cuda.stream(self.copy_stream):
                dev = [torch.empty(tuple(np.shape(a)), dtype=torch.float64, device=self.dev)
                       for a in (s.pos, s.vel, s.mass)]
        else:
            return False
        self.copy_log.append((t0, time.perf_counter(), "alloc", n * STAGED_BYTES_PER_BODY))
        host = [_u8(np.ascontiguousarray(a, dtype=np.float64)) for a in (s.pos, s.vel, s.mass)]
        s.stage_job = (CopyJob([(h, _u8(d)) for h, d in zip(host, dev)], to_device=True), dev, time.perf_counter())
        return True

    def _end_staging(self, s: Session):
        torch = self.torch
        job, dev, t0 = s.stage_job
        ev = torch.cuda.Event()
        ev.record(self.copy_stream)
        s.staged = (dev[0], dev[1], dev[2], ev)
        s.stage_job = None
        self.copy_log.append((t0, time.perf_counter(), "stage", s.n * STAGED_BYTES_PER_BODY))

    def stage_now(self, s: Session):
        """Stage a joining session's bodies completely (it was not staged in
        the background, or only in part)."""
        with self.copy_lock:
            self._stage_now(s)

    def _stage_now(self, s: Session):
        with self.lock:
            if self.staging is s:
                self.staging = None
            elif s in self.to_stage:
                self.to_stage.remove(s)
            else:
                self.staged_bytes += s.n * STAGED_BYTES_PER_BODY
                s.planned = True
        if s.stage_job is None:
            self._start_staging(s, wait=True)
        self.ring.finish(s.stage_job[0], self.copy_stream)
        self._end_staging(s)

    def unstage(self, n_bodies):
        """Give back staging budget, and plan the staging of queued sessions
        that did not fit in it when they were submitted (in queue order)."""
        with self.lock:
            self.staged_bytes -= n_bodies * STAGED_BYTES_PER_BODY
            for ln in self.lanes:
                for s in list(ln.queue)[: self.scan]:
                    if s.planned:
                        continue
                    nb = s.n * STAGED_BYTES_PER_BODY
                    if self.staged_bytes + nb > self.stage_limit:
                        break
                    self.staged_bytes += nb
                    s.planned = True
                    self.to_stage.append(s)

    def pump(self, budget_s: float) -> bool:
        """Result copies first, then staging, one chunk at a time, for about
        `budget_s` seconds (at least one chunk when there is work); False if
        there was nothing to copy."""
        t_end = time.perf_counter() + budget_s
        while True:
            with self.copy_lock:
                if not self._pump_one():
                    return False
            if time.perf_counter() >= t_end:
                return True

    def _pump_one(self) -> bool:
        """One chunk of the oldest result copy, else of the staging in
        progress (starting the next one if none is); False if idle."""
        if self.results:
            s = self.results[0]
            if self.ring.advance(s.pending[0], self.copy_stream):
                self._finish_result(s)
            return True
        with self.lock:
            s = self.staging
            if s is None and self.to_stage:
                s = self.staging = self.to_stage.popleft()
        if s is None:
            return False
        if s.staged is None:
            if s.stage_job is None and not self._start_staging(s):
                with self.lock:  # no room in the arena yet: retry once a region comes back
                    if self.staging is s:
                        self.staging = None
                        self.to_stage.appendleft(s)
                return False
            if not self.ring.advance(s.stage_job[0], self.copy_stream):
                return True
            self._end_staging(s)
        with self.lock:
            if self.staging is s:
                self.staging = None
        return True

    def _finish_result(self, s: Session):
        job, hp, hv = s.pending
        s.result_pos, s.result_vel = hp, hv
        s.pending = None
        if self.results and self.results[0] is s:
            self.results.popleft()
        self.copy_log.append((s.finished_at, time.perf_counter(), "collect", 48 * s.n))

    def collect(self, sessions=None):
        """Finish the final-state copies of finished sessions (all of them, or
        of `sessions`)."""
        with self.copy_lock:
            self._collect(sessions)

    def _collect(self, sessions):
        for s in list(self.results if sessions is None else sessions):
            if s.pending is not None:
                self.ring.finish(s.pending[0], self.copy_stream)
                self._finish_result(s)
                if s in self.results:
                    self.results.remove(s)

    def finished(self, s):
        with self.lock:
            self.done.append(s)
            self.results.append(s)
            self.outstanding -= 1

    def busy(self) -> bool:
        """Sessions submitted and not finished (queued, joining or stepping);
        False once a lane thread has failed (`stop` raises its exception)."""
        return self.outstanding > 0 and self.error is None

    def gate_open(self, lane) -> bool:
        """Admission feedback: the lane's recent steps within the headroom."""
        if self.model is None:
            return True
        return not lane.recent_ratio or max(lane.recent_ratio) <= self.headroom

    # -------------------------------------------------------------- routing
    def lane_for(self, s: Session) -> Lane:
        lane = self.lanes[0]
        for ln in self.lanes:
            if s.n >= ln.lo:
                lane = ln
        return lane

    def submit(self, s: Session, lane=None):
        """Queue a session (any thread; no CUDA call here)."""
        s.submitted_at = time.perf_counter()
        with self.lock:
            if self.staged_bytes + s.n * STAGED_BYTES_PER_BODY <= self.stage_limit:
                self.staged_bytes += s.n * STAGED_BYTES_PER_BODY
                s.planned = True
                self.to_stage.append(s)
            self.outstanding += 1
            (lane or self.lane_for(s)).queue.append(s)

    @property
    def active(self):
        return [s for ln in self.lanes for s in ln.members]

    @property
    def queue(self):
        return [s for ln in self.lanes for s in ln.queue]

    # -------------------------------------------------------------- driving
    def tick(self):
        """Synchronous mode: one tick of every lane that has work."""
        for ln in self.lanes:
            if ln.members or ln.queue:
                ln.tick()

    def run_until_idle(self, max_ticks=1 << 30):
        t = 0
        while self.busy() and t < max_ticks:
            self.tick()
            if not any(ln.members for ln in self.lanes):
                self.pump(0.001)  # admission waits on staging: keep it moving
            t += 1
        self.collect()

    def start(self):
        """Threaded mode: every lane ticks on its own host thread and stream."""

        def loop(ln):
            try:
                self.torch.cuda.set_device(self.device)
                while not self._stop.is_set():
                    if ln.members or ln.queue:
                        ln.tick()
                    if not ln.members:  # idle, or admission refused: copy, else do not spin on the GIL
                        if not (ln is self.lanes[0] and self.pump(0.001)):
                            time.sleep(0.0005)
            except BaseException as e:  # noqa: BLE001 - handed to the caller by stop()
                with self.lock:
                    if self.error is None:
                        self.error = e
                self._stop.set()  # the other lanes stop too

        # lane threads hand the interpreter lock to each other and to the
        # submitting thread between short pieces of host work; the default 5 ms
        # switch interval would add up to that much to a step
        self._switch = sys.getswitchinterval()
        sys.setswitchinterval(2e-4)
        for ln in self.lanes:
            th = threading.Thread(target=loop, args=(ln,), daemon=True)
            th.start()
            self._threads.append(th)

    def stop(self):
        """Stop the lane threads and finish the result copies of the sessions
        that completed; then raise the first exception a lane thread met, if
        any. The error is cleared as it is raised, so the server can be
        started again (sessions that were active on the failed lane stay in
        ``active`` and are not resumed)."""
        self._stop.set()
        for th in self._threads:
            th.join()
        self._threads = []
        self._stop.clear()
        if self._switch is not None:
            sys.setswitchinterval(self._switch)
            self._switch = None
        err, self.error = self.error, None
        try:
            self.collect()
        finally:
            if err is not None:
                raise RuntimeError("serving lane failed") from err

    def report(self) -> dict:
        sess = self.done + self.active
        lat = np.array([m for s in sess for m in s.step_ms]) if sess else np.array([0.0])
        waits = np.array([1e3 * (s.admitted_at - s.submitted_at) for s in sess
                          if s.admitted_at is not None and s.submitted_at is not None])
        busy = max((sum(ln.tick_ms) for ln in self.lanes), default=0.0) * 1e-3
        stepped = sum(ln.bodies_stepped for ln in self.lanes)
        out = {"sessions_done": len(self.done), "ticks": sum(len(ln.tick_ms) for ln in self.lanes),
               "step_ms_p50": float(np.percentile(lat, 50)), "step_ms_p99": float(np.percentile(lat, 99)),
               "bodies_stepped": stepped, "lane_busy_s_max": busy}
        if len(waits):
            out["admission_wait_ms_p50"] = float(np.percentile(waits, 50))
            out["admission_wait_ms_p99"] = float(np.percentile(waits, 99))
        if self.model is not None:
            out["latency_slo"] = self.latency_slo
            out["headroom"] = self.headroom
            out["calibration_n_iso_extra_ms"] = self.model.table()
        return out


def run_session_alone(sess: Session, **kw) -> tuple[np.ndarray, np.ndarray, list]:
    """The same session through its own server, for alone-vs-mix checks."""
    kw = {k: v for k, v in kw.items() if k not in ("latency_slo", "headroom", "model")}
    kw.setdefault("stage_limit_bytes", 0)  # one session: staged when it joins, no pools reserved
    kw.setdefault("lane_reserve_bytes", 0)
    srv = Server(**kw)
    srv.submit(sess.fresh())
    srv.run_until_idle()
    d = srv.done[0]
    return d.result_pos, d.result_vel, d.step_ms
