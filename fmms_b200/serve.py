"""Serving loop: continuous batching of leapfrog sessions on one GPU.

Sessions are N-body systems integrated with kick-drift-kick leapfrog. They
arrive at any time, wait in a queue, and are admitted when the HBM budget
allows. Admitted sessions are routed by size to lanes. A lane owns an engine
context, a CUDA stream and (in threaded mode) a host thread, and advances its
sessions one step per tick: the half kicks and drifts of all its sessions are
one elementwise pass over their concatenated state, and their force
evaluations are batched into ONE forest build + evaluation
(fmmx_build_ensemble_device) -- one tree per session, no interaction across
sessions, each session's result bitwise the one it gets alone. Sessions join a
lane at its next tick and leave (freeing their memory) at the end of the tick
that finishes them, so requests arriving while others run share the GPU. Lanes
run concurrently on their own streams, so small sessions never wait behind the
evaluation of large ones; within a lane the batch is capped so that a tick
stays close to twice the isolated step time of its smallest session.

Every session's bodies, velocities and last accelerations stay resident on the
device between its steps. No reference counterpart (the reference has no
serving component).
"""

from __future__ import annotations

import dataclasses
import threading
import time
from collections import deque

import numpy as np

# Device bytes per body kept resident (pos, vel, acc, pot, mass: 11 FP64) and the
# engine's working memory per body of a forest evaluation (tree, expansions,
# lists) at p=8, leaf 64 with headroom; plus a fixed part per session.
RESIDENT_BYTES_PER_BODY = 88
ENGINE_BYTES_PER_BODY = 640
SESSION_FIXED_BYTES = 1 << 20

# Size classes (lower bounds) of the lanes, and the batch cap of a lane:
# a tick costs about T0 + B / RATE for B bodies, an isolated step of the
# smallest member T0 + n_min / RATE, so B <= T0 * RATE + 2 n_min keeps the tick
# within twice that isolated step.
LANE_BOUNDS = (0, 4_000, 16_000, 64_000, 256_000)
T0_RATE_BODIES = 60_000


@dataclasses.dataclass
class Session:
    sid: int
    mass: np.ndarray
    pos: np.ndarray
    vel: np.ndarray
    steps: int
    dt: float
    arrival: float = 0.0
    # filled by the server
    admitted_at: float | None = None
    finished_at: float | None = None
    steps_done: int = 0
    step_ms: list = dataclasses.field(default_factory=list)
    result_pos: np.ndarray | None = None
    result_vel: np.ndarray | None = None

    @property
    def n(self) -> int:
        return len(self.mass)

    def bytes_needed(self) -> int:
        return self.n * (RESIDENT_BYTES_PER_BODY + ENGINE_BYTES_PER_BODY) + SESSION_FIXED_BYTES


class Lane:
    """One size class: its own context and stream, continuous batching."""

    def __init__(self, server: "Server", lo: int, cap_bodies: int):
        torch = server.torch
        self.srv = server
        self.lo = lo
        self.cap = cap_bodies
        self.stream = torch.cuda.Stream(device=server.device)
        self.fmm = server.fx.Fmm(None, None, server.p, 0.0, server.n_leaf, mac="theta", theta=server.theta,
                                 softening=server.softening, precision=server.precision, device=server.device,
                                 stream=self.stream.cuda_stream)
        self.queue: deque[Session] = deque()
        self.active: list[Session] = []
        self.state = None  # pos, vel, acc, pot, mass of the active sessions (device)
        self.tick_ms: list[float] = []
        self.bodies_stepped = 0

    def offsets(self, sessions):
        return np.concatenate([[0], np.cumsum([s.n for s in sessions])]).astype(np.uint64)

    def evaluate(self, pos, mass, acc, pot, offsets):
        self.fmm.build_ensemble_device(offsets, pos.data_ptr(), mass.data_ptr())
        self.fmm.evaluate_device(pos.data_ptr(), mass.data_ptr(), acc.data_ptr(), pot.data_ptr())

    def admit(self, now):
        new = []
        bodies = sum(s.n for s in self.active)
        while self.queue:
            s = self.queue[0]
            if (self.active or new) and bodies + s.n > self.cap:
                break
            if not self.srv.reserve(s.bytes_needed()):
                break
            self.queue.popleft()
            s.admitted_at = now
            new.append(s)
            bodies += s.n
        return new

    def join(self, new):
        torch = self.srv.torch
        if not new:
            return
        dev = self.srv.dev
        pos = torch.from_numpy(np.concatenate([s.pos for s in new])).to(dev, non_blocking=False)
        vel = torch.from_numpy(np.concatenate([s.vel for s in new])).to(dev)
        mass = torch.from_numpy(np.concatenate([s.mass for s in new])).to(dev)
        acc = torch.empty_like(pos)
        pot = torch.empty_like(mass)
        self.evaluate(pos, mass, acc, pot, self.offsets(new))
        if self.state is None:
            self.state = [pos, vel, acc, pot, mass]
        else:
            self.state = [torch.cat([a, b]) for a, b in zip(self.state, [pos, vel, acc, pot, mass])]
        self.active.extend(new)

    def leave(self, now):
        torch = self.srv.torch
        keep, rows = [], []
        off = self.offsets(self.active)
        pos, vel = self.state[0], self.state[1]
        for i, s in enumerate(self.active):
            a, b = int(off[i]), int(off[i + 1])
            if s.steps_done >= s.steps:
                s.result_pos = pos[a:b].cpu().numpy()
                s.result_vel = vel[a:b].cpu().numpy()
                s.finished_at = now
                self.srv.release(s.bytes_needed())
                self.srv.finished(s)
            else:
                keep.append(s)
                rows.append(torch.arange(a, b, device=self.srv.dev))
        self.active = keep
        if not keep:
            self.state = None
            return
        idx = torch.cat(rows)
        self.state = [t.index_select(0, idx) for t in self.state]

    def tick(self) -> float:
        torch = self.srv.torch
        with torch.cuda.stream(self.stream):
            self.join(self.admit(time.perf_counter()))
            if not self.active:
                return 0.0
            pos, vel, acc, pot, mass = self.state
            dts = torch.from_numpy(np.concatenate([np.full(s.n, s.dt) for s in self.active])).to(self.srv.dev)[:, None]
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(self.stream)
            vel.add_(0.5 * dts * acc)
            pos.add_(dts * vel)
            self.evaluate(pos, mass, acc, pot, self.offsets(self.active))
            vel.add_(0.5 * dts * acc)
            e1.record(self.stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            self.tick_ms.append(ms)
            for s in self.active:
                s.steps_done += 1
                s.step_ms.append(ms)
                self.bodies_stepped += s.n
            self.leave(time.perf_counter())
            return ms


class Server:
    """Front end: HBM admission, routing to lanes, synchronous or threaded."""

    def __init__(self, *, p=8, theta=0.5, softening=1e-3, n_leaf=64, precision="mixed", budget_bytes=160e9,
                 lanes=LANE_BOUNDS, device=0, max_active_bodies=None):
        import torch

        import fmms_b200 as fx

        self.torch = torch
        self.fx = fx
        self.device = device
        self.dev = f"cuda:{device}"
        torch.cuda.set_device(device)
        self.p, self.theta, self.softening, self.n_leaf, self.precision = p, theta, softening, n_leaf, precision
        self.budget = float(budget_bytes)
        self.used = 0.0
        self.lock = threading.Lock()
        bounds = tuple(lanes)
        self.lanes = []
        for i, lo in enumerate(bounds):
            cap = T0_RATE_BODIES + 2 * max(lo, 1000)
            if max_active_bodies is not None:
                cap = min(cap, max_active_bodies) if i < len(bounds) - 1 else max(cap, 1)
            self.lanes.append(Lane(self, lo, cap))
        self.done: list[Session] = []
        self._threads = []
        self._stop = threading.Event()

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

    def finished(self, s):
        with self.lock:
            self.done.append(s)

    # -------------------------------------------------------------- routing
    def lane_for(self, s: Session) -> Lane:
        lane = self.lanes[0]
        for ln in self.lanes:
            if s.n >= ln.lo:
                lane = ln
        return lane

    def submit(self, s: Session):
        with self.lock:
            self.lane_for(s).queue.append(s)

    @property
    def active(self):
        return [s for ln in self.lanes for s in ln.active]

    @property
    def queue(self):
        return [s for ln in self.lanes for s in ln.queue]

    # -------------------------------------------------------------- driving
    def tick(self):
        """Synchronous mode: one tick of every lane that has work."""
        for ln in self.lanes:
            if ln.active or ln.queue:
                ln.tick()

    def run_until_idle(self, max_ticks=1 << 30):
        t = 0
        while (self.active or self.queue) and t < max_ticks:
            self.tick()
            t += 1

    def start(self):
        """Threaded mode: every lane ticks on its own host thread and stream."""

        def loop(ln):
            self.torch.cuda.set_device(self.device)
            while not self._stop.is_set():
                if ln.active or ln.queue:
                    ln.tick()
                else:
                    time.sleep(0.0005)

        for ln in self.lanes:
            th = threading.Thread(target=loop, args=(ln,), daemon=True)
            th.start()
            self._threads.append(th)

    def stop(self):
        self._stop.set()
        for th in self._threads:
            th.join()
        self._threads = []
        self._stop.clear()

    def report(self) -> dict:
        sess = self.done + self.active
        lat = np.array([m for s in sess for m in s.step_ms]) if sess else np.array([0.0])
        busy = max((sum(ln.tick_ms) for ln in self.lanes), default=0.0) * 1e-3
        stepped = sum(ln.bodies_stepped for ln in self.lanes)
        return {"sessions_done": len(self.done), "ticks": sum(len(ln.tick_ms) for ln in self.lanes),
                "step_ms_p50": float(np.percentile(lat, 50)), "step_ms_p99": float(np.percentile(lat, 99)),
                "bodies_stepped": stepped, "lane_busy_s_max": busy}


def run_session_alone(sess: Session, **kw) -> tuple[np.ndarray, np.ndarray, list]:
    """The same session through its own server, for alone-vs-mix checks."""
    srv = Server(**kw)
    srv.submit(dataclasses.replace(sess, step_ms=[], steps_done=0, result_pos=None, result_vel=None))
    srv.run_until_idle()
    d = srv.done[0]
    return d.result_pos, d.result_vel, d.step_ms
