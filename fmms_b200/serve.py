"""Serving loop: continuous batching of leapfrog sessions on one GPU.

Sessions are N-body systems integrated with kick-drift-kick leapfrog. They
arrive at any time, wait in a queue, and are admitted when the HBM budget and
the per-tick work cap allow. Every admitted session's bodies, velocities and
last accelerations stay resident on the device. Each tick advances every
active session by one step: the half kicks and drifts of all sessions are one
elementwise pass over their concatenated state, and their force evaluations
are batched into ONE forest build + evaluation (fmmx_build_ensemble_device):
one tree per session, no interaction across sessions, each session's result
bitwise the one it gets alone. Sessions that finish leave at the end of the
tick and free their memory; queued sessions join the next tick, so requests
that arrive while others are on the GPU share its work.

No reference counterpart (the reference has no serving component).
"""

from __future__ import annotations

import dataclasses
import time
from collections import deque

import numpy as np

# Device bytes per body kept resident (pos, vel, acc, pot, mass: 11 FP64) and the
# engine's working memory per body of a forest evaluation (tree, expansions,
# lists), measured on p=8, leaf 64 workloads with headroom; plus a fixed part.
RESIDENT_BYTES_PER_BODY = 88
ENGINE_BYTES_PER_BODY = 640
SESSION_FIXED_BYTES = 1 << 20


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


class Server:
    """Continuous-batching server over one engine context in forest mode."""

    def __init__(self, *, p=8, theta=0.5, softening=1e-3, n_leaf=64, precision="mixed", budget_bytes=160e9,
                 max_active_bodies=1 << 22, device=0):
        import torch

        import fmms_b200 as fx

        self.torch = torch
        self.fx = fx
        self.dev = f"cuda:{device}"
        torch.cuda.set_device(device)
        self.stream = torch.cuda.current_stream()
        self.fmm = fx.Fmm(None, None, p, 0.0, n_leaf, mac="theta", theta=theta, softening=softening,
                          precision=precision, device=device, stream=self.stream.cuda_stream)
        self.budget = float(budget_bytes)
        self.max_active_bodies = int(max_active_bodies)
        self.queue: deque[Session] = deque()
        self.active: list[Session] = []
        self.done: list[Session] = []
        self.tick_ms: list[float] = []
        self.bodies_stepped = 0
        self._state = None  # (pos, vel, acc, pot, mass) device tensors of the active sessions

    # -------------------------------------------------------------- admission
    def submit(self, s: Session):
        self.queue.append(s)

    def mem_used(self) -> float:
        return float(sum(s.bytes_needed() for s in self.active))

    def _admit(self, now: float) -> list[Session]:
        new = []
        bodies = sum(s.n for s in self.active)
        used = self.mem_used()
        while self.queue:
            s = self.queue[0]
            if used + s.bytes_needed() > self.budget:
                break
            if self.active or new:
                if bodies + s.n > self.max_active_bodies:
                    break
            self.queue.popleft()
            s.admitted_at = now
            new.append(s)
            used += s.bytes_needed()
            bodies += s.n
        return new

    # ------------------------------------------------------------------ state
    def _offsets(self, sessions):
        return np.concatenate([[0], np.cumsum([s.n for s in sessions])]).astype(np.uint64)

    def _evaluate(self, pos, mass, acc, pot, offsets):
        self.fmm.build_ensemble_device(offsets, pos.data_ptr(), mass.data_ptr())
        self.fmm.evaluate_device(pos.data_ptr(), mass.data_ptr(), acc.data_ptr(), pot.data_ptr())

    def _join(self, new: list[Session]):
        """Add admitted sessions: upload their state and evaluate their initial
        accelerations (all new sessions in one forest)."""
        torch = self.torch
        if not new:
            return
        pos = torch.from_numpy(np.concatenate([s.pos for s in new])).to(self.dev)
        vel = torch.from_numpy(np.concatenate([s.vel for s in new])).to(self.dev)
        mass = torch.from_numpy(np.concatenate([s.mass for s in new])).to(self.dev)
        acc = torch.empty_like(pos)
        pot = torch.empty_like(mass)
        self._evaluate(pos, mass, acc, pot, self._offsets(new))
        if self._state is None:
            self._state = [pos, vel, acc, pot, mass]
        else:
            self._state = [torch.cat([a, b]) for a, b in zip(self._state, [pos, vel, acc, pot, mass])]
        self.active.extend(new)

    def _leave(self, now: float):
        torch = self.torch
        keep, rows = [], []
        off = self._offsets(self.active)
        pos, vel = self._state[0], self._state[1]
        for i, s in enumerate(self.active):
            a, b = int(off[i]), int(off[i + 1])
            if s.steps_done >= s.steps:
                s.result_pos = pos[a:b].cpu().numpy()
                s.result_vel = vel[a:b].cpu().numpy()
                s.finished_at = now
                self.done.append(s)
            else:
                keep.append(s)
                rows.append(torch.arange(a, b, device=self.dev))
        self.active = keep
        if not keep:
            self._state = None
            return
        idx = torch.cat(rows)
        self._state = [t.index_select(0, idx) for t in self._state]

    # ------------------------------------------------------------------- tick
    def tick(self, now: float | None = None) -> float:
        """Admit, advance every active session by one KDK step, retire the
        finished ones. Returns the tick's device time in ms."""
        torch = self.torch
        now = time.perf_counter() if now is None else now
        self._join(self._admit(now))
        if not self.active:
            return 0.0
        pos, vel, acc, pot, mass = self._state
        # one dt per session, expanded to its bodies
        dts = torch.from_numpy(np.concatenate([np.full(s.n, s.dt) for s in self.active])).to(self.dev)[:, None]
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(self.stream)
        vel.add_(0.5 * dts * acc)
        pos.add_(dts * vel)
        self._evaluate(pos, mass, acc, pot, self._offsets(self.active))
        vel.add_(0.5 * dts * acc)
        e1.record(self.stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        self.tick_ms.append(ms)
        for s in self.active:
            s.steps_done += 1
            s.step_ms.append(ms)
            self.bodies_stepped += s.n
        self._leave(time.perf_counter())
        return ms

    def run_until_idle(self, max_ticks=1 << 30):
        t = 0
        while (self.active or self.queue) and t < max_ticks:
            self.tick()
            t += 1

    def report(self) -> dict:
        lat = np.array([m for s in self.done + self.active for m in s.step_ms]) if self.done or self.active else np.array([0.0])
        busy = sum(self.tick_ms) * 1e-3
        return {"sessions_done": len(self.done), "ticks": len(self.tick_ms),
                "step_ms_p50": float(np.percentile(lat, 50)), "step_ms_p99": float(np.percentile(lat, 99)),
                "bodies_per_s": self.bodies_stepped / busy if busy > 0 else 0.0}


def run_session_alone(sess: Session, **kw) -> tuple[np.ndarray, np.ndarray, list]:
    """The same session through its own server, for alone-vs-mix checks."""
    srv = Server(**kw)
    srv.submit(dataclasses.replace(sess, step_ms=[], steps_done=0, result_pos=None, result_vel=None))
    srv.run_until_idle()
    d = srv.done[0]
    return d.result_pos, d.result_vel, d.step_ms
