"""Host-side logic of the serving loop, without a GPU: the latency model's
interpolation, the admission rule (latency bound, HBM reservation, overtaking
limit) on lanes stood in for by plain objects, and the per-tick trace
analysis. The serving loop has no reference counterpart; the GPU behaviour
(batched forests bitwise equal to sessions run alone) is in
test_gpu_serve.py."""

from collections import deque
from types import SimpleNamespace

import numpy as np
import pytest

from fmms_b200.serve import TICK_FIELDS, DeviceArena, Lane, LatencyModel, Session, worst_intervals


def session(sid, n, submitted_at=0.0, staged=True):
    s = Session(sid=sid, mass=np.zeros(n), pos=np.zeros((n, 3)), vel=np.zeros((n, 3)), steps=10, dt=1e-3)
    s.submitted_at = submitted_at
    if staged:  # bodies already copied to the device (a stand-in for the tensors and event)
        s.staged = (None, None, None, None)
        s.planned = True
    return s


class LinearModel:
    """iso(n) = 1 ms + n / 1e5 ms, extra(n) = n / 1e5 ms."""

    def iso(self, n):
        return 1.0 + n / 1e5

    def extra(self, n):
        return n / 1e5


def fake_lane(queue, members=(), reserve=lambda b: True, model=None, max_bypass_s=2.0, gate=True):
    srv = SimpleNamespace(model=model if model is not None else LinearModel(), headroom=1.6, scan=256,
                          max_bypass_s=max_bypass_s, gate_open=lambda lane: gate, reserve=reserve)
    return SimpleNamespace(srv=srv, queue=deque(queue), members=list(members), predicted_ms=None,
                           last_interval_ms=None, corr=1.0, departures=0)


def test_latency_model_loglog():
    m = LatencyModel([1e3, 1e4, 1e5], [1.0, 2.0, 8.0], [0.1, 0.5, 4.0])
    assert m.iso(1e3) == pytest.approx(1.0) and m.iso(1e5) == pytest.approx(8.0)
    assert m.iso(np.sqrt(1e3 * 1e4)) == pytest.approx(np.sqrt(2.0))  # geometric midpoint
    assert m.iso(1e6) == pytest.approx(32.0)  # end slope (4x per decade) extrapolated
    assert m.iso(10) == pytest.approx(1.0)  # below the table: its first value
    # calibrations that come out non-monotone are made monotone
    m2 = LatencyModel([1e3, 1e4], [2.0, 1.5], [0.2, 0.1])
    assert m2.iso_ms == [2.0, 2.0] and m2.extra_ms == [0.2, 0.2]


def test_admission_latency_bound_and_overtaking():
    small1, small2, big, small3 = session(0, 1000), session(1, 2000), session(2, 1_000_000), session(3, 3000)
    ln = fake_lane([small1, small2, big, small3])
    new = Lane.admit(ln, now=1.0)
    # empty lane: the first is admitted on its isolated latency; each next one
    # while tau + extra(n) stays within 1.6 iso(smallest); the big one would
    # break the bound (1.03 + 10 > 1.6 * 1.01) and the small one behind it
    # overtakes it (it has waited less than max_bypass_s)
    assert new == [small1, small2, small3]
    assert list(ln.queue) == [big]
    assert ln.predicted_ms == pytest.approx(1.01 + 0.02 + 0.03)
    assert all(s.admitted_at == 1.0 for s in new)


def test_admission_no_overtaking_past_a_long_wait():
    member = session(9, 1000)
    small1, big, small2 = session(0, 1000), session(1, 1_000_000, submitted_at=0.0), session(2, 1000)
    ln = fake_lane([small1, big, small2], members=[member], max_bypass_s=2.0)
    ln.last_interval_ms = 1.01
    new = Lane.admit(ln, now=5.0)  # big has waited 5 s > 2 s: nobody passes it while the lane runs
    assert new == [small1] and list(ln.queue) == [big, small2]


def test_admission_fresh_batch_takes_sessions_that_fit_past_a_long_wait():
    """In an empty lane the oldest session starts a batch; sessions that fit
    beside it start with it even past one that has waited long, which heads
    the next batch (their steps end together, so it waits no longer)."""
    small1, big, small2 = session(0, 1000), session(1, 1_000_000, submitted_at=0.0), session(2, 1000)
    ln = fake_lane([small1, big, small2], max_bypass_s=2.0)
    assert Lane.admit(ln, now=5.0) == [small1, small2]
    assert list(ln.queue) == [big]
    ln2 = fake_lane([big, small1, small2], max_bypass_s=2.0)
    assert Lane.admit(ln2, now=5.0) == [big]  # 10.01 + 0.01 > 1.6 * iso(1000)
    assert list(ln2.queue) == [small1, small2]


def test_admission_followers_must_be_staged():
    """Only the first session of an empty lane may join before its bodies
    are on the device; an unstaged one is passed over, not waited for."""
    head, cold, warm = session(0, 1000, staged=False), session(1, 1000, staged=False), session(2, 1000)
    ln = fake_lane([head, cold, warm])
    assert Lane.admit(ln, now=1.0) == [head, warm]
    assert list(ln.queue) == [cold]
    member = session(9, 1000)
    ln2 = fake_lane([session(3, 1000, staged=False)], members=[member])
    ln2.last_interval_ms = 1.01
    assert Lane.admit(ln2, now=1.0) == []


def test_unstage_plans_queued_sessions_in_order():
    """Staging budget given back goes to queued sessions that did not fit in
    it when they were submitted, in queue order, up to the limit."""
    import threading

    from fmms_b200.serve import STAGED_BYTES_PER_BODY, Server

    a, b, c = session(0, 1000, staged=False), session(1, 2000, staged=False), session(2, 500, staged=False)
    lane = SimpleNamespace(queue=deque([a, b, c]))
    srv = SimpleNamespace(lock=threading.Lock(), lanes=[lane], scan=256, to_stage=deque(),
                          stage_limit=2500 * STAGED_BYTES_PER_BODY, staged_bytes=2000 * STAGED_BYTES_PER_BODY)
    Server.unstage(srv, 1000)  # 1000 bodies' worth left in use, room for 1500 more
    assert list(srv.to_stage) == [a] and a.planned and not b.planned and not c.planned
    assert srv.staged_bytes == 2000 * STAGED_BYTES_PER_BODY


def test_admission_hbm_reservation_and_gate():
    a, b = session(0, 1000), session(1, 1000)
    budget = {"left": a.bytes_needed()}

    def reserve(nbytes):
        if nbytes > budget["left"]:
            return False
        budget["left"] -= nbytes
        return True

    ln = fake_lane([a, b], reserve=reserve)
    assert Lane.admit(ln, now=0.5) == [a]
    assert list(ln.queue) == [b]
    closed = fake_lane([session(2, 1000)], gate=False)  # recent steps over the bound
    assert Lane.admit(closed, now=0.5) == [] and len(closed.queue) == 1


def test_admission_waits_for_a_departure_after_an_undone_join():
    s = session(0, 1000)
    s.retry_after = 3  # evicted when the lane had seen 3 departures
    ln = fake_lane([s])
    ln.departures = 3
    assert Lane.admit(ln, now=0.1) == []
    ln.departures = 4
    assert Lane.admit(ln, now=0.1) == [s]


def test_admission_scales_prediction_by_learned_correction():
    member = session(0, 10_000)
    joiner = session(1, 10_000)
    ln = fake_lane([joiner], members=[member])
    ln.last_interval_ms = 1.1  # iso(1e4) = 1.1, extra = 0.1: 1.2 <= 1.6 * 1.1
    assert Lane.admit(ln, now=0.0) == [joiner]
    ln2 = fake_lane([session(2, 10_000)], members=[member])
    ln2.last_interval_ms = 1.1
    ln2.corr = 1.5  # joins were under-predicted: 1.2 * 1.5 > 1.76
    assert Lane.admit(ln2, now=0.0) == []


def test_worst_intervals_split_and_copy_overlap():
    assert len(TICK_FIELDS) == 14

    def rec(t0, join, kd, built, ev, launched, synced, end, dev_ms):
        # TICK_FIELDS order: start, joined, launched, synced, end, device_ms, members, bodies, joined,
        # undone, left, kick_drift, built, evaluated
        return (t0, join, launched, synced, end, dev_ms, 1, 1000, 0, 0, 0, kd, built, ev)

    tr = [rec(0.000, 0.0001, 0.0002, 0.0005, 0.0010, 0.0011, 0.0020, 0.0021, 1.0),
          rec(0.0025, 0.0026, 0.0027, 0.0030, 0.0900, 0.0901, 0.0950, 0.0951, 92.0),
          rec(0.0960, 0.0961, 0.0962, 0.0965, 0.0970, 0.0971, 0.0980, 0.0981, 1.0)]
    copies = [(0.0028, 0.0400, "stage", 5e6), (0.2, 0.3, "collect", 1e6)]
    w = worst_intervals(tr, k=2, copies=copies)
    assert len(w) == 2
    top = w[0]
    assert top["interval_ms"] == pytest.approx(93.0)
    assert top["gap_ms"] == pytest.approx(0.4)
    assert top["evaluate_ms"] == pytest.approx(87.0)  # the stalled call
    assert top["build_ms"] == pytest.approx(0.3)
    assert top["device_ms"] == 92.0
    assert top["copy_overlap_ms"] == pytest.approx(37.2)
    assert top["copies"] == [["stage", pytest.approx(0.7), pytest.approx(37.2), 5.0]]
    assert w[1]["interval_ms"] == pytest.approx(3.0) and w[1]["copy_overlap_ms"] == 0.0


def test_arena_first_fit_reuse_and_coalescing():
    """The staging arena hands out 256-byte aligned regions first fit, reuses
    a region only once its event has completed, and merges neighbours."""
    import torch

    class Ev:
        def __init__(self, done):
            self.done = done

        def query(self):
            return self.done

    a = DeviceArena(torch, "cpu", 4096)
    r1, r2, r3 = a.alloc(1000), a.alloc(1024), a.alloc(2000)
    assert r1 == (0, 1024) and r2 == (1024, 1024) and r3 == (2048, 2048)
    assert a.alloc(1) is None  # full
    pending = Ev(False)
    a.release(r2, pending)
    assert a.alloc(256) is None  # the reader of r2 has not finished
    pending.done = True
    assert a.alloc(256) == (1024, 256)
    a.release((1024, 256))
    a.release(r1)
    a.release(r3)
    assert a.alloc(4096) == (0, 4096)  # all merged back into one region


def test_admission_no_joins_after_a_slow_step():
    """A session's p99 step latency allows one slow step in a hundred: a
    running batch one of whose sessions already had a step over the latency
    target takes no more joins (they would stretch another of its steps)."""
    member = session(9, 1000)
    member.slow_steps = 1
    ln = fake_lane([session(0, 1000)], members=[member])
    ln.last_interval_ms = 1.01
    assert Lane.admit(ln, now=0.0) == []
    member.slow_steps = 0
    assert len(Lane.admit(ln, now=0.0)) == 1
