"""Serving loop: continuous batching of leapfrog sessions (fmms_b200.serve).

Each session's trajectory must be the same alone and in the mix (the forest
evaluation and the elementwise updates are per session), sessions arriving
while others run must join at the next tick, and admission must respect the
memory budget."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def make_sessions():
    import fmms_b200 as fx
    from fmms_b200.serve import Session

    out = []
    for i, (n, steps) in enumerate([(3000, 7), (20000, 4), (1200, 9), (8000, 5)]):
        if i % 2 == 0:
            mass, pos, vel = fx.gen_plummer_ic(n, 1.0, 1.0, 20.0, 50 + i)
        else:
            mass, pos = fx.gen_uniform_lognormal(n, 0.5, 60 + i)
            vel = np.zeros_like(pos)
        out.append(Session(sid=i, mass=mass, pos=pos, vel=vel, steps=steps, dt=1e-3))
    return out


def test_sessions_same_alone_and_in_the_mix():
    from fmms_b200.serve import Server, run_session_alone

    kw = dict(p=8, theta=0.5, softening=1e-3, n_leaf=64, precision="mixed")
    sess = make_sessions()
    srv = Server(**kw)
    srv.submit(sess[0])
    srv.submit(sess[1])
    srv.tick()
    srv.tick()
    srv.submit(sess[2])  # arrives while the first two are running
    srv.tick()
    srv.submit(sess[3])
    srv.run_until_idle()
    assert len(srv.done) == 4
    for s in srv.done:
        assert s.steps_done == s.steps
        pos, vel, _ = run_session_alone(s, **kw)
        assert np.array_equal(s.result_pos, pos), s.sid
        assert np.array_equal(s.result_vel, vel), s.sid


def test_admission_respects_budget():
    from fmms_b200.serve import Server

    sess = make_sessions()
    budget = sess[1].bytes_needed() + sess[0].bytes_needed() // 2  # room for one big session at a time
    srv = Server(p=6, theta=0.5, softening=1e-3, n_leaf=64, precision="mixed", budget_bytes=budget)
    for s in sess:
        srv.submit(s)
    peak = 0.0
    while srv.active or srv.queue:
        srv.tick()
        peak = max(peak, srv.mem_used())
        assert srv.mem_used() <= budget
    assert len(srv.done) == 4 and peak > 0


def test_forest_tree_reuse_in_serving():
    """refresh_every 3: a lane keeps its forest's tree and lists for up to 3
    ticks while its members do not change. Each session's trajectory stays
    within the FMM's force error of the one it gets alone (their rebuild times
    differ), and every session completes its steps."""
    from fmms_b200.serve import Server, run_session_alone

    kw = dict(p=8, theta=0.5, softening=1e-3, n_leaf=64, precision="mixed", refresh_every=3)
    sess = make_sessions()
    srv = Server(**kw)
    for s in sess:
        srv.submit(s)
    srv.run_until_idle()
    assert len(srv.done) == len(sess)
    for s in srv.done:
        assert len(s.step_ms) == s.steps
        pa, va, _ = run_session_alone(s, **kw)
        scale = np.abs(pa).max()
        assert np.max(np.abs(s.result_pos - pa)) < 1e-7 * scale
