"""Failure paths made on the host, with no GPU fault: a device-memory budget
that the inputs exceed (FMMX_OVER_BUDGET, the reference GPU backend's
OverBudget, crates/visual/src/gpufmm.rs:1653-1672), walk buffers too small
for the walk (the overflow-and-retry path), and corrupted ensemble offsets.
After each failure the context stays usable and gives the same bits as a
context that never failed."""

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

OVER_BUDGET, INVALID_ARG = 3, 1


def fx():
    import fmms_b200

    return fmms_b200


def test_over_budget_then_recovers():
    mass_big, pos_big = fx().gen_plummer(200_000, seed=3)
    mass, pos = fx().gen_plummer(2048, seed=4)
    kw = dict(mac="theta", theta=0.5, softening=1e-3)
    g = fx().Fmm(None, None, 6, 0.0, 16, device_budget_bytes=8 << 20, **kw)
    with pytest.raises(fx().FmmError) as e:
        g.refresh(mass_big, pos_big)
    assert e.value.status == OVER_BUDGET
    assert "budget 8.0 MiB" in str(e.value)
    assert g.stats()["device_bytes"] <= 8 << 20
    g.refresh(mass, pos)  # the same context, a system that fits
    r = g.run()
    ref = fx().Fmm(mass, pos, 6, 0.0, 16, **kw).run()
    assert np.array_equal(r.accel, ref.accel) and np.array_equal(r.pot, ref.pot)
    assert g.stats()["device_bytes"] <= 8 << 20


def test_over_budget_in_evaluate():
    """A budget that holds the tree but not the walk and expansions: the
    evaluation fails with OVER_BUDGET, a smaller system then runs."""
    mass, pos = fx().gen_plummer(100_000, seed=5)
    probe = fx().Fmm(mass, pos, 8, 1e-5, 16)
    after_build = probe.stats()["device_bytes"]
    probe.run()
    after_eval = probe.stats()["device_bytes"]
    probe.close()
    assert after_eval > after_build
    g = fx().Fmm(None, None, 8, 1e-5, 16, device_budget_bytes=(after_build + after_eval) // 2)
    g.refresh(mass, pos)
    with pytest.raises(fx().FmmError) as e:
        g.run()
    assert e.value.status == OVER_BUDGET
    m2, p2 = fx().gen_plummer(1000, seed=6)
    g.refresh(m2, p2)
    r = g.run()
    ref = fx().Fmm(m2, p2, 8, 1e-5, 16).run()
    assert np.array_equal(r.accel, ref.accel)


def test_walk_overflow_retry_gives_the_same_bits(monkeypatch):
    """Walk buffers of 64 pairs (FMMX_TEST_WALK_CAPACITY): the walk overflows
    and is redone with larger buffers until it fits; the lists, and so every
    result bit, are those of a context sized for the tree."""
    mass, pos, _ = fx().gen_plummer_ic(30_000, 1.0, 1.0, 20.0, 8)
    kw = dict(mac="theta", theta=0.5, softening=1e-3)
    for precision in ("plain", "mixed"):
        ref = fx().Fmm(mass, pos, 8, 0.0, 32, precision=precision, **kw)
        r0 = ref.run()
        monkeypatch.setenv("FMMX_TEST_WALK_CAPACITY", "64")
        g = fx().Fmm(mass, pos, 8, 0.0, 32, precision=precision, **kw)
        monkeypatch.delenv("FMMX_TEST_WALK_CAPACITY")
        r1 = g.run()
        assert g.stats()["walk_retries"] > ref.stats()["walk_retries"]
        assert np.array_equal(r0.accel, r1.accel) and np.array_equal(r0.pot, r1.pot)
        assert g.stats()["n_m2l"] == ref.stats()["n_m2l"] and g.stats()["n_p2p"] == ref.stats()["n_p2p"]


def test_corrupted_ensemble_offsets():
    m1, p1 = fx().gen_plummer(3000, seed=1)
    m2, p2 = fx().gen_plummer(2000, seed=2)
    mass, pos = np.concatenate([m1, m2]), np.concatenate([p1, p2])
    g = fx().Fmm(None, None, 6, 1e-4, 16)
    bad = [np.array([1, 3000, 5000], dtype=np.uint64),  # does not start at 0
           np.array([0, 3000, 3000, 5000], dtype=np.uint64),  # an empty system
           np.array([0, 4000, 3000, 5000], dtype=np.uint64)]  # decreasing
    for off in bad:
        with pytest.raises(fx().FmmError) as e:
            g.build_ensemble(off, mass, pos)
        assert e.value.status == INVALID_ARG
    g.build_ensemble(np.array([0, 3000, 5000], dtype=np.uint64), mass, pos)
    r = g.run()
    alone = fx().Fmm(m1, p1, 6, 1e-4, 16).run()
    assert np.array_equal(r.accel[:3000], alone.accel)
