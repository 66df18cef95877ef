"""Batched ensemble (forest mode): many independent systems in one build and
one evaluation. Every system's result must be the one it gets alone, and the
plain form must still match the oracle system by system."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def systems():
    import fmms_b200 as fx

    parts = []
    for i, n in enumerate([1000, 4096, 1, 2, 7777, 300]):
        if n < 3:
            mass = np.full(n, 1.0 / n)
            pos = np.random.default_rng(i).random((n, 3)) + 10 * i
        elif i % 2:
            mass, pos, _ = fx.gen_plummer_ic(n, 1.0, 0.5 + 0.3 * i, 20.0, 100 + i)
        else:
            mass, pos = fx.gen_uniform_lognormal(n, 0.5, 200 + i)
            pos = pos * (i + 1) - 3.0
        parts.append((mass, pos))
    off = np.concatenate([[0], np.cumsum([len(m) for m, _ in parts])]).astype(np.uint64)
    return parts, off


@pytest.mark.parametrize("precision", ["plain", "mixed"])
def test_ensemble_equals_each_system_alone(precision):
    import fmms_b200 as fx

    parts, off = systems()
    mass = np.concatenate([m for m, _ in parts])
    pos = np.concatenate([p for _, p in parts])
    kw = dict(mac="theta", theta=0.5, softening=1e-3, precision=precision)
    g = fx.Fmm(None, None, 8, 0.0, 32, **kw)
    g.build_ensemble(off, mass, pos)
    res = g.run()
    assert g.stats()["n_cells"] >= len(parts)
    for s, (m, p) in enumerate(parts):
        alone = fx.Fmm(m, p, 8, 0.0, 32, **kw).run()
        a, b = int(off[s]), int(off[s + 1])
        assert np.array_equal(res.accel[a:b], alone.accel), s
        assert np.array_equal(res.pot[a:b], alone.pot), s


def test_ensemble_plain_matches_oracle(orc):
    import fmms_b200 as fx

    parts, off = systems()
    mass = np.concatenate([m for m, _ in parts])
    pos = np.concatenate([p for _, p in parts])
    g = fx.Fmm(None, None, 6, 1e-5, 16)
    g.build_ensemble(off, mass, pos)
    res = g.run()
    for s, (m, p) in enumerate(parts):
        a, b = int(off[s]), int(off[s + 1])
        acc_o, pot_o = orc.Fmm(m, p, 6, 1e-5, 16).run()
        rel = np.linalg.norm(res.accel[a:b] - acc_o, axis=1) / np.maximum(np.linalg.norm(acc_o, axis=1), 1e-300)
        if len(m) > 1:
            assert rel.max() < 1e-12, (s, rel.max())
        else:
            assert np.all(res.accel[a:b] == 0)


def test_ensemble_rejects_empty_system():
    import fmms_b200 as fx

    g = fx.Fmm(None, None, 4, 1e-3, 16)
    with pytest.raises(fx.FmmError):
        g.build_ensemble(np.array([0, 5, 5, 9], dtype=np.uint64), np.ones(9), np.random.default_rng(0).random((9, 3)))
