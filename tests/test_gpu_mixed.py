"""Mixed-precision form (FP32 expansions and P2P, FP64 centre differences,
MAC and top-level M2M/L2L): accuracy against the FP64 direct sum, and the
same interaction lists as the plain form (the MAC stays FP64)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_err(a, ref):
    return np.linalg.norm(a - ref, axis=1) / np.linalg.norm(ref, axis=1)


def targets(n, k=2048, seed=5):
    return np.sort(np.random.default_rng(seed).choice(n, size=min(k, n), replace=False)).astype(np.uint32)


@pytest.mark.parametrize("p,theta", [(4, 0.5), (8, 0.5), (10, 0.5), (12, 0.4), (14, 0.5), (16, 0.5)])
def test_mixed_accuracy_plummer(p, theta):
    import fmms_b200 as fx

    mass, pos, _ = fx.gen_plummer_ic(32768, seed=11)
    soft = 1e-3
    g = fx.Fmm(mass, pos, p, 0.0, 64, mac="theta", theta=theta, softening=soft, precision="mixed")
    res = g.run()
    t = targets(len(mass))
    a_ref, pot_ref, _ = fx.direct_targets(mass, pos, t, softening=soft)
    e = rel_err(res.accel[t], a_ref)
    plain = fx.Fmm(mass, pos, p, 0.0, 64, mac="theta", theta=theta, softening=soft).run()
    ep = rel_err(plain.accel[t], a_ref)
    # FP32 arithmetic sets a floor near 1e-6; truncation error dominates above it
    assert np.percentile(e, 99) < max(3 * np.percentile(ep, 99), 2e-6), (np.percentile(e, 99), np.percentile(ep, 99))
    assert np.percentile(e, 50) < max(3 * np.percentile(ep, 50), 5e-7)
    pe = np.abs(res.pot[t] - pot_ref) / np.abs(pot_ref)
    pp = np.abs(plain.pot[t] - pot_ref) / np.abs(pot_ref)
    assert np.percentile(pe, 99) < max(3 * np.percentile(pp, 99), 2e-6)


def test_mixed_uniform_cube_lognormal():
    import fmms_b200 as fx

    mass, pos = fx.gen_uniform_lognormal(1 << 17, 0.5, 22)
    g = fx.Fmm(mass, pos, 10, 0.0, 64, mac="theta", theta=0.5, softening=1e-4, precision="mixed")
    res = g.run()
    t = targets(len(mass))
    a_ref, _, _ = fx.direct_targets(mass, pos, t, softening=1e-4)
    e = rel_err(res.accel[t], a_ref)
    assert np.percentile(e, 99) < 1e-5 and np.percentile(e, 50) < 1e-6


def test_mixed_clustered_deep_tree():
    import fmms_b200 as fx

    mass, pos, _ = fx.gen_clusters(1 << 17, 64, 1e-3, 1e-1, 33)
    kw = dict(mac="theta", theta=0.4, softening=1e-5)
    res = fx.Fmm(mass, pos, 12, 0.0, 32, precision="mixed", **kw).run()
    plain = fx.Fmm(mass, pos, 12, 0.0, 32, **kw).run()
    t = targets(len(mass))
    a_ref, _, _ = fx.direct_targets(mass, pos, t, softening=1e-5)
    e = rel_err(res.accel[t], a_ref)
    ep = rel_err(plain.accel[t], a_ref)
    assert np.all(np.isfinite(res.accel))
    # on this 14-level clustered tree the error is truncation, the same in both forms
    assert np.percentile(e, 99) < 1.2 * np.percentile(ep, 99) + 2e-6, (np.percentile(e, 99), np.percentile(ep, 99))
    assert np.percentile(e, 50) < 1e-6


def test_mixed_dehnen_lists_match_plain(orc):
    """With the reference's MAC the mixed form walks the same lists as the
    plain form (bit-exact FP64 MAC inputs), and stays accurate."""
    import fmms_b200 as fx

    mass, pos = orc.plummer(16384, seed=2024)
    gm = fx.Fmm(mass, pos, 8, 1e-6, 16, precision="mixed")
    rm = gm.run()
    gp = fx.Fmm(mass, pos, 8, 1e-6, 16)
    rp = gp.run()
    for a, b in zip(gm.export_lists(), gp.export_lists()):
        sa = np.sort(np.ascontiguousarray(a).view(np.uint64).ravel())
        sb = np.sort(np.ascontiguousarray(b).view(np.uint64).ravel())
        assert np.array_equal(sa, sb)
    e = rel_err(rm.accel, rp.accel)
    assert np.percentile(e, 99) < 2e-6


def test_mixed_full_size_c2():
    """The headline configuration at full size (N = 2^20 uniform cube, log-normal
    masses, softening 1e-4, p = 10, theta 0.5, leaf 64), mixed form: p99 relative
    force error against the FP64 direct sum on 1024 targets below 2e-6, and the
    same interaction lists as the plain form."""
    import fmms_b200 as fx

    mass, pos = fx.gen_uniform_lognormal(1 << 20, 0.5, 22)
    kw = dict(mac="theta", theta=0.5, softening=1e-4)
    g = fx.Fmm(mass, pos, 10, 0.0, 64, precision="mixed", **kw)
    res = g.run()
    t = targets(len(mass), k=1024)
    a_ref, _, _ = fx.direct_targets(mass, pos, t, softening=1e-4)
    e = rel_err(res.accel[t], a_ref)
    assert np.percentile(e, 99) < 2e-6, np.percentile(e, 99)
    h = fx.Fmm(mass, pos, 10, 0.0, 64, **kw)
    h.run()
    for a, b in zip(g.export_lists(), h.export_lists()):
        assert len(a) == len(b)


@pytest.mark.parametrize("tile", [128, 512, 1024])
def test_mixed_p2p_giant_leaf_and_tiles(tile):
    """A leaf far above the leaf capacity (5000 bodies inside a cube of side
    1e-9, below the tree's finest level) next to an ordinary Plummer sphere:
    the near field takes such a leaf as a chunk of its own (more bodies than
    its shared-memory leaf table holds). With tiles of 128, 512 and 1024 bodies the
    mixed form agrees with the plain FP64 form on the same tree and lists to
    the FP32 floor (against the softened direct sum both forms carry the
    unsoftened far field's error next to a unit mass in one point)."""
    import fmms_b200 as fx

    rng = np.random.default_rng(3)
    m1, p1, _ = fx.gen_plummer_ic(6000, seed=12)
    p2 = 0.5 + 1e-9 * rng.random((5000, 3))
    mass = np.concatenate([m1, np.full(5000, 1.0 / 5000)])
    pos = np.concatenate([p1, p2])
    kw = dict(mac="theta", theta=0.5, softening=1e-2)
    g = fx.Fmm(mass, pos, 8, 0.0, 32, precision="mixed", p2p_tile=tile, **kw)
    res = g.run()
    assert g.stats()["n_leaves"] > 1
    ref = fx.Fmm(mass, pos, 8, 0.0, 32, precision="plain", **kw).run()
    assert np.all(np.isfinite(res.accel)) and np.all(np.isfinite(res.pot))
    for part in (slice(0, 6000), slice(6000, 11000)):  # the sphere, the point mass
        e = rel_err(res.accel[part], ref.accel[part])
        assert np.percentile(e, 99) < 1e-5 and np.max(e) < 1e-4, (np.percentile(e, 99), np.max(e))
        pe = np.abs(res.pot[part] - ref.pot[part]) / np.abs(ref.pot[part])
        assert np.max(pe) < 1e-5, np.max(pe)
