"""The benchmark workload generators (no reference counterpart; defined by the
benchmark configurations): the engine's generators give the same bits as the
oracle's independent restatement, and the samples have the properties the
configurations state (truncation radius, distribution-function velocities in
virial balance, log-normal masses, Dirichlet cluster sizes summing to N)."""

import numpy as np
import pytest


def fx():
    import fmms_b200

    return fmms_b200


@pytest.mark.parametrize("seed", [11, 12345])
def test_engine_and_oracle_generators_agree(orc, seed):
    m1, p1, v1 = fx().gen_plummer_ic(20000, 1.0, 1.0, 20.0, seed)
    m2, p2, v2 = orc.gen_plummer_ic(20000, 1.0, 1.0, 20.0, seed)
    assert np.array_equal(m1, m2) and np.array_equal(p1, p2) and np.array_equal(v1, v2)
    m1, p1 = fx().gen_uniform_lognormal(30000, 0.5, seed)
    m2, p2 = orc.gen_uniform_lognormal(30000, 0.5, seed)
    assert np.array_equal(m1, m2) and np.array_equal(p1, p2)
    m1, p1, v1 = fx().gen_clusters(50000, 64, 1e-3, 1e-1, seed)
    m2, p2, v2 = orc.gen_clusters(50000, 64, 1e-3, 1e-1, seed)
    assert np.array_equal(m1, m2) and np.array_equal(p1, p2) and np.array_equal(v1, v2)


def test_plummer_ic_truncation_and_virial_ratio(orc):
    """C1: r <= 20 a; the DF velocities of a Plummer sphere are in virial
    balance, 2T/|W| = 1 with W = -3 pi G M^2 / (32 a) for the untruncated
    sphere (the cut at 20 a changes W by well under 1 %)."""
    n, a, mtot = 200_000, 1.0, 1.0
    mass, pos, vel = fx().gen_plummer_ic(n, mtot, a, 20.0, 11)
    r = np.linalg.norm(pos, axis=1)
    assert r.max() <= 20.0 * a
    assert abs(mass.sum() - mtot) < 1e-12 and np.all(mass == mass[0])
    # half-mass radius of a Plummer sphere: a / sqrt(2^(2/3) - 1) = 1.305 a
    assert abs(np.median(r) - 1.3048 * a) < 0.01
    t = 0.5 * (mass * (vel**2).sum(1)).sum()
    w = -3.0 * np.pi * mtot**2 / (32.0 * a)
    assert abs(2.0 * t / abs(w) - 1.0) < 0.02
    # isotropy: the mean velocity vanishes and each axis carries a third of T
    assert np.linalg.norm((mass[:, None] * vel).sum(0)) / (mass * np.linalg.norm(vel, axis=1)).sum() < 0.01
    share = (mass[:, None] * vel**2).sum(0) / (2.0 * t)
    assert np.all(np.abs(share - 1.0 / 3.0) < 0.01)
    # a scaled sphere: radii scale with a, speeds with sqrt(M / a)
    _, p2, v2 = fx().gen_plummer_ic(n, 4.0, 0.5, 20.0, 11)
    assert np.allclose(p2, 0.5 * pos, rtol=0, atol=1e-12)
    assert np.allclose(v2, np.sqrt(4.0 / 0.5) * vel, rtol=1e-12)


def test_uniform_lognormal_moments():
    """C2: positions uniform in [0,1)^3; log m ~ N(mu, 0.5^2) before the
    normalisation to sum 1."""
    n = 400_000
    mass, pos = fx().gen_uniform_lognormal(n, 0.5, 22)
    assert pos.min() >= 0.0 and pos.max() < 1.0
    assert np.all(np.abs(pos.mean(0) - 0.5) < 0.003)
    assert np.all(np.abs(pos.var(0) - 1.0 / 12.0) < 0.002)
    assert abs(mass.sum() - 1.0) < 1e-12
    lm = np.log(mass)
    assert abs(lm.std() - 0.5) < 0.003
    # normalisation: sum exp(0.5 Z) = n e^{0.125}, so mean(log m) = -log n - 0.125
    assert abs(lm.mean() - (-np.log(n) - 0.125)) < 0.005
    skew = ((lm - lm.mean()) ** 3).mean() / lm.std() ** 3
    assert abs(skew) < 0.02


def test_clusters_dirichlet_split(orc):
    """C3: 64 Plummer spheres whose sizes sum to N, scale radii in [1e-3, 1e-1],
    centres in the unit cube; equal masses summing to 1."""
    n = 1 << 18
    mass, pos, vel = fx().gen_clusters(n, 64, 1e-3, 1e-1, 33)
    assert len(mass) == n and abs(mass.sum() - 1.0) < 1e-12 and np.all(mass == 1.0 / n)
    # the clusters come out one after another; recover them from the stream
    u = orc.rng_units(33, 64 * 5)
    w = -np.log(1.0 - u[0::5])
    a = 1e-3 * np.exp(np.log(100.0) * u[1::5])
    cen = np.stack([u[2::5], u[3::5], u[4::5]], axis=1)
    cnt = np.floor(n * w / w.sum()).astype(np.int64)
    for j in range(n - int(cnt.sum())):
        cnt[j % 64] += 1
    assert cnt.sum() == n and np.all(cnt >= 0)
    assert a.min() >= 1e-3 and a.max() <= 1e-1
    off = np.concatenate([[0], np.cumsum(cnt)])
    for j in range(64):
        if cnt[j] == 0:
            continue
        d = np.linalg.norm(pos[off[j]:off[j + 1]] - cen[j], axis=1)
        assert d.max() <= 20.0 * a[j] * (1 + 1e-12)
        if cnt[j] > 2000:
            assert abs(np.median(d) / a[j] - 1.3048) < 0.1
    # Dirichlet(1) over 64 parts: the fractions are Beta(1, 63), mean 1/64
    frac = cnt / n
    assert abs(frac.mean() - 1.0 / 64) < 1e-12 and frac.max() < 0.2
