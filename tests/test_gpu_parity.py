"""Parity of the CUDA engine (plain FP64 form) with the oracle.

Bar: Morton keys, slot order, every cell field, multipoles, multipole power,
the f pre-pass and fmin bit-exact; the M2L and P2P pair sets equal as sets;
locals, accelerations and potentials within 1e-12 relative (per body, normwise
over the three components). Every call goes through the C ABI (libfmmx.so).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ACC_TOL = 1e-12  # relative, per body


def fx():
    import fmms_b200

    return fmms_b200


def pair_set(a):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    return np.sort(a.view(np.uint64).ravel())


def rel_rows(a, b):
    den = np.linalg.norm(b, axis=-1) if b.ndim > 1 else np.abs(b)
    num = np.linalg.norm(a - b, axis=-1) if b.ndim > 1 else np.abs(a - b)
    return num / np.maximum(den, 1e-300)


def check_case(orc, mass, pos, p, eps, n_leaf, *, acc_tol=ACC_TOL, loc_tol=1e-11, **kw):
    okw = {}
    if kw.get("mac") == "theta":
        okw["mac"] = orc.MAC_THETA
        okw["theta"] = kw["theta"]
    if "softening" in kw:
        okw["softening"] = kw["softening"]
    if kw.get("center") == "sphere":
        okw["center"] = 1
    if "soft_gap" in kw:
        okw["soft_gap"] = kw["soft_gap"]
    g = fx().Fmm(mass, pos, p, eps, n_leaf, **kw)
    res = g.run()
    o = orc.Fmm(mass, pos, p, eps, n_leaf, **okw)
    acc_o, pot_o = o.run()

    order_g, keys_g, cells_g = g.export_tree()
    order_o, keys_o = o.order()
    assert np.array_equal(keys_g, keys_o)
    assert np.array_equal(order_g, order_o)
    cells_o = o.cells()
    for k in ("first", "count", "level", "leaf", "children", "cen", "mass", "rho"):
        assert np.array_equal(cells_g[k], cells_o[k]), k
    ex = g.export_expansions()
    assert np.array_equal(ex["moments"], o.moments())
    assert np.array_equal(ex["pows"], o.pows())
    if kw.get("mac", "dehnen") == "dehnen":
        f_o, fmin_o = o.fprepass()
        assert np.array_equal(ex["f"], f_o)
        assert np.array_equal(ex["fmin"], fmin_o)
    m2l_g, p2p_g = g.export_lists()
    m2l_o, p2p_o = o.lists()
    assert np.array_equal(pair_set(m2l_g), pair_set(m2l_o))
    assert np.array_equal(pair_set(p2p_g), pair_set(p2p_o))
    loc_o = o.locals()
    scale = np.abs(loc_o).max(axis=1, keepdims=True) + 1e-300
    assert np.max(np.abs(ex["locals"] - loc_o) / scale) < loc_tol
    ra = rel_rows(res.accel, acc_o)
    rp = rel_rows(res.pot, pot_o)
    assert ra.max() < acc_tol, f"acc rel err {ra.max():.3e}"
    assert rp.max() < acc_tol, f"pot rel err {rp.max():.3e}"
    return g, res


def test_plummer_small(orc):
    mass, pos = orc.plummer(4096, seed=1234)
    check_case(orc, mass, pos, 6, 1e-4, 16)


@pytest.mark.parametrize("p,eps,n_leaf", [(2, 1e-2, 16), (4, 1e-4, 8), (8, 1e-5, 16), (10, 1e-6, 32), (12, 1e-7, 64)])
def test_plummer_orders(orc, p, eps, n_leaf):
    mass, pos = orc.plummer(16384, seed=2024)
    check_case(orc, mass, pos, p, eps, n_leaf)


def test_hernquist(orc):
    mass, pos = orc.hernquist(8192, seed=7)
    check_case(orc, mass, pos, 5, 1e-5, 32)


def test_theta_mac_softened(orc):
    mass, pos = orc.plummer(16384, seed=99)
    check_case(orc, mass, pos, 8, 0.0, 64, mac="theta", theta=0.5, softening=1e-3)


@pytest.mark.parametrize("mac", ["theta", "dehnen"])
def test_softening_gap(orc, mac):
    """M2L only between cells whose bodies are soft_gap * softening apart
    (extension): the same pair sets as the oracle, forces to 1e-12."""
    mass, pos = orc.plummer(16384, seed=7)
    kw = dict(mac="theta", theta=0.5) if mac == "theta" else {}
    g, _ = check_case(orc, mass, pos, 8, 1e-6, 32, softening=0.02, soft_gap=10.0, **kw)
    m2l_g, _ = g.export_lists()
    h, _ = check_case(orc, mass, pos, 8, 1e-6, 32, softening=0.02, **kw)
    m2l_h, _ = h.export_lists()
    assert len(m2l_g) < len(m2l_h)  # the condition removed pairs


def test_rotation_m2l(orc):
    """Rotation M2L (the reference's p >= 20 kernel) against the oracle's naive
    M2L: same lists, forces within the rotation-vs-naive contract."""
    mass, pos = orc.plummer(8192, seed=5)
    check_case(orc, mass, pos, 8, 1e-5, 16, m2l="rotation", acc_tol=1e-11)


def test_rotation_high_order(orc):
    """p = 20 takes the rotation kernel in both engines (ROT_P, rotation.rs:45)."""
    mass, pos = orc.plummer(4096, seed=5)
    # rotation.rs:545 bounds the rotation kernel against naive at 1e-9 relative
    check_case(orc, mass, pos, 20, 1e-10, 16, acc_tol=1e-10, loc_tol=1e-9)


def test_sphere_centres(orc):
    mass, pos = orc.plummer(8192, seed=3)
    check_case(orc, mass, pos, 6, 1e-5, 16, center="sphere")


def test_grid_73_cells(orc):
    """tree.rs:466-480 on the device: 4x4x4 grid, n_leaf 1 -> 73 cells."""
    pos = np.array([[i % 4, (i // 4) % 4, i // 16] for i in range(64)], dtype=float)
    mass = np.ones(64)
    g, res = check_case(orc, mass, pos, 2, 1e-3, 1)
    assert res.n_cells == 73


def test_two_bodies(orc):
    mass = np.array([1.0, 2.0])
    pos = np.array([[0.0, 0.0, 0.0], [3.0, 0.0, 0.0]])
    g, res = check_case(orc, mass, pos, 2, 1e-3, 1)
    assert abs(res.accel[0, 0] - 2.0 / 9.0) < 1e-15
    assert abs(res.accel[1, 0] + 1.0 / 9.0) < 1e-15


def test_single_body():
    g = fx().Fmm(np.array([1.0]), np.zeros((1, 3)), 4, 1e-3, 16)
    res = g.run()
    assert res.n_cells == 1 and np.all(res.accel == 0) and res.pot[0] == 0


def test_degenerate_points_tree(orc):
    """tree.rs:482-496: identical points cannot be split -> one leaf."""
    mass = np.full(5, 2.0)
    pos = np.ones((5, 3))
    g = fx().Fmm(mass, pos, 2, 1e-3, 5)
    _, _, cells = g.export_tree()
    assert len(cells["mass"]) == 1 and cells["leaf"][0] and cells["mass"][0] == 10.0


def test_deep_chain(orc):
    """Tight clumps force single-child chains down to level 21 (fat leaves at the cut)."""
    rng = np.random.default_rng(3)
    pos = np.concatenate([rng.normal(0, 1e-7, (300, 3)), rng.uniform(-1, 1, (700, 3))])
    mass = np.full(1000, 1e-3)
    check_case(orc, mass, pos, 4, 1e-4, 8)


def test_refresh_and_reuse(orc):
    """Fmm::refresh == fresh build; run with other positions uses the built tree."""
    mass, pos = orc.plummer(4096, seed=99)
    g = fx().Fmm(mass, pos + np.array([5.0, -3.0, 1.0]), 4, 1e-4, 16)
    g.refresh(mass, pos)
    r1 = g.run()
    g2 = fx().Fmm(mass, pos, 4, 1e-4, 16)
    r2 = g2.run()
    assert np.array_equal(r1.accel, r2.accel) and np.array_equal(r1.pot, r2.pot)
    # deterministic: a second evaluation is bitwise identical
    r3 = g2.run()
    assert np.array_equal(r2.accel, r3.accel)


def test_invalid_inputs():
    with pytest.raises(fx().FmmError):
        fx().Fmm(np.array([]), np.zeros((0, 3)), 4, 1e-3, 16)
    pos = np.zeros((4, 3))
    pos[2, 1] = np.nan
    with pytest.raises(fx().FmmError):
        fx().Fmm(np.ones(4), pos, 4, 1e-3, 16)


def test_direct_targets(orc):
    mass, pos = orc.plummer(20000, seed=11)
    t = orc.sample_targets(len(mass), 7, 300)
    a_g, p_g, f_g = fx().direct_targets(mass, pos, t, softening=1e-3)
    a_o, p_o, f_o = orc.direct_targets(mass, pos, t, softening=1e-3)
    assert np.max(rel_rows(a_g, a_o)) < 1e-12
    assert np.max(rel_rows(p_g, p_o)) < 1e-12 and np.max(rel_rows(f_g, f_o)) < 1e-12


def test_momentum_conserved_gpu(orc):
    """tests/integration.rs:44-68 on the device (mutual lists, directed kernels)."""
    mass, pos = orc.plummer(512, seed=99)
    res = fx().Fmm(mass, pos, 4, 1e-4, 16).run()
    fsum = (mass[:, None] * res.accel).sum(0)
    ftot = (mass * np.linalg.norm(res.accel, axis=1)).sum()
    assert np.linalg.norm(fsum) / ftot < 1e-13


def test_full_size_c2_plain(orc):
    """The headline configuration at full size, N = 2^20 (uniform cube, log-normal
    masses, softening 1e-4, p = 10, theta 0.5, leaf 64): Morton keys, slot order
    and both pair sets equal to the oracle's, accelerations and potentials within
    1e-12 relative per body (the oracle runs threaded on the host)."""
    import os

    mass, pos = fx().gen_uniform_lognormal(1 << 20, 0.5, 22)
    kw = dict(mac="theta", theta=0.5, softening=1e-4)
    g = fx().Fmm(mass, pos, 10, 0.0, 64, **kw)
    res = g.run()
    o = orc.Fmm(mass, pos, 10, 0.0, 64, mac=orc.MAC_THETA, theta=0.5, softening=1e-4)
    acc_o, pot_o = o.run(nthreads=os.cpu_count() or 1)
    order_g, keys_g, _ = g.export_tree()
    order_o, keys_o = o.order()
    assert np.array_equal(keys_g, keys_o)
    assert np.array_equal(order_g, order_o)
    m2l_g, p2p_g = g.export_lists()
    m2l_o, p2p_o = o.lists()
    assert np.array_equal(pair_set(m2l_g), pair_set(m2l_o))
    assert np.array_equal(pair_set(p2p_g), pair_set(p2p_o))
    ra = rel_rows(res.accel, acc_o)
    rp = rel_rows(res.pot, pot_o)
    assert ra.max() < ACC_TOL, f"acc rel err {ra.max():.3e}"
    assert rp.max() < ACC_TOL, f"pot rel err {rp.max():.3e}"


def test_c1_plummer_ic(orc):
    """The C1 workload through its own generator (Plummer sphere truncated at
    r <= 20, distribution-function velocities; N = 16384, softening 1e-3, p 8,
    theta 0.5, leaf 64) on the full parity bar."""
    mass, pos, _ = fx().gen_plummer_ic(16384, 1.0, 1.0, 20.0, 11)
    check_case(orc, mass, pos, 8, 0.0, 64, mac="theta", theta=0.5, softening=1e-3)


@pytest.mark.parametrize("p", [4, 8])
def test_naive_m2l(orc, p):
    """m2l='naive' (k_m2l_naive_f64, the reference's O(p^4) convolution of
    translate.rs:47-136) against the oracle: same lists, locals and forces."""
    mass, pos = orc.plummer(8192, seed=17)
    check_case(orc, mass, pos, p, 1e-5, 16, m2l="naive")
    mass, pos, _ = fx().gen_plummer_ic(8192, 1.0, 1.0, 20.0, 3)
    check_case(orc, mass, pos, p, 0.0, 32, m2l="naive", mac="theta", theta=0.5, softening=1e-3)


def test_c3_clusters_plain(orc):
    """The clustered deep-tree workload's generator and settings (64 Plummer
    clusters, scale radii log-uniform in [1e-3, 1e-1], leaf 32, p 12, theta
    0.4, softening 1e-5) at N = 2^20 on the plain form: Morton keys, slot
    order, every cell field, both pair sets equal to the oracle's, and
    accelerations and potentials within 1e-12 relative per body (oracle
    threaded on the host)."""
    import os

    mass, pos, _ = fx().gen_clusters(1 << 20, 64, 1e-3, 1e-1, 33)
    kw = dict(mac="theta", theta=0.4, softening=1e-5)
    g = fx().Fmm(mass, pos, 12, 0.0, 32, **kw)
    res = g.run()
    o = orc.Fmm(mass, pos, 12, 0.0, 32, mac=orc.MAC_THETA, theta=0.4, softening=1e-5)
    acc_o, pot_o = o.run(nthreads=os.cpu_count() or 1)
    order_g, keys_g, cells_g = g.export_tree()
    order_o, keys_o = o.order()
    assert np.array_equal(keys_g, keys_o)
    assert np.array_equal(order_g, order_o)
    cells_o = o.cells()
    for k in ("first", "count", "level", "leaf", "children", "cen", "mass", "rho"):
        assert np.array_equal(cells_g[k], cells_o[k]), k
    assert cells_g["level"].max() >= 12  # a deep tree
    m2l_g, p2p_g = g.export_lists()
    m2l_o, p2p_o = o.lists()
    assert np.array_equal(pair_set(m2l_g), pair_set(m2l_o))
    assert np.array_equal(pair_set(p2p_g), pair_set(p2p_o))
    ra = rel_rows(res.accel, acc_o)
    rp = rel_rows(res.pot, pot_o)
    assert ra.max() < ACC_TOL, f"acc rel err {ra.max():.3e}"
    assert rp.max() < ACC_TOL, f"pot rel err {rp.max():.3e}"


def test_walk_statistics_n1e6_published(orc, golden):
    """The engine's dual walk at the reference's published walk statistics
    (golden values: 205,395 leaves, 26.7M pops, 20.6M M2L pairs, 2.60M P2P
    leaf-pair calls at N = 1e6, plummer(n, 0, 42), p = 8, eps = 1e-5, leaf
    16; PERF-ANALYSIS.md:50-52)."""
    import fmms_b200 as fx

    g = golden["walk_stats_n1e6"]
    mass, pos = orc.plummer(1_000_000, seed=42)
    f = fx.Fmm(mass, pos, 8, 1e-5, 16)
    f.run()
    st = f.stats()
    leaves = int(st["n_leaves"])
    assert leaves == g["leaves"]
    assert round(st["walk_pops"] / 1e6, 1) == g["pops_millions"]
    assert round(st["n_m2l"] / 1e6, 1) == g["m2l_pairs_millions"]
    assert round((st["n_p2p"] - leaves) / 1e6, 2) == g["p2p_calls_millions"]


def test_exit_gate_n1e4_published(orc, golden):
    """tests/exit_gate.rs:11-24 on the device: the scaled errors against the
    direct sum reproduce the reference's published release run (todo.md:586)
    to its printed digits."""
    import fmms_b200 as fx

    g = golden["exit_gate_n1e4"]
    mass, pos = orc.plummer(10_000, seed=2024)
    acc = fx.Fmm(mass, pos, 5, 1e-5, 32).run().accel
    a_ref, _ = orc.direct(mass, pos)
    max_s, _, rms_s, _ = orc.scaled_error(a_ref, acc, mass, pos)
    assert round(max_s, g["printed_digits"]["max_s"]) == g["max_s"], max_s
    assert round(rms_s, g["printed_digits"]["rms_s"]) == g["rms_s"], rms_s
