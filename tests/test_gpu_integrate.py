"""Device-resident leapfrog (fmmx_leapfrog_device).

The energy smoke test mirrors crates/fmm/tests/energy_gate.rs:235-251: a
virialised Plummer sphere (N=1024, local Maxwellian of seed 43, COM removed,
rescaled to virial balance), 100 drift-kick-drift steps of dt=1e-4 with the
reference MAC at p=4, eps=1e-3: E0 ~ -0.147, momentum < 1e-12, drift < 1e-2.
"""

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def warm_start(orc, mass, pos, pot):
    """energy_gate.rs:39-79 (local Maxwellian sigma^2 = 1/(6 sqrt(1+r^2)))."""
    n = len(mass)
    u = orc.rng_units(43, 6 * n)  # two draws per Gaussian, three per body
    vel = np.empty((n, 3))
    q = 0
    for i in range(n):
        r2 = float(pos[i] @ pos[i])
        sigma = math.sqrt(1.0 / (6.0 * math.sqrt(1.0 + r2)))
        for d in range(3):
            u1 = max(u[q], 1e-15)
            u2 = u[q + 1]
            q += 2
            vel[i, d] = sigma * math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * math.pi * u2)
    mtot = mass.sum()
    vel -= (mass[:, None] * vel).sum(0) / mtot
    t0 = 0.5 * (mass * (vel**2).sum(1)).sum()
    w0 = -0.5 * (mass * pot).sum()
    vel *= math.sqrt(-0.5 * w0 / t0)
    return vel


def energy(mass, vel, pot):
    return 0.5 * (mass * (vel**2).sum(1)).sum() - 0.5 * (mass * pot).sum()


def momentum_rel(mass, vel):
    p = (mass[:, None] * vel).sum(0)
    return np.linalg.norm(p) / (mass * np.linalg.norm(vel, axis=1)).sum()


def run_leapfrog(mass, pos, vel, fmm_kw, dt, steps, scheme, refresh_every):
    import torch

    import fmms_b200 as fx

    n = len(mass)
    d_pos = torch.from_numpy(pos.copy()).cuda()
    d_vel = torch.from_numpy(vel.copy()).cuda()
    d_mass = torch.from_numpy(mass).cuda()
    d_acc = torch.empty((n, 3), dtype=torch.float64, device="cuda")
    d_pot = torch.empty(n, dtype=torch.float64, device="cuda")
    g = fx.Fmm(None, None, **fmm_kw, stream=torch.cuda.current_stream().cuda_stream)
    g.build_device(d_pos.data_ptr(), d_mass.data_ptr(), n)
    g.evaluate_device(d_pos.data_ptr(), d_mass.data_ptr(), d_acc.data_ptr(), d_pot.data_ptr())
    g.leapfrog_device(d_pos.data_ptr(), d_vel.data_ptr(), d_mass.data_ptr(), d_acc.data_ptr(), d_pot.data_ptr(), dt,
                      steps, scheme, refresh_every)
    torch.cuda.synchronize()
    return d_pos.cpu().numpy(), d_vel.cpu().numpy(), d_acc.cpu().numpy(), d_pot.cpu().numpy()


def test_energy_conservation_smoke(orc):
    """energy_gate.rs:235-251 on the device (drift-kick-drift, rebuild every step)."""
    import fmms_b200 as fx

    mass, pos = fx.gen_plummer(1024, seed=42)
    kw = dict(p=4, eps=1e-3, n_leaf=16)
    pot0 = fx.Fmm(mass, pos, **kw).run().pot
    vel = warm_start(orc, mass, pos, pot0)
    e0 = energy(mass, vel, pot0)
    assert abs(e0 + 0.147) < 0.03
    x, v, a, pot = run_leapfrog(mass, pos, vel, kw, 1e-4, 100, "dkd", 1)
    e1 = energy(mass, v, pot)
    assert momentum_rel(mass, v) < 1e-12
    assert abs((e1 - e0) / e0) < 1e-2


@pytest.mark.parametrize("precision,refresh", [("plain", 1), ("mixed", 1), ("mixed", 4)])
def test_kdk_matches_host_loop(precision, refresh):
    """KDK on the device follows a host-side KDK around build + evaluate; with
    tree reuse (refresh 4) it stays within the FMM error of the rebuilt run."""
    import fmms_b200 as fx

    mass, pos, vel = fx.gen_plummer_ic(8192, seed=5)
    kw = dict(p=8, eps=0.0, n_leaf=32, mac="theta", theta=0.5, softening=1e-3, precision=precision)
    dt, steps = 1e-3, 6
    x, v, a, pot = run_leapfrog(mass, pos, vel, kw, dt, steps, "kdk", refresh)
    # host loop, rebuild every step
    g = fx.Fmm(mass, pos, **kw)
    hx, hv = pos.copy(), vel.copy()
    ha = g.run().accel
    for _ in range(steps):
        hv += 0.5 * dt * ha
        hx += dt * hv
        g.refresh(mass, hx)
        ha = g.run().accel
        hv += 0.5 * dt * ha
    scale = np.abs(hx).max()
    tol = 1e-13 if refresh == 1 else 1e-6
    assert np.max(np.abs(x - hx)) < tol * scale
    rel = np.linalg.norm(a - ha, axis=1) / np.linalg.norm(ha, axis=1)
    assert np.percentile(rel, 99) < (1e-11 if refresh == 1 else 1e-4)


@pytest.mark.parametrize("use_graphs", [False, True])
def test_mixed_reuse_after_drift_stays_finite(use_graphs):
    """Mixed form, leaves of 64 and a tree reused for 4 steps while the bodies
    drift: a cell whose built radius is tiny (a tight pair) must be normalised
    with its radius about the build's centre at the current positions, else
    its FP32 moments overflow. The forces stay finite and within the FMM error
    of the same steps with a rebuild every step."""
    import torch

    import fmms_b200 as fx

    mass, pos, vel = fx.gen_plummer_ic(3000, seed=50)
    kw = dict(p=8, eps=0.0, n_leaf=64, mac="theta", theta=0.5, softening=1e-3, precision="mixed",
              use_graphs=use_graphs)
    with torch.cuda.stream(torch.cuda.Stream()):  # graphs are recorded on a non-default stream only
        x4, v4, a4, p4 = run_leapfrog(mass, pos, vel, kw, 1e-3, 4, "kdk", 8)
        x1, v1, a1, p1 = run_leapfrog(mass, pos, vel, kw, 1e-3, 4, "kdk", 1)
    assert np.all(np.isfinite(a4)) and np.all(np.isfinite(x4)) and np.all(np.isfinite(p4))
    rel = np.linalg.norm(a4 - a1, axis=1) / np.linalg.norm(a1, axis=1)
    assert np.percentile(rel, 99) < 1e-4
    assert np.max(np.abs(x4 - x1)) < 1e-6 * np.abs(x1).max()


@pytest.mark.parametrize("precision", ["plain", "mixed"])
def test_graph_replay_matches_launches(precision):
    """Steps on a reused tree replayed from a CUDA graph give the bits of the
    same steps launched one by one (refresh every 4 steps: captures after
    every rebuild, replays in between)."""
    import fmms_b200 as fx

    import torch

    mass, pos, vel = fx.gen_plummer_ic(8192, seed=9)
    out = []
    side = torch.cuda.Stream()  # the legacy default stream cannot be captured
    for graphs in (False, True):
        kw = dict(p=8, eps=0.0, n_leaf=32, mac="theta", theta=0.5, softening=1e-3, precision=precision,
                  use_graphs=graphs)
        with torch.cuda.stream(side):
            out.append(run_leapfrog(mass, pos, vel, kw, 1e-3, 11, "kdk", 4))
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("precision", ["plain", "mixed"])
def test_graph_dropped_by_new_lists(precision):
    """A full evaluation between two graph-replayed leapfrog calls rebuilds the
    interaction lists (new buffers and sizes); the next leapfrog call must not
    replay the graph recorded against the old lists. Bitwise equal to the same
    sequence without graphs."""
    import torch

    import fmms_b200 as fx

    mass, pos, vel = fx.gen_plummer_ic(8192, seed=21)
    n = len(mass)
    side = torch.cuda.Stream()
    out = []
    counts = []
    for graphs in (False, True):
        # the reference MAC: its decisions follow the moments, so the walk on
        # moved bodies gives other lists for the same tree
        kw = dict(p=8, eps=1e-5, n_leaf=32, softening=1e-3, precision=precision, use_graphs=graphs)
        with torch.cuda.stream(side):
            d_pos = torch.from_numpy(pos.copy()).cuda()
            d_vel = torch.from_numpy(vel.copy()).cuda()
            d_mass = torch.from_numpy(mass).cuda()
            d_acc = torch.empty((n, 3), dtype=torch.float64, device="cuda")
            d_pot = torch.empty(n, dtype=torch.float64, device="cuda")
            g = fx.Fmm(None, None, **kw, stream=side.cuda_stream)
            ptrs = (d_pos.data_ptr(), d_vel.data_ptr(), d_mass.data_ptr(), d_acc.data_ptr(), d_pot.data_ptr())
            g.build_device(d_pos.data_ptr(), d_mass.data_ptr(), n)
            g.evaluate_device(d_pos.data_ptr(), d_mass.data_ptr(), d_acc.data_ptr(), d_pot.data_ptr())
            g.leapfrog_device(*ptrs, 1e-3, 3, "kdk", 8)  # records and replays a graph
            c0 = (g.stats()["n_m2l"], g.stats()["n_p2p"])
            # move the bodies so that the walk changes, then a full evaluation
            d_pos.mul_(1.3)
            g.evaluate_device(d_pos.data_ptr(), d_mass.data_ptr(), d_acc.data_ptr(), d_pot.data_ptr())
            counts.append((c0, (g.stats()["n_m2l"], g.stats()["n_p2p"])))
            g.leapfrog_device(*ptrs, 1e-3, 3, "kdk", 8)
            side.synchronize()
            out.append([t.cpu().numpy() for t in (d_pos, d_vel, d_acc, d_pot)])
            g.close()
    assert counts[0][0] != counts[0][1]  # the lists did change
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)


def test_energy_gate_mixed(orc):
    """Mixed form on the reference's energy-gate setup (energy_gate.rs:143-219
    with the smoke's IC, :235-251): a virialised Plummer sphere, here N = 2^16
    with the reference MAC (eps 1e-5, p 8, leaf 16), 400 kick-drift-kick steps
    of dt = 1e-3 with a rebuild every step. The gate of :253-290 on energy:
    drift and maximum deviation < 1e-3, secular slope < 1e-6 per step; the
    drift is also checked in each window of 100 steps. Momentum: the mixed
    form's near field is FP32, so its bound is 1e-6 instead of 1e-12."""
    import torch

    import fmms_b200 as fx

    n, steps, dt = 1 << 16, 400, 1e-3
    mass, pos = fx.gen_plummer(n, seed=42)
    kw = dict(p=8, eps=1e-5, n_leaf=16, precision="mixed")
    pot0 = fx.Fmm(mass, pos, **kw).run().pot
    vel = warm_start(orc, mass, pos, pot0)
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        d_pos = torch.from_numpy(pos.copy()).cuda()
        d_vel = torch.from_numpy(vel.copy()).cuda()
        d_mass = torch.from_numpy(mass).cuda()
        d_acc = torch.empty((n, 3), dtype=torch.float64, device="cuda")
        d_pot = torch.empty(n, dtype=torch.float64, device="cuda")
        g = fx.Fmm(None, None, **kw, stream=side.cuda_stream)
        g.build_device(d_pos.data_ptr(), d_mass.data_ptr(), n)
        g.evaluate_device(d_pos.data_ptr(), d_mass.data_ptr(), d_acc.data_ptr(), d_pot.data_ptr())

        def e_now():
            return float((0.5 * (d_mass * (d_vel * d_vel).sum(1)).sum() - 0.5 * (d_mass * d_pot).sum()).item())

        e0 = e_now()
        es = []
        for _ in range(steps):
            g.leapfrog_device(d_pos.data_ptr(), d_vel.data_ptr(), d_mass.data_ptr(), d_acc.data_ptr(),
                              d_pot.data_ptr(), dt, 1, "kdk", 1)
            es.append(e_now())
        v = d_vel.cpu().numpy()
        g.close()
    es = np.array(es)
    assert abs(e0 + 0.147) < 0.03
    drift = (es[-1] - e0) / abs(e0)
    max_dev = np.max(np.abs(es - e0)) / abs(e0)
    t = np.arange(1, steps + 1, dtype=float)
    slope = np.polyfit(t, es, 1)[0] / abs(e0)
    windows = [(es[k + 99] - (es[k - 1] if k else e0)) / abs(e0) for k in range(0, steps, 100)]
    assert abs(drift) < 1e-3, drift
    assert max_dev < 1e-3, max_dev
    assert abs(slope) < 1e-6, slope
    assert max(abs(w) for w in windows) < 1e-3, windows
    assert momentum_rel(mass, v) < 1e-6


@pytest.mark.parametrize("refresh", [1, 3])
def test_kdk_step_rows(refresh):
    """fmmx_kdk_step_device with the same time step on every row gives the
    bits of fmmx_leapfrog_device (KDK, same refresh cadence, graphs off); rows
    with a zero step keep their positions and velocities exactly."""
    import torch

    import fmms_b200 as fx

    mass, pos, vel = fx.gen_plummer_ic(6000, seed=13)
    n = len(mass)
    kw = dict(p=8, eps=0.0, n_leaf=32, mac="theta", theta=0.5, softening=1e-3, precision="mixed", use_graphs=False)
    side = torch.cuda.Stream()  # torch's work and the engine's on one stream
    with torch.cuda.stream(side):
        x1, v1, a1, _ = run_leapfrog(mass, pos, vel, kw, 1e-3, 6, "kdk", refresh)
        kdk_rows_run(fx, torch, side, mass, pos, vel, kw, refresh, x1, v1, a1)


def kdk_rows_run(fx, torch, side, mass, pos, vel, kw, refresh, x1, v1, a1):
    n = len(mass)
    d_pos = torch.from_numpy(pos.copy()).cuda()
    d_vel = torch.from_numpy(vel.copy()).cuda()
    d_mass = torch.from_numpy(mass).cuda()
    d_acc = torch.empty((n, 3), dtype=torch.float64, device="cuda")
    d_pot = torch.empty(n, dtype=torch.float64, device="cuda")
    d_dt = torch.full((n,), 1e-3, dtype=torch.float64, device="cuda")
    g = fx.Fmm(None, None, **kw, stream=side.cuda_stream)
    g.build_device(d_pos.data_ptr(), d_mass.data_ptr(), n)
    g.evaluate_device(d_pos.data_ptr(), d_mass.data_ptr(), d_acc.data_ptr(), d_pot.data_ptr())
    ptrs = (d_pos.data_ptr(), d_vel.data_ptr(), d_mass.data_ptr(), d_acc.data_ptr(), d_pot.data_ptr(), d_dt.data_ptr())
    for k in range(6):
        g.kdk_step_device(*ptrs, rebuild=(k + 1) % refresh == 0)
    torch.cuda.synchronize()
    assert np.array_equal(d_pos.cpu().numpy(), x1) and np.array_equal(d_vel.cpu().numpy(), v1)
    assert np.array_equal(d_acc.cpu().numpy(), a1)
    # a zero step on the second half of the rows: those bodies stay put
    x0, v0 = d_pos.cpu().numpy(), d_vel.cpu().numpy()
    d_dt[n // 2:] = 0.0
    g.kdk_step_device(*ptrs, offsets=np.array([0, n], dtype=np.uint64))
    torch.cuda.synchronize()
    xa, va = d_pos.cpu().numpy(), d_vel.cpu().numpy()
    assert np.array_equal(xa[n // 2:], x0[n // 2:]) and np.array_equal(va[n // 2:], v0[n // 2:])
    assert not np.array_equal(xa[: n // 2], x0[: n // 2])
    g.close()
