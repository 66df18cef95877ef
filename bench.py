#!/usr/bin/env python
"""Benchmark of the FMM force engine on B200.

Metric: bodies/s of kick-drift-kick leapfrog steps (each a complete force
evaluation: tree build, upward pass, dual walk, lists, M2L, L2L, P2P, L2P)
on one GPU, in the mixed-precision form against the plain FP64 form, both at
a setting where the p99 relative force error against the FP64 direct sum on
4096 seeded targets is <= 1e-5; p50/p99 step times beside it.

Workload (default, --config c3): the clustered deep-tree system, N = 4,194,304
bodies in 64 Plummer spheres (scale radii log-uniform in [1e-3, 1e-1], centres
uniform in the unit cube, Dirichlet(1) sizes, equal masses summing to 1,
distribution-function velocities), softening 1e-5, leaf capacity 32, KDK steps
of dt = 1e-4 with a rebuild every step; seeded synthetic data. The configured
order and opening angle (p = 12, theta = 0.4) leave p99 at 2.1e-4 in both
forms (the unsoftened far field against a softened direct sum); the bench runs
p = 10, theta = 0.5 with M2L pairs kept soft_gap = 200 softening lengths
apart, where both forms meet the bound.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision mixed|plain]
    python bench.py --config c2 ...         # one force evaluation, N = 2^20 uniform cube
    python bench.py --impl reference ...    # the reference FMM on the host cores (oracle/)

Under torchrun every rank runs its own replica (the evaluation does not shard;
no collective on the data path); rank 0 prints one JSON line.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

def max_over_ranks(ms: float, world: int, device) -> float:
    """The slowest replica's time: every rank passes its own total, all take
    the same collective steps (an all-reduce with MAX, then a barrier). With
    one rank it is the rank's own time."""
    if world <= 1:
        return ms
    import torch
    import torch.distributed as dist

    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.barrier()
    return float(t.item())


def replicas_value(units_per_rank: float, steps: int, max_total_ms: float, world: int) -> float:
    """Whole-job throughput of `world` replicas: the units all ranks processed
    over the slowest rank's time."""
    return world * units_per_rank * steps / (max_total_ms * 1e-3)


CONFIGS = {
    "c1": dict(gen="plummer_ic", n=16384, p=8, theta=0.5, softening=1e-3, n_leaf=64,
               workload="Plummer N=16384 (r<=20, DF velocities), softening 1e-3, p=8, theta=0.5, leaf 64"),
    "c2": dict(gen="uniform", n=1 << 20, p=10, theta=0.5, softening=1e-4, n_leaf=64,
               workload="uniform cube N=1048576, log-normal masses sigma=0.5, softening 1e-4, p=10, theta=0.5, leaf 64"),
    "c3": dict(gen="clusters", n=1 << 22, p=12, theta=0.4, softening=1e-5, n_leaf=32,
               workload="64 Plummer clusters N=4194304, a log-uniform[1e-3,1e-1], softening 1e-5, p=12, theta=0.4, leaf 32"),
}
# The headline: the clustered system in KDK steps at the setting where both
# forms meet p99 <= 1e-5 (from the accuracy sweep, --config c3 --sweep).
HEADLINE = dict(CONFIGS["c3"], p=10, theta=0.5, soft_gap=200.0, dt=1e-4,
                workload="64 Plummer clusters N=4194304 (a log-uniform[1e-3,1e-1], Dirichlet(1) sizes, DF velocities), "
                         "softening 1e-5, leaf 32, KDK steps dt=1e-4 with a rebuild every step; p=10, theta=0.5, "
                         "soft_gap=200 (both forms meet p99<=1e-5 there; the configured p=12, theta=0.4 give "
                         "p99 2.1e-4 in both forms)")
EXTRA_CONFIGS = {
    "c4": dict(gen="ensemble", n=0, p=8, theta=0.5, softening=1e-3, n_leaf=64, workload="ensemble"),
    "c5": dict(gen="serve", n=0, p=8, theta=0.5, softening=1e-3, n_leaf=64, workload="serving"),
}
SEEDS = {"plummer_ic": 11, "uniform": 22, "clusters": 33}
METRIC = "bodies/s at p99 force err <=1e-5 (mixed vs FP64 plain, 1 B200); p50/p99 step ms"


def make_inputs(gen, cfg, velocities=False):
    """Seeded inputs of a configuration from `gen`: the engine package
    (fmms_b200) in the GPU arm, the oracle in the CPU arm (the two give the
    same bits, tests/test_generators.py)."""
    n = cfg["n"]
    if cfg["gen"] == "uniform":
        mass, pos = gen.gen_uniform_lognormal(n, 0.5, SEEDS["uniform"])
        vel = np.zeros_like(pos)
    elif cfg["gen"] == "plummer_ic":
        mass, pos, vel = gen.gen_plummer_ic(n, 1.0, 1.0, 20.0, SEEDS["plummer_ic"])
    else:
        mass, pos, vel = gen.gen_clusters(n, 64, 1e-3, 1e-1, SEEDS["clusters"])
    return (mass, pos, vel) if velocities else (mass, pos)


# ------------------------------------------------------------------ roofline
def m2l_flops_per_translation(p: int, kernel: str) -> float:
    """Flops (FMA = 2) of one directed M2L translation as the kernel runs it.

    rotation (warp kernel, m >= 0 half basis): per degree k (K = k+1 terms)
    four real swap products, each 2 flops per structurally nonzero entry of
    its two (K x K) half-basis matrices (about half the entries: Pm[r][q] != 0
    needs r + q + k even, Qm[r][q] != 0 needs r, q >= 1 and r + q + k odd),
    plus 25K for phases and scaling; the axial translation 4 per (n, m, k)
    term plus 4 per output; the lane reduction 2 per output; phases and
    geometry about 12(p+1) + 50.
    naive: 8 per complex term of sum_{n,m} (p-n+1)^2 (translate.rs:47-136).
    """
    if kernel == "naive":
        return 8.0 * sum((2 * n + 1) * (p - n + 1) ** 2 for n in range(p + 1))
    h = (p + 1) * (p + 2) // 2

    def nz(k):  # structural nonzeros of Pm and Qm of degree k
        r = range(k + 1)
        return (sum(1 for a in r for b in r if (a + b + k) % 2 == 0)
                + sum(1 for a in r for b in r if a >= 1 and b >= 1 and (a + b + k) % 2 == 1))

    rot = sum(8 * nz(k) + 25 * (k + 1) for k in range(p + 1))
    axial = sum(max(0, p - n - m + 1) for m in range(p + 1) for n in range(m, p + 1))
    return rot + 4 * axial + 6 * h + 12 * (p + 1) + 50


def p2p_flops(interactions: int) -> float:
    """16 flops per directed body-body interaction (crates/fmm/src/roofline.rs:15-19)."""
    return 16.0 * interactions


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50", "-f", self.path], stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
            t0 = time.time()  # the timed region starts once the sampler is writing
            while time.time() - t0 < 5 and os.path.getsize(self.path) == 0:
                time.sleep(0.02)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.12)  # at least one sample after the last timed step
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ CPU arm
def oracle_fmm(cfg, mass, pos):
    import oracle

    return oracle.Fmm(mass, pos, cfg["p"], 0.0, cfg["n_leaf"], mac=oracle.MAC_THETA, theta=cfg["theta"],
                      softening=cfg["softening"], soft_gap=cfg.get("soft_gap", 0.0))


def cpu_fmm_sample(cfg, sample_n, nthreads):
    """Time the oracle's restatement of the reference FMM (tree build and the
    threaded run_impl) on a bounded sample of the workload (the same generator
    at sample_n bodies); returns (bodies/s, seconds)."""
    import oracle

    sub = dict(cfg)
    sub["n"] = sample_n
    mass, pos = make_inputs(oracle, sub)
    t0 = time.perf_counter()
    f = oracle_fmm(cfg, mass, pos)
    f.run(nthreads=nthreads)
    dt = time.perf_counter() - t0
    return sample_n / dt, dt


def run_reference(args, cfg, rank, headline):
    """--impl reference: the reference FMM on the box's host cores, restated in
    oracle/ (the Rust reference cannot be built here: no Rust toolchain). It
    loads nothing but the oracle. The headline arm runs the same system at the
    same N and settings: each step a kick-drift-kick step whose force
    evaluation is the oracle's tree build (Fmm::refresh) and threaded run
    (Fmm::run_threaded) on all host threads, the kicks and drifts on the host;
    the warm-up steps run on a 65,536-body system of the same generator (the
    CPU arm has nothing to warm but its allocator). --ref-sample N times an
    N-body sample instead of the full system."""
    if rank != 0:
        return
    import oracle

    nthreads = os.cpu_count() or 1
    full = cfg["n"]
    sample_n = args.ref_sample if args.ref_sample > 0 else full
    sub = dict(cfg, n=sample_n)
    mass, pos, vel = make_inputs(oracle, sub, velocities=True)
    warm = dict(cfg, n=min(65536, sample_n))
    wm, wp = make_inputs(oracle, warm)
    for _ in range(args.warmup):
        oracle_fmm(cfg, wm, wp).run(nthreads=nthreads)
    dt_step = cfg.get("dt", 0.0)
    f = oracle_fmm(cfg, mass, pos)
    # the first kick uses zero accelerations: a full untimed evaluation before
    # the first step would double the arm's run time and the timed work (a
    # tree build and an evaluation per step) does not depend on them
    acc = np.zeros_like(pos)
    times = []
    t_start = time.perf_counter()
    for _ in range(args.steps):
        if times and time.perf_counter() - t_start > args.ref_budget_s:
            break  # time-bounded: every step is the full workload, fewer of them
        t0 = time.perf_counter()
        if headline:  # kick-drift-kick around a rebuild and a threaded evaluation
            vel += 0.5 * dt_step * acc
            pos += dt_step * vel
            f.refresh(mass, pos)
            acc, _ = f.run(nthreads=nthreads)
            vel += 0.5 * dt_step * acc
        else:
            f.refresh(mass, pos)
            f.run(nthreads=nthreads)
        times.append(time.perf_counter() - t0)
    mean = sum(times) / len(times)
    value = sample_n / mean
    what = ("one kick-drift-kick step (oracle tree build + threaded evaluation, host kicks and drifts)"
            if headline else "one force evaluation (oracle tree build + threaded evaluation)")
    sample = (f"the full system ({sample_n} bodies)" if sample_n == full else
              f"{sample_n} bodies of the same generator and settings")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "bodies/s", "n_gpus": args.gpus,
        "steps": len(times), "steps_requested": args.steps, "warmup": args.warmup, "ms_per_step": mean * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": bench_config(cfg, args.gpus, headline),
        "step_ms_p50": float(np.percentile(times, 50)) * 1e3, "step_ms_p99": float(np.percentile(times, 99)) * 1e3,
        "cpu_baseline": {"value": value, "unit": "bodies/s", "cores": nthreads, "kind": "port",
                         "sample": f"{sample}, {what} per step, on {nthreads} host threads; warm-up steps on "
                                   f"{warm['n']} bodies (oracle/fmm_oracle.cpp, the C++ restatement of "
                                   f"crates/fmm run_impl); timed steps stop once {args.ref_budget_s:.0f} s "
                                   f"have passed (at least one)"},
        "e2e": {"value": value, "unit": "bodies/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def bench_config(cfg, world, headline):
    """The `config` object of the JSON line; the same in both arms."""
    c = {"workload": cfg["workload"], "n": cfg["n"], "p": cfg["p"], "theta": cfg["theta"],
         "softening": cfg["softening"], "n_leaf": cfg["n_leaf"]}
    if headline:
        c.update(soft_gap=cfg["soft_gap"], dt=cfg["dt"], refresh_every=1,
                 l2="flushed between timed steps (and the inputs are larger than L2)")
    else:
        c.update(l2="flushed between timed steps")
    c["parallelism"] = "replicas" if world > 1 else "single"
    return c


# ------------------------------------------------------------------ GPU arm
def measure_eval(args, cfg, precision, mass, pos, dev, world, clk_sampler=None):
    """Time one force evaluation (build + evaluate) per step on device-resident
    inputs, then the same through the host API (e2e), then the accuracy."""
    import torch

    import fmms_b200 as fx

    stream = torch.cuda.current_stream()
    n = len(mass)
    d_pos = torch.from_numpy(pos).to(f"cuda:{dev}")
    d_mass = torch.from_numpy(mass).to(f"cuda:{dev}")
    d_acc = torch.empty((n, 3), dtype=torch.float64, device=f"cuda:{dev}")
    d_pot = torch.empty(n, dtype=torch.float64, device=f"cuda:{dev}")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{dev}")
    kw = dict(mac="theta", theta=cfg["theta"], softening=cfg["softening"], precision=precision, m2l=args.m2l,
              device=dev, stream=stream.cuda_stream)
    g = fx.Fmm(None, None, cfg["p"], 0.0, cfg["n_leaf"], **kw)

    def step():
        g.build_device(d_pos.data_ptr(), d_mass.data_ptr(), n)
        g.evaluate_device(d_pos.data_ptr(), d_mass.data_ptr(), d_acc.data_ptr(), d_pot.data_ptr())

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    torch.cuda.synchronize()
    times, m2l_ms, p2p_ms, st = [], [], [], None
    ctx_clk = clk_sampler if clk_sampler is not None else _NullCtx()
    with ctx_clk:
        for _ in range(args.steps):
            flush.zero_()  # L2 flush between timed steps (untimed)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
            st = g.stats()
            m2l_ms.append(st["ms_m2l"])
            p2p_ms.append(st["ms_p2p"])
    torch.cuda.synchronize()
    total_ms = max_over_ranks(sum(times), world, f"cuda:{dev}")

    # end to end through the host API: pinned host inputs in, host results out
    h_pos = torch.from_numpy(pos).pin_memory()
    h_mass = torch.from_numpy(mass).pin_memory()
    h_acc = torch.empty((n, 3), dtype=torch.float64).pin_memory()
    h_pot = torch.empty(n, dtype=torch.float64).pin_memory()
    e2e_times = []
    for i in range(args.warmup + args.steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st_b = fx.lib().fmmx_build(g._h, n, fx._ptr(h_pos.numpy()), fx._ptr(h_mass.numpy()))
        st_e = fx.lib().fmmx_evaluate(g._h, None, None, fx._ptr(h_acc.numpy()), fx._ptr(h_pot.numpy()))
        e1.record(stream)
        e1.synchronize()
        assert st_b == 0 and st_e == 0, fx.lib().fmmx_last_error(g._h)
        if i >= args.warmup:
            e2e_times.append(e0.elapsed_time(e1))
    e2e_ms = max_over_ranks(sum(e2e_times) / len(e2e_times), world, f"cuda:{dev}")

    # accuracy against the FP64 direct sum on 4096 seeded targets
    rng = np.random.default_rng(4096)
    tg = np.sort(rng.choice(n, size=min(4096, n), replace=False)).astype(np.uint32)
    a_ref, _, _ = fx.direct_targets(mass, pos, tg, softening=cfg["softening"], device=dev)
    acc = h_acc.numpy()
    rel = np.linalg.norm(acc[tg] - a_ref, axis=1) / np.linalg.norm(a_ref, axis=1)
    g.close()

    # the M2L and P2P kernels alone on the device (one stream, nothing beside
    # them), for the roofline: in the timed steps the P2P runs beside the M2L
    solo = fx.Fmm(None, None, cfg["p"], 0.0, cfg["n_leaf"], **kw, overlap=False)
    m2l_solo, p2p_solo = [], []
    for i in range(2 + max(args.steps, 1)):
        flush.zero_()
        solo.build_device(d_pos.data_ptr(), d_mass.data_ptr(), n)
        solo.evaluate_device(d_pos.data_ptr(), d_mass.data_ptr(), d_acc.data_ptr(), d_pot.data_ptr())
        if i >= 2:
            sst = solo.stats()
            m2l_solo.append(sst["ms_m2l"])
            p2p_solo.append(sst["ms_p2p"])
    solo.close()
    return dict(times=times, total_ms=total_ms, m2l_ms=sum(m2l_solo) / len(m2l_solo),
                p2p_ms=sum(p2p_solo) / len(p2p_solo), m2l_ms_in_step=sum(m2l_ms) / len(m2l_ms),
                p2p_ms_in_step=sum(p2p_ms) / len(p2p_ms), st=st, e2e_ms=e2e_ms, rel=rel, ntargets=len(tg))


class _NullCtx:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


# DRAM bytes (read + write) per directed M2L translation, from one ncu capture of
# the M2L launch at N = 262144 (uniform cube, p = 10, theta 0.5, leaf 64: 5,809,554
# directed translations); the expansions are L2-resident, so the traffic grows
# with the translation count.
M2L_DRAM_BYTES_PER_TRANSLATION = {("mixed", 10): (34.537728e6 + 0.07424e6) / 5809554,
                                  ("plain", 10): (84.023808e6 + 21.590272e6) / 5809554}


def roofline(args, cfg, r, precision, dev):
    import fmms_b200 as fx

    st = r.get("solo_st") or r["st"]  # the counts of the evaluations the kernels were timed in
    kernel = "naive" if args.m2l == "naive" else "rotation"
    fl = st["m2l_directed"] * m2l_flops_per_translation(cfg["p"], kernel)
    fp64 = precision == "plain"
    peak = fx.probe_fma_peak(fp64=fp64, device=dev)
    achieved = fl / (r["m2l_ms"] * 1e-3) / 1e12
    bpt = M2L_DRAM_BYTES_PER_TRANSLATION.get((precision, cfg["p"])) if kernel == "rotation" else None
    traffic = bpt * st["m2l_directed"] if bpt is not None else None
    return {"bound": "fp64" if fp64 else "fp32", "kernel": "m2l", "achieved": achieved, "peak": peak,
            "unit": "TFLOP/s", "frac": achieved / peak, "traffic": traffic,
            "traffic_note": "DRAM bytes per launch, scaled by directed translations from an ncu capture at "
                            "N=262144" if traffic is not None else "no capture for this order",
            "peak_source": "measured: FMA loop on every SM (fmmx_probe_fma_peak); MEASURED_PEAKS.json holds only "
                           "HBM and bf16-tensor peaks",
            "algorithmic_flops_per_launch": fl, "launch_ms": r["m2l_ms"],
            "launch_timing": "CUDA events around the kernel on its stream, the evaluation on one stream (nothing "
                             "beside it); in the timed steps the P2P runs beside it on a second stream: "
                             f"{r['m2l_ms_in_step']:.3f} ms there",
            "p2p": {"achieved": p2p_flops(st["p2p_interactions"]) / (r["p2p_ms"] * 1e-3) / 1e12,
                    "unit": "TFLOP/s", "ms": r["p2p_ms"]}}


def run_gpu(args, cfg, rank, world, local_rank):
    import torch

    import fmms_b200 as fx

    dev = local_rank
    torch.cuda.set_device(dev)
    mass, pos = make_inputs(fx, cfg)
    n = len(mass)
    clk = ClockSampler(dev)
    main = measure_eval(args, cfg, args.precision, mass, pos, dev, world, clk)
    other = None
    if not args.no_compare:
        other_prec = "plain" if args.precision == "mixed" else "mixed"
        other = measure_eval(args, cfg, other_prec, mass, pos, dev, world)
    if rank != 0:
        return
    value = replicas_value(n, args.steps, main["total_ms"], world)
    st = main["st"]
    rel = main["rel"]
    cpu = None
    if world == 1 and not args.no_cpu:
        nth = os.cpu_count() or 1
        bps, dt = cpu_fmm_sample(cfg, args.cpu_sample, nth)
        cpu = {"value": bps, "unit": "bodies/s", "cores": nth, "kind": "port",
               "sample": f"{args.cpu_sample} bodies of the same generator and settings, one threaded evaluation "
                         f"of the oracle's restatement of the reference FMM ({dt:.1f} s)"}
    fp64 = args.precision == "plain"
    line = {
        "metric": METRIC, "value": value, "unit": "bodies/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": main["total_ms"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if fp64 else "f32+f64", "data": "synthetic",
        "precision": args.precision, "config": bench_config(cfg, world, False),
        "step_ms_p50": float(np.percentile(main["times"], 50)),
        "step_ms_p99": float(np.percentile(main["times"], 99)),
        "force_err": {"p50": float(np.percentile(rel, 50)), "p99": float(np.percentile(rel, 99)),
                      "max": float(rel.max()), "targets": main["ntargets"], "reference": "FP64 direct sum"},
        "e2e": {"value": world * n / (main["e2e_ms"] * 1e-3), "unit": "bodies/s", "h2d_bytes_per_step": 32 * n,
                "d2h_bytes_per_step": 32 * n, "ms_per_step": main["e2e_ms"]},
        "gpu_launches": int(st["kernel_launches"]) * args.steps,
        "stages_ms": {k[3:]: round(v, 3) for k, v in st.items() if k.startswith("ms_")},
        "counts": {k: int(st[k]) for k in ("n_cells", "n_leaves", "n_m2l", "n_p2p", "p2p_interactions")},
        "roofline": roofline(args, cfg, main, args.precision, dev), "cpu_baseline": cpu, "clocks": clk.summary(),
    }
    if other is not None:
        orel = other["rel"]
        ov = replicas_value(n, args.steps, other["total_ms"], world)
        line["compare"] = {"precision": "plain" if args.precision == "mixed" else "mixed", "value": ov,
                           "ms_per_step": other["total_ms"] / args.steps,
                           "force_err_p50": float(np.percentile(orel, 50)),
                           "force_err_p99": float(np.percentile(orel, 99)),
                           "stages_ms": {k[3:]: round(v, 3) for k, v in other["st"].items() if k.startswith("ms_")},
                           "speedup_of_main": value / ov}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ headline: C3 KDK steps
def measure_kdk(args, cfg, precision, mass, pos, vel, tg, dev, world, clk_sampler=None):
    """W untimed and K timed kick-drift-kick steps (a rebuild every step) on
    device-resident state, the force error against the FP64 direct sum at the
    seeded targets after every timed step; then the same steps end to end
    through the host API (pinned host buffers, the reference's loop:
    host kick and drift, Fmm::refresh = fmmx_build, Fmm::run = fmmx_evaluate);
    then the M2L and P2P alone on the device for the roofline."""
    import torch

    import fmms_b200 as fx

    stream = torch.cuda.current_stream()
    n = len(mass)
    cuda = f"cuda:{dev}"
    d_pos = torch.from_numpy(pos.copy()).to(cuda)
    d_vel = torch.from_numpy(vel.copy()).to(cuda)
    d_mass = torch.from_numpy(mass).to(cuda)
    d_acc = torch.empty((n, 3), dtype=torch.float64, device=cuda)
    d_pot = torch.empty(n, dtype=torch.float64, device=cuda)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=cuda)
    d_tg = torch.from_numpy(tg.view(np.int32)).to(cuda)
    t_idx = torch.from_numpy(tg.astype(np.int64)).to(cuda)
    d_aref = torch.empty((len(tg), 3), dtype=torch.float64, device=cuda)
    kw = dict(mac="theta", theta=cfg["theta"], softening=cfg["softening"], precision=precision, m2l=args.m2l,
              soft_gap=cfg["soft_gap"], device=dev, stream=stream.cuda_stream)
    g = fx.Fmm(None, None, cfg["p"], 0.0, cfg["n_leaf"], **kw)
    ptrs = (d_pos.data_ptr(), d_vel.data_ptr(), d_mass.data_ptr(), d_acc.data_ptr(), d_pot.data_ptr())
    g.build_device(d_pos.data_ptr(), d_mass.data_ptr(), n)
    g.evaluate_device(d_pos.data_ptr(), d_mass.data_ptr(), d_acc.data_ptr(), d_pot.data_ptr())

    def step():
        g.leapfrog_device(*ptrs, cfg["dt"], 1, "kdk", 1)

    def force_err():  # the FP64 direct sum at the targets, on the device (no allocation)
        fx.direct_targets_noalloc(n, d_pos.data_ptr(), d_mass.data_ptr(), len(tg), d_tg.data_ptr(),
                                  d_aref.data_ptr(), softening=cfg["softening"], device=dev,
                                  stream=stream.cuda_stream)
        rel = torch.linalg.norm(d_acc[t_idx] - d_aref, dim=1) / torch.linalg.norm(d_aref, dim=1)
        return rel.cpu().numpy()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    torch.cuda.synchronize()
    times, errs, st = [], [], None
    with (clk_sampler if clk_sampler is not None else _NullCtx()):
        for _ in range(args.steps):
            flush.zero_()  # L2 flush between timed steps (untimed)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
            st = g.stats()
            errs.append(force_err())
    torch.cuda.synchronize()
    total_ms = max_over_ranks(sum(times), world, cuda)
    g.close()

    # end to end: the reference's loop through the host API
    h_pos = torch.from_numpy(pos.copy()).pin_memory()
    h_vel = torch.from_numpy(vel.copy()).pin_memory()
    h_mass = torch.from_numpy(mass).pin_memory()
    h_acc = torch.empty((n, 3), dtype=torch.float64).pin_memory()
    h_pot = torch.empty(n, dtype=torch.float64).pin_memory()
    xp, xv, xm, xa, xpot = (t.numpy() for t in (h_pos, h_vel, h_mass, h_acc, h_pot))
    ge = fx.Fmm(None, None, cfg["p"], 0.0, cfg["n_leaf"], **kw)
    L = fx.lib()

    def host_eval():
        stb = L.fmmx_build(ge._h, n, fx._ptr(xp), fx._ptr(xm))
        ste = L.fmmx_evaluate(ge._h, None, None, fx._ptr(xa), fx._ptr(xpot))
        assert stb == 0 and ste == 0, L.fmmx_last_error(ge._h)

    host_eval()
    dt = cfg["dt"]
    e2e_times = []
    for i in range(args.warmup + args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        # the host's kicks and drift, in place on the pinned buffers (torch's
        # CPU kernels use all host threads)
        h_vel.add_(h_acc, alpha=0.5 * dt)
        h_pos.add_(h_vel, alpha=dt)
        host_eval()
        h_vel.add_(h_acc, alpha=0.5 * dt)
        if i >= args.warmup:
            e2e_times.append((time.perf_counter() - t0) * 1e3)
    ge.close()

    # the M2L and P2P kernels alone on the device (one stream, nothing beside
    # them), for the roofline; in the timed steps the P2P runs beside the M2L
    solo = fx.Fmm(None, None, cfg["p"], 0.0, cfg["n_leaf"], **kw, overlap=False)
    m2l_solo, p2p_solo = [], []
    for i in range(2 + max(min(args.steps, 5), 1)):
        flush.zero_()
        solo.build_device(d_pos.data_ptr(), d_mass.data_ptr(), n)
        solo.evaluate_device(d_pos.data_ptr(), d_mass.data_ptr(), d_acc.data_ptr(), d_pot.data_ptr())
        if i >= 2:
            sst = solo.stats()
            m2l_solo.append(sst["ms_m2l"])
            p2p_solo.append(sst["ms_p2p"])
    solo.close()
    p99s = [float(np.percentile(e, 99)) for e in errs]
    p50s = [float(np.percentile(e, 50)) for e in errs]
    e2e_ms = max_over_ranks(float(np.mean(e2e_times)), world, cuda)
    return dict(times=times, total_ms=total_ms, st=st, e2e_ms=e2e_ms, p99s=p99s, p50s=p50s,
                m2l_ms=float(np.mean(m2l_solo)), p2p_ms=float(np.mean(p2p_solo)), m2l_ms_in_step=st["ms_m2l"],
                ntargets=len(tg), solo_st=sst)


def run_headline(args, cfg, rank, world, local_rank):
    import torch

    import fmms_b200 as fx

    dev = local_rank
    torch.cuda.set_device(dev)
    mass, pos, vel = make_inputs(fx, cfg, velocities=True)
    n = len(mass)
    tg = np.sort(np.random.default_rng(4096).choice(n, size=min(4096, n), replace=False)).astype(np.uint32)
    clk = ClockSampler(dev)
    main = measure_kdk(args, cfg, args.precision, mass, pos, vel, tg, dev, world, clk)
    other = None
    if not args.no_compare:
        other_prec = "plain" if args.precision == "mixed" else "mixed"
        other = measure_kdk(args, cfg, other_prec, mass, pos, vel, tg, dev, world)
    if rank != 0:
        return
    value = replicas_value(n, args.steps, main["total_ms"], world)
    st = main["st"]
    cpu = None
    if world == 1 and not args.no_cpu:
        nth = os.cpu_count() or 1
        bps, dt = cpu_fmm_sample(cfg, args.cpu_sample, nth)
        cpu = {"value": bps, "unit": "bodies/s", "cores": nth, "kind": "port",
               "sample": f"{args.cpu_sample} bodies of the same generator and settings, one tree build and "
                         f"threaded evaluation of the oracle's restatement of the reference FMM ({dt:.1f} s)"}
    fp64 = args.precision == "plain"
    line = {
        "metric": METRIC, "value": value, "unit": "bodies/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": main["total_ms"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if fp64 else "f32+f64", "data": "synthetic",
        "precision": args.precision, "config": bench_config(cfg, world, True),
        "step_ms_p50": float(np.percentile(main["times"], 50)),
        "step_ms_p99": float(np.percentile(main["times"], 99)),
        "force_err": {"p50": float(np.median(main["p50s"])), "p99": float(np.max(main["p99s"])),
                      "p99_per_step": main["p99s"], "targets": main["ntargets"],
                      "reference": "FP64 direct sum, after every timed step; p99 is the largest per-step p99"},
        "e2e": {"value": world * n / (main["e2e_ms"] * 1e-3), "unit": "bodies/s", "h2d_bytes_per_step": 32 * n,
                "d2h_bytes_per_step": 32 * n, "ms_per_step": main["e2e_ms"],
                "path": "host loop as the reference's energy gate: kick and drift on the host, fmmx_build "
                        "(Fmm::refresh) and fmmx_evaluate (Fmm::run) from pinned host buffers"},
        "gpu_launches": (int(st["kernel_launches"]) + 3) * args.steps,
        "stages_ms": {k[3:]: round(v, 3) for k, v in st.items() if k.startswith("ms_")},
        "counts": {k: int(st[k]) for k in ("n_cells", "n_leaves", "n_m2l", "n_p2p", "p2p_interactions")},
        "roofline": roofline(args, cfg, main, args.precision, dev), "cpu_baseline": cpu, "clocks": clk.summary(),
    }
    if other is not None:
        ov = replicas_value(n, args.steps, other["total_ms"], world)
        line["compare"] = {"precision": "plain" if args.precision == "mixed" else "mixed", "value": ov,
                           "ms_per_step": other["total_ms"] / args.steps,
                           "force_err_p50": float(np.median(other["p50s"])),
                           "force_err_p99": float(np.max(other["p99s"])),
                           "e2e_value": world * n / (other["e2e_ms"] * 1e-3),
                           "stages_ms": {k[3:]: round(v, 3) for k, v in other["st"].items() if k.startswith("ms_")},
                           "speedup_of_main": value / ov}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ C3: KDK
def run_kdk(args, cfg, rank, world, local_rank):
    """Clustered deep-tree workload: --kdk-steps (10) timed kick-drift-kick
    steps (dt = 1e-4) after --warmup untimed ones, mixed and plain, force
    error against the direct sum at every timed step."""
    import torch

    import fmms_b200 as fx

    dev = local_rank
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream()
    mass, pos, vel = fx.gen_clusters(cfg["n"], 64, 1e-3, 1e-1, SEEDS["clusters"])
    n = len(mass)
    rng = np.random.default_rng(4096)
    tg = np.sort(rng.choice(n, size=4096, replace=False)).astype(np.uint32)
    out = {}
    for prec in ([args.precision] + ([] if args.no_compare else ["plain" if args.precision == "mixed" else "mixed"])):
        d_pos = torch.from_numpy(pos.copy()).to(f"cuda:{dev}")
        d_vel = torch.from_numpy(vel.copy()).to(f"cuda:{dev}")
        d_mass = torch.from_numpy(mass).to(f"cuda:{dev}")
        d_acc = torch.empty((n, 3), dtype=torch.float64, device=f"cuda:{dev}")
        d_pot = torch.empty(n, dtype=torch.float64, device=f"cuda:{dev}")
        g = fx.Fmm(None, None, cfg["p"], 0.0, cfg["n_leaf"], mac="theta", theta=cfg["theta"],
                   softening=cfg["softening"], precision=prec, device=dev, stream=stream.cuda_stream)
        g.build_device(d_pos.data_ptr(), d_mass.data_ptr(), n)
        g.evaluate_device(d_pos.data_ptr(), d_mass.data_ptr(), d_acc.data_ptr(), d_pot.data_ptr())
        if args.warmup > 0:  # untimed steps: buffers reach their working sizes
            g.leapfrog_device(d_pos.data_ptr(), d_vel.data_ptr(), d_mass.data_ptr(), d_acc.data_ptr(),
                              d_pot.data_ptr(), 1e-4, args.warmup, "kdk", args.refresh_every)
        step_ms, errs = [], []
        for k in range(args.kdk_steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            g.leapfrog_device(d_pos.data_ptr(), d_vel.data_ptr(), d_mass.data_ptr(), d_acc.data_ptr(),
                              d_pot.data_ptr(), 1e-4, 1, "kdk", args.refresh_every)
            e1.record(stream)
            e1.synchronize()
            step_ms.append(e0.elapsed_time(e1))
            p_now = d_pos.cpu().numpy()
            a_ref, _, _ = fx.direct_targets(mass, p_now, tg, softening=cfg["softening"], device=dev)
            a = d_acc.cpu().numpy()[tg]
            rel = np.linalg.norm(a - a_ref, axis=1) / np.linalg.norm(a_ref, axis=1)
            errs.append({"p50": float(np.percentile(rel, 50)), "p99": float(np.percentile(rel, 99))})
        out[prec] = {"bodies_per_s": n * len(step_ms) / (sum(step_ms) * 1e-3), "step_ms": step_ms,
                     "force_err_per_step": errs, "stages_ms_last": {k[3:]: round(v, 3) for k, v in g.stats().items()
                                                                    if k.startswith("ms_")}}
        g.close()
    if rank != 0:
        return
    main = out[args.precision]
    line = {"metric": METRIC, "value": main["bodies_per_s"], "unit": "bodies/s", "n_gpus": world,
            "steps": args.kdk_steps, "warmup": args.warmup, "ms_per_step": float(np.mean(main["step_ms"])),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "data": "synthetic",
            "dtype": "f64" if args.precision == "plain" else "f32+f64",
            "config": {"workload": cfg["workload"] + f", {args.kdk_steps} KDK steps dt=1e-4 after {args.warmup} untimed",
                       "refresh_every": args.refresh_every},
            "step_ms_p50": float(np.percentile(main["step_ms"], 50)),
            "step_ms_p99": float(np.percentile(main["step_ms"], 99)), "kdk": out}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ graphs on a reused tree
def run_graphs(args, cfg, rank, world, local_rank):
    """Device leapfrog on the given configuration with tree reuse
    (refresh_every, default 8): steps launched one by one against steps
    replayed from a CUDA graph, same inputs, mixed precision."""
    import torch

    import fmms_b200 as fx

    if rank != 0:
        return
    dev = local_rank
    torch.cuda.set_device(dev)
    mass, pos = make_inputs(fx, cfg)
    n = len(mass)
    vel = np.zeros_like(pos)
    refresh = args.refresh_every if args.refresh_every > 1 else 8
    res = {}
    side = torch.cuda.Stream(device=dev)
    with torch.cuda.stream(side):
        for graphs in (False, True):
            d_pos = torch.from_numpy(pos.copy()).to(f"cuda:{dev}")
            d_vel = torch.from_numpy(vel.copy()).to(f"cuda:{dev}")
            d_mass = torch.from_numpy(mass).to(f"cuda:{dev}")
            d_acc = torch.empty((n, 3), dtype=torch.float64, device=f"cuda:{dev}")
            d_pot = torch.empty(n, dtype=torch.float64, device=f"cuda:{dev}")
            g = fx.Fmm(None, None, cfg["p"], 0.0, cfg["n_leaf"], mac="theta", theta=cfg["theta"],
                       softening=cfg["softening"], precision=args.precision, device=dev,
                       stream=side.cuda_stream, use_graphs=graphs)
            g.build_device(d_pos.data_ptr(), d_mass.data_ptr(), n)
            g.evaluate_device(d_pos.data_ptr(), d_mass.data_ptr(), d_acc.data_ptr(), d_pot.data_ptr())
            g.leapfrog_device(d_pos.data_ptr(), d_vel.data_ptr(), d_mass.data_ptr(), d_acc.data_ptr(),
                              d_pot.data_ptr(), 1e-3, refresh, "kdk", refresh)  # warm-up cycle
            steps = refresh * 8
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(side)
            g.leapfrog_device(d_pos.data_ptr(), d_vel.data_ptr(), d_mass.data_ptr(), d_acc.data_ptr(),
                              d_pot.data_ptr(), 1e-3, steps, "kdk", refresh)
            e1.record(side)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / steps
            res["graphs" if graphs else "launches"] = {"ms_per_step": ms, "bodies_per_s": n / (ms * 1e-3),
                                                       "final_pos_checksum": float(d_pos.sum().item())}
            g.close()
    main = res["graphs"]
    line = {"metric": METRIC, "value": main["bodies_per_s"], "unit": "bodies/s", "n_gpus": 1, "steps": refresh * 8,
            "warmup": refresh, "ms_per_step": main["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "data": "synthetic", "dtype": "f64" if args.precision == "plain" else "f32+f64",
            "config": {"workload": cfg["workload"] + f", KDK dt=1e-3, tree refreshed every {refresh} steps",
                       "precision": args.precision},
            "graphs": res, "speedup": res["launches"]["ms_per_step"] / main["ms_per_step"]}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ C3: same-error comparison
# (p, theta, soft_gap): soft_gap > 0 keeps M2L pairs soft_gap * softening apart
SWEEP_SETTINGS = ((12, 0.4, 0.0), (16, 0.4, 0.0), (12, 0.3, 0.0), (12, 0.4, 100.0), (12, 0.4, 300.0),
                  (10, 0.5, 100.0), (10, 0.5, 200.0), (10, 0.5, 300.0), (8, 0.5, 300.0), (8, 0.4, 300.0),
                  (10, 0.6, 300.0), (12, 0.5, 300.0))


def run_accuracy_sweep(args, cfg, rank, world, local_rank):
    """The clustered workload's force evaluation at several (p, theta) in both
    precisions: bodies/s and p99 relative error against the FP64 direct sum
    on 4096 seeded targets; then, per precision, the fastest setting whose p99
    error is <= 1e-5, and the ratio of the two (mixed over plain at the same
    error bound)."""
    import torch

    import fmms_b200 as fx

    if rank != 0:
        return
    dev = local_rank
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream()
    mass, pos, _ = fx.gen_clusters(cfg["n"], 64, 1e-3, 1e-1, SEEDS["clusters"])
    n = len(mass)
    tg = np.sort(np.random.default_rng(4096).choice(n, size=4096, replace=False)).astype(np.uint32)
    a_ref, _, _ = fx.direct_targets(mass, pos, tg, softening=cfg["softening"], device=dev)
    d_pos = torch.from_numpy(pos).to(f"cuda:{dev}")
    d_mass = torch.from_numpy(mass).to(f"cuda:{dev}")
    d_acc = torch.empty((n, 3), dtype=torch.float64, device=f"cuda:{dev}")
    d_pot = torch.empty(n, dtype=torch.float64, device=f"cuda:{dev}")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{dev}")
    rows = []
    for prec in ("mixed", "plain"):
        for p, theta, gap in SWEEP_SETTINGS:
            g = fx.Fmm(None, None, p, 0.0, cfg["n_leaf"], mac="theta", theta=theta, softening=cfg["softening"],
                       precision=prec, device=dev, stream=stream.cuda_stream, soft_gap=gap)
            ms = []
            for it in range(3):  # one warm-up, two timed
                flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                g.build_device(d_pos.data_ptr(), d_mass.data_ptr(), n)
                g.evaluate_device(d_pos.data_ptr(), d_mass.data_ptr(), d_acc.data_ptr(), d_pot.data_ptr())
                e1.record(stream)
                e1.synchronize()
                if it:
                    ms.append(e0.elapsed_time(e1))
            a = d_acc.cpu().numpy()[tg]
            rel = np.linalg.norm(a - a_ref, axis=1) / np.linalg.norm(a_ref, axis=1)
            st = g.stats()
            g.close()
            rows.append({"precision": prec, "p": p, "theta": theta, "soft_gap": gap, "ms": float(np.mean(ms)),
                         "bodies_per_s": n / (np.mean(ms) * 1e-3), "err_p50": float(np.percentile(rel, 50)),
                         "err_p99": float(np.percentile(rel, 99)), "m2l_ms": st["ms_m2l"], "p2p_ms": st["ms_p2p"],
                         "n_m2l": int(st["n_m2l"]), "p2p_interactions": int(st["p2p_interactions"])})
            print(json.dumps(rows[-1]), file=sys.stderr, flush=True)
    best = {}
    for prec in ("mixed", "plain"):
        ok = [r for r in rows if r["precision"] == prec and r["err_p99"] <= 1e-5]
        best[prec] = max(ok, key=lambda r: r["bodies_per_s"]) if ok else None
    ratio = (best["mixed"]["bodies_per_s"] / best["plain"]["bodies_per_s"]
             if best["mixed"] and best["plain"] else None)
    main = best["mixed"] or max((r for r in rows if r["precision"] == "mixed"), key=lambda r: -r["err_p99"])
    line = {"metric": METRIC, "value": main["bodies_per_s"], "unit": "bodies/s", "n_gpus": 1, "steps": 2,
            "warmup": 1, "ms_per_step": main["ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "data": "synthetic", "dtype": "f32+f64",
            "config": {"workload": cfg["workload"].split(", p=")[0] + ", one force evaluation per setting",
                       "settings_p_theta_softgap": [list(t) for t in SWEEP_SETTINGS], "n_leaf": cfg["n_leaf"],
                       "l2": "flushed between timed evaluations"},
            "same_error": {"bound_p99": 1e-5, "mixed": best["mixed"], "plain": best["plain"],
                           "mixed_over_plain": ratio},
            "sweep": rows}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ C4: ensemble
def run_ensemble(args, cfg, rank, world, local_rank):
    """512 independent Plummer spheres (N log-uniform in [1e3, 1e5], scale
    radius U[0.5, 2], mass 1 each) in one forest; per-system error on 256
    seeded targets each."""
    import torch

    import fmms_b200 as fx

    dev = local_rank
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream()
    rng = np.random.default_rng(512)
    sizes = np.exp(rng.uniform(np.log(1e3), np.log(1e5), args.nsys)).astype(np.int64)
    radii = rng.uniform(0.5, 2.0, args.nsys)
    parts = [fx.gen_plummer_ic(int(nn), 1.0, float(a), 20.0, 1000 + i, velocities=False)[:2]
             for i, (nn, a) in enumerate(zip(sizes, radii))]
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint64)
    mass = np.concatenate([m for m, _ in parts])
    pos = np.concatenate([p for _, p in parts])
    n = len(mass)
    tune = None
    n_leaf, p_use, tile, theta, gap = cfg["n_leaf"], cfg["p"], 0, cfg["theta"], 0.0
    if args.autotune:
        from fmms_b200.autotune import tune_ensemble

        tune = tune_ensemble(parts, p=cfg["p"], theta=cfg["theta"], softening=cfg["softening"],
                             precision=args.precision, device=dev)
        n_leaf, p_use, tile, theta, gap = tune["n_leaf"], tune["p"], tune["p2p_tile"], tune["theta"], tune["soft_gap"]
    d_pos = torch.from_numpy(pos).to(f"cuda:{dev}")
    d_mass = torch.from_numpy(mass).to(f"cuda:{dev}")
    d_acc = torch.empty((n, 3), dtype=torch.float64, device=f"cuda:{dev}")
    d_pot = torch.empty(n, dtype=torch.float64, device=f"cuda:{dev}")
    g = fx.Fmm(None, None, p_use, 0.0, n_leaf, mac="theta", theta=theta, softening=cfg["softening"],
               precision=args.precision, device=dev, stream=stream.cuda_stream, p2p_tile=tile, soft_gap=gap)

    def step():
        g.build_ensemble_device(off, d_pos.data_ptr(), d_mass.data_ptr())
        g.evaluate_device(d_pos.data_ptr(), d_mass.data_ptr(), d_acc.data_ptr(), d_pot.data_ptr())

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    times = []
    for _ in range(args.steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    acc = d_acc.cpu().numpy()
    p99s = []
    for i, (m, p) in enumerate(parts):
        t = np.sort(np.random.default_rng(i).choice(len(m), size=min(256, len(m)), replace=False)).astype(np.uint32)
        a_ref, _, _ = fx.direct_targets(m, p, t, softening=cfg["softening"], device=dev)
        a = acc[int(off[i]):int(off[i + 1])][t]
        rel = np.linalg.norm(a - a_ref, axis=1) / np.linalg.norm(a_ref, axis=1)
        p99s.append(float(np.percentile(rel, 99)))
    if rank != 0:
        return
    st = g.stats()
    ms = float(np.mean(times))
    line = {"metric": METRIC, "value": n / (ms * 1e-3), "unit": "bodies/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "data": "synthetic", "dtype": "f64" if args.precision == "plain" else "f32+f64",
            "config": {"workload": f"{args.nsys} Plummer systems, N log-uniform[1e3,1e5] (total {n}), one forest",
                       "p": p_use, "n_leaf": n_leaf, "p2p_tile": tile, "theta": theta, "soft_gap": gap,
                       "autotune": {k: v for k, v in (tune or {}).items() if k != "candidates"},
                       "autotune_candidates": [[c["theta"], c["soft_gap"], c["p"], c["n_leaf"], c["p2p_tile"],
                                                round(c["ms"], 2), float("%.3g" % c["err_p99_worst"])]
                                               for c in (tune or {}).get("candidates", [])],
                       "autotune_candidate_fields": ["theta", "soft_gap", "p", "n_leaf", "p2p_tile",
                                                     "ms (sampled forest)", "p99 err (worst sampled system)"]},
            "per_system_force_err_p99": {"median": float(np.median(p99s)), "max": float(np.max(p99s)),
                                         "systems_over_1e-5": int(np.sum(np.asarray(p99s) > 1e-5))},
            "launches_per_evaluation": int(st["kernel_launches"]),
            "stages_ms": {k[3:]: round(v, 3) for k, v in st.items() if k.startswith("ms_")},
            "gpu_launches": int(st["kernel_launches"]) * args.steps}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ C5: serving
def run_serve(args, cfg, rank, world, local_rank):
    """Poisson arrivals (args.rate per second for args.duration seconds) of
    Plummer or uniform-cube sessions (50/50), N log-uniform in [1e3, 1e6], 100
    KDK steps of dt = 1e-3 each, admitted under the HBM budget."""
    import fmms_b200 as fx
    from fmms_b200.serve import Server, Session, run_session_alone, worst_intervals

    if rank != 0:
        return
    rng = np.random.default_rng(5)
    arrivals = np.cumsum(rng.exponential(1.0 / args.rate, size=int(args.rate * args.duration * 2) + 10))
    arrivals = arrivals[arrivals < args.duration]
    sessions = []
    for i, t in enumerate(arrivals):
        nn = int(np.exp(rng.uniform(np.log(1e3), np.log(args.serve_nmax))))
        if rng.random() < 0.5:
            m, p, v = fx.gen_plummer_ic(nn, 1.0, 1.0, 20.0, 7000 + i)
        else:
            m, p = fx.gen_uniform_lognormal(nn, 0.5, 7000 + i)
            v = np.zeros_like(p)
        sessions.append(Session(sid=i, mass=m, pos=p, vel=v, steps=args.serve_steps, dt=1e-3, arrival=float(t)))
    kw = dict(p=cfg["p"], theta=cfg["theta"], softening=cfg["softening"], n_leaf=cfg["n_leaf"],
              precision=args.precision, budget_bytes=args.budget_gb * 1e9, refresh_every=args.refresh_every)
    srv = Server(**kw, latency_slo=args.latency_slo,  # calibrates the isolated step time first
                 headroom=args.headroom if args.headroom > 0 else None)
    srv.start()  # every lane on its own thread and stream
    t0 = time.perf_counter()
    k = 0
    occ = []  # (sessions, bodies) admitted, sampled every 2 ms while arrivals last
    while True:
        now = time.perf_counter() - t0
        while k < len(sessions) and sessions[k].arrival <= now:
            srv.submit(sessions[k])
            k += 1
        if now <= args.duration:
            act = srv.active
            occ.append((len(act), sum(s.n for s in act)))
        if now > args.duration and (not srv.busy() or now > args.duration + args.drain):
            break
        time.sleep(0.002)
    srv.stop()
    wall = time.perf_counter() - t0
    rep = srv.report()
    rep["bodies_per_s"] = rep["bodies_stepped"] / wall
    # isolated step latency of completed sessions of every lane, against the mix
    ratios = []
    by_n = sorted(srv.done, key=lambda s: s.n)  # evenly spaced over the sizes that finished
    picked = [by_n[i] for i in sorted({int(round(j)) for j in np.linspace(0, len(by_n) - 1, args.isolated_samples)})] \
        if by_n else []
    for s in picked:
        _, _, alone_ms = run_session_alone(s, **kw)
        a50 = float(np.percentile(alone_ms, 50))
        ratios.append({"n": s.n, "mix_p99_ms": float(np.percentile(s.step_ms, 99)), "alone_p50_ms": a50,
                       "alone_p99_ms": float(np.percentile(alone_ms, 99)),
                       "mix_p50_ms": float(np.percentile(s.step_ms, 50)), "mix_max_ms": float(np.max(s.step_ms)),
                       "steps_over_2x": int(np.sum(np.asarray(s.step_ms) > 2 * a50)), "steps": len(s.step_ms)})
    # like for like: the p99 step latency in the mix over the p99 of the same
    # session alone (with a tree refreshed every few steps, the rebuild steps
    # are the p99 of both); and over the isolated median
    rr = [r["mix_p99_ms"] / max(r["alone_p99_ms"], 1e-6) for r in ratios]
    rr50 = [r["mix_p99_ms"] / max(r["alone_p50_ms"], 1e-6) for r in ratios]
    # batching: sessions per tick of the ticks that stepped a batch (trace field 6: members)
    per_tick = [t[6] for ln in srv.lanes for t in ln.trace]
    batching = {"ticks": len(per_tick),
                "sessions_per_tick_mean": float(np.mean(per_tick)) if per_tick else 0.0,
                "ticks_with_more_than_one": float(np.mean([m > 1 for m in per_tick])) if per_tick else 0.0,
                "sessions_per_tick_max": int(max(per_tick)) if per_tick else 0}
    line = {"metric": METRIC, "value": rep["bodies_per_s"], "unit": "bodies/s", "n_gpus": 1, "steps": rep["ticks"],
            "warmup": 0, "ms_per_step": rep["step_ms_p50"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "data": "synthetic",
            "dtype": "f64" if args.precision == "plain" else "f32+f64",
            "config": {"workload": f"serving: Poisson {args.rate}/s for {args.duration}s, N log-uniform[1e3,"
                                   f"{args.serve_nmax:.0e}], {args.serve_steps} KDK steps", "budget_gb": args.budget_gb,
                       "refresh_every": args.refresh_every},
            "serve": {**rep, "wall_s": wall, "arrived": len(sessions), "submitted": k, "batching": batching,
                      "queued_at_end": len(srv.queue), "active_at_end": len(srv.active),
                      "admitted_sessions_mean": float(np.mean([o[0] for o in occ])) if occ else 0.0,
                      "admitted_bodies_mean": float(np.mean([o[1] for o in occ])) if occ else 0.0,
                      "lanes": [{"n_from": ln.lo, "stream_priority": ln.priority, "ticks": len(ln.tick_ms),
                                 "joins_undone": ln.evictions, "worst_intervals": worst_intervals(ln.trace, copies=srv.copy_log),
                                 "tick_ms_p50": float(np.percentile(ln.tick_ms, 50)) if ln.tick_ms else None}
                                for ln in srv.lanes],
                      "p99_over_isolated": {"median": float(np.median(rr)) if rr else None,
                                            "max": float(np.max(rr)) if rr else None,
                                            "definition": "mix p99 step ms / the same session alone, p99 step ms"},
                      "p99_over_isolated_p50": {"median": float(np.median(rr50)) if rr50 else None,
                                                "max": float(np.max(rr50)) if rr50 else None,
                                                "definition": "mix p99 step ms / the same session alone, p50 step ms"},
                      "isolated_samples": ratios}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="fmmx", choices=["fmmx", "reference"])
    ap.add_argument("--config", default="c3", choices=sorted(CONFIGS) + ["c4", "c5"])
    ap.add_argument("--precision", default="mixed", choices=["plain", "mixed"])
    ap.add_argument("--no-compare", action="store_true", help="skip the other precision's run")
    ap.add_argument("--kdk-steps", type=int, default=10)
    ap.add_argument("--refresh-every", type=int, default=1)
    ap.add_argument("--nsys", type=int, default=512)
    ap.add_argument("--autotune", action="store_true")
    ap.add_argument("--rate", type=float, default=50.0)
    ap.add_argument("--duration", type=float, default=60.0)
    ap.add_argument("--drain", type=float, default=20.0)
    ap.add_argument("--serve-steps", type=int, default=100)
    ap.add_argument("--serve-nmax", type=float, default=1e6)
    ap.add_argument("--budget-gb", type=float, default=160.0)
    ap.add_argument("--isolated-samples", type=int, default=10)
    ap.add_argument("--latency-slo", type=float, default=2.0)
    ap.add_argument("--headroom", type=float, default=0.0,
                    help="c5: admission bound as a multiple of isolated latency (0: 0.8 x latency-slo)")
    ap.add_argument("--m2l", default="auto", choices=["auto", "naive", "rotation"])
    ap.add_argument("--cpu-sample", type=int, default=262144)
    ap.add_argument("--ref-budget-s", type=float, default=150.0,
                    help="--impl reference: stop timing full-size steps once this many seconds have passed")
    ap.add_argument("--ref-sample", type=int, default=0,
                    help="--impl reference: time an N-body sample instead of the full system (0: full)")
    ap.add_argument("--kdk", action="store_true",
                    help="c3: the earlier KDK report at the configured p=12, theta=0.4 (no accuracy bound)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--n", type=int, default=0, help="override N (small cases for profiling)")
    ap.add_argument("--graphs", action="store_true",
                    help="device leapfrog with tree reuse: launches against CUDA-graph replay")
    ap.add_argument("--sweep", action="store_true",
                    help="c3: force evaluations at several (p, theta) in both precisions, compared at p99 <= 1e-5")
    args = ap.parse_args()
    headline = args.config == "c3" and not (args.sweep or args.kdk or args.graphs)
    cfg = dict(HEADLINE if headline else (CONFIGS.get(args.config) or EXTRA_CONFIGS[args.config]))
    if args.n > 0:
        cfg["n"] = args.n
        cfg["workload"] += f" (N overridden: {args.n})"
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, cfg, rank, headline)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        runner = {"c3": run_headline if headline else (run_accuracy_sweep if args.sweep else run_kdk),
                  "c4": run_ensemble, "c5": run_serve}.get(args.config, run_gpu)
        if args.graphs:
            runner = run_graphs
        runner(args, cfg, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
