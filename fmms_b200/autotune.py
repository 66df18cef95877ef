"""Autotuner for the batched ensemble: picks the leaf capacity, the expansion
order and the P2P tile shape that evaluate a forest fastest while every
sampled system keeps its p99 relative force error within the target.

It times one forest build + evaluation per candidate on a subsample of the
systems (every k-th, so the size mix is kept) and checks the error against the
FP64 direct sum on 64 seeded targets per sampled system. No reference
counterpart (the reference has no tuner).
"""

from __future__ import annotations

import time

import numpy as np


def _forest(parts):
    off = np.concatenate([[0], np.cumsum([len(m) for m, _ in parts])]).astype(np.uint64)
    mass = np.concatenate([m for m, _ in parts])
    pos = np.concatenate([p for _, p in parts])
    return off, mass, pos


def tune_ensemble(parts, *, p=8, theta=0.5, softening=1e-3, precision="mixed", device=0, err_target=1e-5,
                  leaves=(16, 32, 48, 64, 96, 128), orders=None, tiles=(128, 256), sample_every=8, repeats=2):
    import torch

    import fmms_b200 as fx

    sample = parts[::sample_every] or parts[:1]
    off, mass, pos = _forest(sample)
    n = len(mass)
    torch.cuda.set_device(device)
    stream = torch.cuda.current_stream()
    d_pos = torch.from_numpy(pos).to(f"cuda:{device}")
    d_mass = torch.from_numpy(mass).to(f"cuda:{device}")
    d_acc = torch.empty((n, 3), dtype=torch.float64, device=f"cuda:{device}")
    d_pot = torch.empty(n, dtype=torch.float64, device=f"cuda:{device}")
    # direct-sum references on a few targets per sampled system
    refs = []
    for i, (m, q) in enumerate(sample):
        t = np.sort(np.random.default_rng(i).choice(len(m), size=min(64, len(m)), replace=False)).astype(np.uint32)
        a_ref, _, _ = fx.direct_targets(m, q, t, softening=softening, device=device)
        refs.append((t, a_ref))
    orders = orders or (max(2, p - 2), p, min(16, p + 2))
    cands = []
    for pp in orders:
        for nl in leaves:
            for tile in tiles:
                g = fx.Fmm(None, None, pp, 0.0, nl, mac="theta", theta=theta, softening=softening,
                           precision=precision, device=device, stream=stream.cuda_stream, p2p_tile=tile)
                best = float("inf")
                for _ in range(repeats + 1):
                    torch.cuda.synchronize()
                    t0 = time.perf_counter()
                    g.build_ensemble_device(off, d_pos.data_ptr(), d_mass.data_ptr())
                    g.evaluate_device(d_pos.data_ptr(), d_mass.data_ptr(), d_acc.data_ptr(), d_pot.data_ptr())
                    torch.cuda.synchronize()
                    best = min(best, time.perf_counter() - t0)
                g.close()
                acc = d_acc.cpu().numpy()
                worst = 0.0
                for i, (t, a_ref) in enumerate(refs):
                    a = acc[int(off[i]):int(off[i + 1])][t]
                    rel = np.linalg.norm(a - a_ref, axis=1) / np.linalg.norm(a_ref, axis=1)
                    worst = max(worst, float(np.percentile(rel, 99)))
                cands.append({"p": pp, "n_leaf": nl, "p2p_tile": tile, "ms": best * 1e3, "err_p99_worst": worst})
    ok = [c for c in cands if c["err_p99_worst"] <= err_target]
    if ok:
        pick = min(ok, key=lambda c: c["ms"])
    else:  # nothing meets the target: the most accurate, then the fastest of those
        best_err = min(c["err_p99_worst"] for c in cands)
        pick = min((c for c in cands if c["err_p99_worst"] <= 1.05 * best_err), key=lambda c: c["ms"])
    return {"p": pick["p"], "n_leaf": pick["n_leaf"], "p2p_tile": pick["p2p_tile"], "met_target": bool(ok),
            "err_target": err_target, "sampled_systems": len(sample), "candidates": cands}
