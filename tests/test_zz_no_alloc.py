"""The allocation-free direct sum (fmmx_direct_targets_noalloc) against the
allocating entry point (fmmx_direct_targets).

The no-alloc form is for callers that cannot allocate device memory: a physics
step in a fixed-latency frame loop, where cudaMalloc/cudaFree can block and
synchronise the device, and hosts whose device memory belongs to their own pool
allocator. Its scratch is a static device array, shared by every call, so the
test makes two calls in a row with different inputs and checks both against
the allocating form, within the 1e-12 relative tolerance of the other direct
sum tests. This file is collected last so that a failure here cannot hide
another test's result; it also passes alone in a fresh process.
"""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    if b.ndim > 1:
        return np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)
    return np.abs(a - b) / np.abs(b)


def test_noalloc_direct_matches_allocating_form_on_two_calls():
    import torch

    import fmms_b200 as fx

    stream = torch.cuda.current_stream()
    cases = [(20000, 3, 4096, 1e-3), (7001, 9, 1500, 0.0)]
    for n, seed, nt, soft in cases:
        mass, pos = fx.gen_plummer(n, seed=seed)
        t = np.sort(np.random.default_rng(seed).choice(n, size=nt, replace=False)).astype(np.uint32)
        a_ref, p_ref, f_ref = fx.direct_targets(mass, pos, t, softening=soft)

        d_pos = torch.from_numpy(pos).cuda()
        d_mass = torch.from_numpy(mass).cuda()
        d_t = torch.from_numpy(t.view(np.int32)).cuda()
        d_acc = torch.full((nt, 3), float("nan"), dtype=torch.float64, device="cuda")
        d_pot = torch.full((nt,), float("nan"), dtype=torch.float64, device="cuda")
        d_f = torch.full((nt,), float("nan"), dtype=torch.float64, device="cuda")
        fx.direct_targets_noalloc(n, d_pos.data_ptr(), d_mass.data_ptr(), nt, d_t.data_ptr(), d_acc.data_ptr(),
                                  d_pot.data_ptr(), d_f.data_ptr(), softening=soft, device=0,
                                  stream=stream.cuda_stream)
        stream.synchronize()
        assert np.max(_rel(d_acc.cpu().numpy(), a_ref)) < TOL
        assert np.max(_rel(d_pot.cpu().numpy(), p_ref)) < TOL
        assert np.max(_rel(d_f.cpu().numpy(), f_ref)) < TOL


def test_noalloc_out_of_range_target_is_nan_only_there():
    """A target id >= n cannot be checked on the host (the ids are in device
    memory): that target's results are NaN, every other target's are exact."""
    import torch

    import fmms_b200 as fx

    stream = torch.cuda.current_stream()
    n, nt = 5000, 64
    mass, pos = fx.gen_plummer(n, seed=31)
    t = np.arange(0, 2 * nt, 2, dtype=np.uint32)
    a_ref, p_ref, f_ref = fx.direct_targets(mass, pos, t, softening=1e-3)
    bad = t.copy()
    bad[5] = n + 7
    d_pos = torch.from_numpy(pos).cuda()
    d_mass = torch.from_numpy(mass).cuda()
    d_t = torch.from_numpy(bad.view(np.int32)).cuda()
    d_acc = torch.zeros((nt, 3), dtype=torch.float64, device="cuda")
    d_pot = torch.zeros((nt,), dtype=torch.float64, device="cuda")
    d_f = torch.zeros((nt,), dtype=torch.float64, device="cuda")
    fx.direct_targets_noalloc(n, d_pos.data_ptr(), d_mass.data_ptr(), nt, d_t.data_ptr(), d_acc.data_ptr(),
                              d_pot.data_ptr(), d_f.data_ptr(), softening=1e-3, device=0, stream=stream.cuda_stream)
    stream.synchronize()
    acc, pot, f = d_acc.cpu().numpy(), d_pot.cpu().numpy(), d_f.cpu().numpy()
    ok = np.arange(nt) != 5
    assert np.all(np.isnan(acc[5])) and np.isnan(pot[5]) and np.isnan(f[5])
    assert np.max(_rel(acc[ok], a_ref[ok])) < TOL
    assert np.max(_rel(pot[ok], p_ref[ok])) < TOL
    assert np.max(_rel(f[ok], f_ref[ok])) < TOL


def test_noalloc_rejects_more_targets_than_its_scratch_holds():
    import fmms_b200 as fx

    st = fx.lib().fmmx_direct_targets_noalloc(0, None, 10, 1, 1, 0.0, fx.DIRECT_NOALLOC_MAX_TARGETS + 1, 1, 1,
                                             None, None)
    assert st == 1  # FMMX_INVALID_ARG, before touching any pointer
