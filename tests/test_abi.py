"""CPU checks of the C-ABI boundary: the library loads, exports every symbol
include/fmmx.h declares, and refuses work cleanly without a device."""

import ctypes as C
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "fmmx.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(fmmx_[a-z_0-9]+)\s*\(", txt)))


def test_library_exports_every_header_symbol():
    import fmms_b200

    L = fmms_b200.lib()
    syms = header_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(L, s), f"{s} missing from libfmmx.so"
    assert set(syms) == set(fmms_b200.SIGNATURES), "ctypes signatures out of sync with fmmx.h"


def test_config_default_and_status_strings():
    import fmms_b200 as fx

    cfg = fx.Config()
    fx.lib().fmmx_config_default(C.byref(cfg))
    assert cfg.p == 8 and cfg.n_leaf == 16 and cfg.mac_mode == fx.MAC_DEHNEN and cfg.precision == fx.PLAIN_FP64
    assert fx.lib().fmmx_status_string(0) == b"ok"
    assert fx.lib().fmmx_status_string(8) == b"no CUDA device"


def test_create_rejects_bad_config_before_touching_a_device():
    import fmms_b200 as fx

    cfg = fx.Config()
    fx.lib().fmmx_config_default(C.byref(cfg))
    h = C.c_void_p()
    for field, bad in (("p", 0), ("p", 99), ("n_leaf", -1), ("mac_mode", 7), ("precision", 5)):
        c2 = fx.Config.from_buffer_copy(cfg)
        setattr(c2, field, bad)
        assert fx.lib().fmmx_create(C.byref(c2), C.byref(h)) == 1
    c3 = fx.Config.from_buffer_copy(cfg)
    c3.mac_mode = fx.MAC_THETA
    c3.theta = 0.0
    assert fx.lib().fmmx_create(C.byref(c3), C.byref(h)) == 1


def test_null_context_calls_fail_cleanly():
    import fmms_b200 as fx

    L = fx.lib()
    assert L.fmmx_build(None, 10, None, None) == 1
    assert L.fmmx_evaluate(None, None, None, None, None) == 1
    assert L.fmmx_get_stats(None, None) == 1
    assert L.fmmx_last_error(None) == b"null context"


def test_generator_matches_reference_sampler(orc):
    """fmmx_gen_plummer reproduces models::plummer bit for bit."""
    import fmms_b200 as fx

    for seed in (1, 42, 1234):
        m1, p1 = fx.gen_plummer(5000, seed=seed)
        m2, p2 = orc.plummer(5000, seed=seed)
        assert np.array_equal(m1, m2) and np.array_equal(p1, p2)
    m1, p1 = fx.gen_hernquist(3000, center=(1.0, -2.0, 0.5), seed=7)
    m2, p2 = orc.hernquist(3000, center=(1.0, -2.0, 0.5), seed=7)
    assert np.array_equal(p1, p2)


def test_noalloc_limit_matches_header():
    """The Python constant of the allocation-free direct sum's target limit is
    the header's FMMX_DIRECT_NOALLOC_MAX_TARGETS."""
    import fmms_b200 as fx

    txt = open(os.path.join(ROOT, "include", "fmmx.h")).read()
    m = re.search(r"#define\s+FMMX_DIRECT_NOALLOC_MAX_TARGETS\s+(\d+)", txt)
    assert m and int(m.group(1)) == fx.DIRECT_NOALLOC_MAX_TARGETS


def test_config_and_stats_layout_match_header():
    """The ctypes structures hold every field of fmmx_config and fmmx_stats,
    in the header's order (new fields appended at the end)."""
    import fmms_b200 as fx

    txt = open(os.path.join(ROOT, "include", "fmmx.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    for name, cls in (("fmmx_config", fx.Config), ("fmmx_stats", fx.Stats)):
        body = re.search(r"typedef struct " + name + r" \{(.*?)\} " + name + ";", txt, flags=re.S).group(1)
        fields = re.findall(r"\b([a-z_0-9]+)\s*;", body)
        assert fields == [f for f, _ in cls._fields_], name
