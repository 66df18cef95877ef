"""The oracle: test infrastructure only.

A ctypes front end to ``liboracle.so``, the C++ restatement of the reference
FMM (crates/fmm of Vedant9500/FMMS) in ``fmm_oracle.cpp``. Only the tests, the
smoke check and the benchmark's CPU-baseline leg use it, and only as the
checker; the engine never imports it.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None

_dp = C.POINTER(C.c_double)
_u32p = C.POINTER(C.c_uint32)
_i32p = C.POINTER(C.c_int32)
_u64p = C.POINTER(C.c_uint64)
_sz = C.c_size_t


def build() -> str:
    """Compile liboracle.so from fmm_oracle.cpp (make, in this directory)."""
    subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    return _LIB


def _ptr(a, t):
    return a.ctypes.data_as(t) if a is not None else None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(
            os.path.join(_HERE, "fmm_oracle.cpp")
        ):
            build()
        L = C.CDLL(_LIB)
        L.orc_plummer.argtypes = [_sz, C.c_double, C.c_double, C.c_double, C.c_uint64, _dp, _dp]
        L.orc_hernquist.argtypes = [_sz, C.c_double, C.c_double, C.c_double, C.c_uint64, _dp, _dp]
        L.orc_rng_units.argtypes = [C.c_uint64, _sz, _dp]
        L.orc_gen_plummer_ic.argtypes = [_sz, C.c_double, C.c_double, C.c_double, C.c_uint64, _dp, _dp, _dp]
        L.orc_gen_uniform_lognormal.argtypes = [_sz, C.c_double, C.c_uint64, _dp, _dp]
        L.orc_gen_clusters.argtypes = [_sz, C.c_int, C.c_double, C.c_double, C.c_uint64, _dp, _dp, _dp]
        L.orc_theta_table.argtypes = [_dp, _sz, _dp]
        L.orc_upsilon_table.argtypes = [_dp, _sz, _dp]
        L.orc_dilate.argtypes = [C.c_uint64]
        L.orc_dilate.restype = C.c_uint64
        L.orc_factorials.argtypes = [_sz, _dp]
        L.orc_binomials.argtypes = [_sz, _dp]
        L.orc_blocksum.argtypes = [_sz]
        L.orc_blocksum.restype = _sz
        L.orc_swap_matrices.argtypes = [_sz, _dp]
        L.orc_fmm_new.argtypes = [_sz, _dp, _dp, _sz, C.c_int, C.c_double, C.c_double, C.c_double, _sz, C.c_int]
        L.orc_fmm_new.restype = C.c_void_p
        L.orc_fmm_refresh.argtypes = [C.c_void_p, _sz, _dp, _dp]
        L.orc_fmm_free.argtypes = [C.c_void_p]
        L.orc_fmm_set_gap.argtypes = [C.c_void_p, C.c_double]
        L.orc_fmm_run.argtypes = [C.c_void_p, _sz, _dp, _dp, C.c_int, _dp, _dp]
        L.orc_fmm_walk.argtypes = [C.c_void_p, _sz, _dp, _dp, C.c_int]
        L.orc_fmm_ncells.argtypes = [C.c_void_p]
        L.orc_fmm_ncells.restype = _sz
        L.orc_fmm_cells.argtypes = [C.c_void_p, _u32p, _i32p, _dp, _dp, _dp]
        L.orc_fmm_order.argtypes = [C.c_void_p, _u32p, _u64p]
        L.orc_fmm_bbox.argtypes = [C.c_void_p, _dp]
        L.orc_fmm_moments.argtypes = [C.c_void_p, _dp]
        L.orc_fmm_locals.argtypes = [C.c_void_p, C.c_int, _dp]
        L.orc_fmm_pows.argtypes = [C.c_void_p, _dp]
        L.orc_fmm_fprepass.argtypes = [C.c_void_p, _dp, _dp]
        L.orc_fmm_near.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp]
        L.orc_fmm_n_m2l.argtypes = [C.c_void_p]
        L.orc_fmm_n_m2l.restype = _sz
        L.orc_fmm_n_p2p.argtypes = [C.c_void_p]
        L.orc_fmm_n_p2p.restype = _sz
        L.orc_fmm_pops.argtypes = [C.c_void_p]
        L.orc_fmm_pops.restype = C.c_uint64
        L.orc_fmm_lists.argtypes = [C.c_void_p, _u32p, _u32p]
        L.orc_m2l_pair_test.argtypes = [_sz, _dp, _dp, _dp, _dp, C.c_int, _dp, _dp]
        L.orc_p2p_test.argtypes = [_sz, _dp, _dp, _dp, _dp, _sz, _sz, _sz, _sz, C.c_double, _dp, _dp, _dp, _dp]
        L.orc_direct.argtypes = [_sz, _dp, _dp, C.c_double, _dp, _dp]
        L.orc_direct_targets.argtypes = [_sz, _dp, _dp, C.c_double, _sz, _u32p, _dp, _dp, _dp, C.c_int]
        L.orc_scaled_error.argtypes = [_sz, _dp, _dp, _dp, _dp, _dp]
        L.orc_sample_targets.argtypes = [_sz, C.c_uint64, _sz, _u32p]
        _lib = L
    return _lib


def dim(p: int) -> int:
    return (p + 1) * (p + 1)


def idx(n: int, m: int) -> int:
    return n * (n + 1) + m


# ----------------------------------------------------------------- generators
def plummer(n: int, center=(0.0, 0.0, 0.0), seed: int = 42):
    """models.rs:35-58 -> (mass[n], pos[n,3])."""
    mass = np.empty(n)
    pos = np.empty((n, 3))
    lib().orc_plummer(n, center[0], center[1], center[2], seed, _ptr(mass, _dp), _ptr(pos, _dp))
    return mass, pos


def hernquist(n: int, center=(0.0, 0.0, 0.0), seed: int = 7):
    mass = np.empty(n)
    pos = np.empty((n, 3))
    lib().orc_hernquist(n, center[0], center[1], center[2], seed, _ptr(mass, _dp), _ptr(pos, _dp))
    return mass, pos


def gen_plummer_ic(n, mtot=1.0, a=1.0, rmax=20.0, seed=1, velocities=True):
    """Benchmark workload (no reference counterpart): Plummer sphere truncated
    at r <= rmax*a with distribution-function velocities -> (mass, pos, vel)."""
    mass, pos = np.empty(n), np.empty((n, 3))
    vel = np.empty((n, 3)) if velocities else None
    lib().orc_gen_plummer_ic(n, mtot, a, rmax, seed, _ptr(mass, _dp), _ptr(pos, _dp), _ptr(vel, _dp))
    return mass, pos, vel


def gen_uniform_lognormal(n, sigma=0.5, seed=2):
    """Benchmark workload: uniform unit cube, log-normal masses summing to 1."""
    mass, pos = np.empty(n), np.empty((n, 3))
    lib().orc_gen_uniform_lognormal(n, sigma, seed, _ptr(mass, _dp), _ptr(pos, _dp))
    return mass, pos


def gen_clusters(n, nclust=64, amin=1e-3, amax=1e-1, seed=3, velocities=True):
    """Benchmark workload: nclust Plummer spheres, Dirichlet(1) sizes."""
    mass, pos = np.empty(n), np.empty((n, 3))
    vel = np.empty((n, 3)) if velocities else None
    lib().orc_gen_clusters(n, nclust, amin, amax, seed, _ptr(mass, _dp), _ptr(pos, _dp), _ptr(vel, _dp))
    return mass, pos, vel


def rng_units(seed: int, n: int):
    out = np.empty(n)
    lib().orc_rng_units(seed, n, _ptr(out, _dp))
    return out


# ------------------------------------------------------------------ harmonics
def theta_table(r, p):
    r = np.ascontiguousarray(r, dtype=np.float64)
    out = np.empty(2 * dim(p))
    lib().orc_theta_table(_ptr(r, _dp), p, _ptr(out, _dp))
    return out[0::2] + 1j * out[1::2]


def upsilon_table(r, p):
    r = np.ascontiguousarray(r, dtype=np.float64)
    out = np.empty(2 * dim(p))
    lib().orc_upsilon_table(_ptr(r, _dp), p, _ptr(out, _dp))
    return out[0::2] + 1j * out[1::2]


def dilate(x: int) -> int:
    return int(lib().orc_dilate(x))


def factorials(p):
    out = np.empty(2 * p + 1)
    lib().orc_factorials(p, _ptr(out, _dp))
    return out


def binomials(p):
    out = np.empty(p + 1)
    lib().orc_binomials(p, _ptr(out, _dp))
    return out


def swap_matrices(p):
    """Block-layout B_n, n = 0..p, as a list of (2n+1)x(2n+1) arrays."""
    bs = lib().orc_blocksum(p)
    out = np.empty(bs)
    lib().orc_swap_matrices(p, _ptr(out, _dp))
    mats = []
    off = 0
    for n in range(p + 1):
        nb = 2 * n + 1
        mats.append(out[off : off + nb * nb].reshape(nb, nb))
        off += nb * nb
    return mats


def _cplx(a):
    a = np.ascontiguousarray(a, dtype=np.complex128)
    return a.view(np.float64)


def m2l_pair(p, cen_a, cen_b, mom_a, mom_b, rotation=False):
    d = dim(p)
    ca = np.ascontiguousarray(cen_a, dtype=np.float64)
    cb = np.ascontiguousarray(cen_b, dtype=np.float64)
    ma = _cplx(mom_a)
    mb = _cplx(mom_b)
    la = np.zeros(2 * d)
    lb = np.zeros(2 * d)
    lib().orc_m2l_pair_test(p, _ptr(ca, _dp), _ptr(cb, _dp), _ptr(ma, _dp), _ptr(mb, _dp), int(rotation),
                            _ptr(la, _dp), _ptr(lb, _dp))
    return la.view(np.complex128), lb.view(np.complex128)


def p2p(x, y, z, m, a_first, a_count, b_first, b_count, softening=0.0):
    n = len(x)
    arrs = [np.ascontiguousarray(v, dtype=np.float64) for v in (x, y, z, m)]
    outs = [np.zeros(n) for _ in range(4)]
    lib().orc_p2p_test(n, *[_ptr(v, _dp) for v in arrs], a_first, a_count, b_first, b_count, softening,
                       *[_ptr(v, _dp) for v in outs])
    return outs  # ax, ay, az, pot


def direct(mass, pos, softening=0.0):
    n = len(mass)
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    mass = np.ascontiguousarray(mass, dtype=np.float64)
    acc = np.empty((n, 3))
    pot = np.empty(n)
    lib().orc_direct(n, _ptr(pos, _dp), _ptr(mass, _dp), softening, _ptr(acc, _dp), _ptr(pot, _dp))
    return acc, pot


def direct_targets(mass, pos, targets, softening=0.0, nthreads=None):
    """Exact acc, pot and f = sum m/r^2 at the given target ids."""
    n = len(mass)
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    mass = np.ascontiguousarray(mass, dtype=np.float64)
    t = np.ascontiguousarray(targets, dtype=np.uint32)
    acc = np.empty((len(t), 3))
    pot = np.empty(len(t))
    f = np.empty(len(t))
    nth = nthreads or os.cpu_count() or 1
    lib().orc_direct_targets(n, _ptr(pos, _dp), _ptr(mass, _dp), softening, len(t), _ptr(t, _u32p),
                             _ptr(acc, _dp), _ptr(pot, _dp), _ptr(f, _dp), nth)
    return acc, pot, f


def scaled_error(a_ref, a_fmm, mass, pos):
    """direct.rs:35-78 -> (max_scaled, max_rel, rms_scaled, rms_rel)."""
    n = len(mass)
    out = np.empty(4)
    ar = np.ascontiguousarray(a_ref, dtype=np.float64)
    af = np.ascontiguousarray(a_fmm, dtype=np.float64)
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    mass = np.ascontiguousarray(mass, dtype=np.float64)
    lib().orc_scaled_error(n, _ptr(ar, _dp), _ptr(af, _dp), _ptr(pos, _dp), _ptr(mass, _dp), _ptr(out, _dp))
    return tuple(out)


def sample_targets(n, seed, samp):
    out = np.empty(samp, dtype=np.uint32)
    lib().orc_sample_targets(n, seed, samp, _ptr(out, _u32p))
    return out


# ------------------------------------------------------------------------ FMM
MAC_DEHNEN = 0
MAC_THETA = 1


class Fmm:
    """Mirror of fmm::Fmm (fmm.rs:10-142) over the oracle."""

    def __init__(self, mass, pos, p, eps, n_leaf, *, mac=MAC_DEHNEN, theta=0.5, softening=0.0, center=0,
                 soft_gap=0.0):
        self.mass = np.ascontiguousarray(mass, dtype=np.float64)
        self.pos = np.ascontiguousarray(pos, dtype=np.float64)
        self.n = len(self.mass)
        self.p = p
        self._h = lib().orc_fmm_new(self.n, _ptr(self.pos, _dp), _ptr(self.mass, _dp), p, mac, eps, theta,
                                    softening, n_leaf, center)
        if not self._h:
            raise ValueError("empty input")
        if soft_gap:
            lib().orc_fmm_set_gap(self._h, soft_gap * softening)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().orc_fmm_free(h)
            self._h = None

    def refresh(self, mass, pos):
        self.mass = np.ascontiguousarray(mass, dtype=np.float64)
        self.pos = np.ascontiguousarray(pos, dtype=np.float64)
        lib().orc_fmm_refresh(self._h, self.n, _ptr(self.pos, _dp), _ptr(self.mass, _dp))

    def run(self, mass=None, pos=None, nthreads=1):
        mass = self.mass if mass is None else np.ascontiguousarray(mass, dtype=np.float64)
        pos = self.pos if pos is None else np.ascontiguousarray(pos, dtype=np.float64)
        acc = np.empty((self.n, 3))
        pot = np.empty(self.n)
        lib().orc_fmm_run(self._h, self.n, _ptr(pos, _dp), _ptr(mass, _dp), nthreads, _ptr(acc, _dp),
                          _ptr(pot, _dp))
        return acc, pot

    def walk(self, nthreads=1):
        """Moments, power, f pre-pass and the dual walk's record phase only
        (the walk statistics of crates/bench/src/main.rs:554-641); returns
        (mutual M2L pairs, P2P leaf pairs incl. self pairs, pops)."""
        lib().orc_fmm_walk(self._h, self.n, _ptr(self.pos, _dp), _ptr(self.mass, _dp), nthreads)
        return int(lib().orc_fmm_n_m2l(self._h)), int(lib().orc_fmm_n_p2p(self._h)), self.pops

    @property
    def ncells(self):
        return int(lib().orc_fmm_ncells(self._h))

    def cells(self):
        nc = self.ncells
        info = np.empty((nc, 4), dtype=np.uint32)
        ch = np.empty((nc, 8), dtype=np.int32)
        cen = np.empty((nc, 3))
        mass = np.empty(nc)
        rho = np.empty(nc)
        lib().orc_fmm_cells(self._h, _ptr(info, _u32p), _ptr(ch, _i32p), _ptr(cen, _dp), _ptr(mass, _dp),
                            _ptr(rho, _dp))
        return dict(first=info[:, 0], count=info[:, 1], level=info[:, 2], leaf=info[:, 3].astype(bool),
                    children=ch, cen=cen, mass=mass, rho=rho)

    def order(self):
        o = np.empty(self.n, dtype=np.uint32)
        k = np.empty(self.n, dtype=np.uint64)
        lib().orc_fmm_order(self._h, _ptr(o, _u32p), _ptr(k, _u64p))
        return o, k

    def bbox(self):
        out = np.empty(8)
        lib().orc_fmm_bbox(self._h, _ptr(out, _dp))
        return out

    def moments(self):
        out = np.empty(2 * self.ncells * dim(self.p))
        lib().orc_fmm_moments(self._h, _ptr(out, _dp))
        return out.view(np.complex128).reshape(self.ncells, dim(self.p))

    def locals(self, after_l2l=True):
        out = np.empty(2 * self.ncells * dim(self.p))
        lib().orc_fmm_locals(self._h, int(after_l2l), _ptr(out, _dp))
        return out.view(np.complex128).reshape(self.ncells, dim(self.p))

    def pows(self):
        out = np.empty(self.ncells * (self.p + 1))
        lib().orc_fmm_pows(self._h, _ptr(out, _dp))
        return out.reshape(self.ncells, self.p + 1)

    def fprepass(self):
        f = np.empty(self.n)
        fm = np.empty(self.ncells)
        lib().orc_fmm_fprepass(self._h, _ptr(f, _dp), _ptr(fm, _dp))
        return f, fm

    def near(self):
        outs = [np.empty(self.n) for _ in range(4)]
        lib().orc_fmm_near(self._h, *[_ptr(v, _dp) for v in outs])
        return outs

    def lists(self):
        nm = int(lib().orc_fmm_n_m2l(self._h))
        npp = int(lib().orc_fmm_n_p2p(self._h))
        m2l = np.empty((nm, 2), dtype=np.uint32)
        p2p = np.empty((npp, 2), dtype=np.uint32)
        lib().orc_fmm_lists(self._h, _ptr(m2l, _u32p), _ptr(p2p, _u32p))
        return m2l, p2p

    @property
    def pops(self):
        return int(lib().orc_fmm_pops(self._h))
