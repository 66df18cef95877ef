"""fmms_b200 — host-side mirror of the reference FMM's solver API over the
B200 engine (libfmmx.so, C ABI in include/fmmx.h).

The reference API is ``fmm::Fmm`` (crates/fmm/src/fmm.rs:10-142)::

    Fmm::new(parts, p, eps, n_leaf)      -> Fmm          (builds the tree)
    fmm.refresh(parts)                                     (rebuild in place)
    fmm.run(parts) / run_threaded(parts, n) -> Result{accel, pot, n_cells}

Here ``parts`` is a pair ``(mass[n], pos[n, 3])`` of float64 arrays, and the
same calls exist with the same meaning. Errors that the reference raises as
panics (empty input, p out of range) raise ``FmmError`` here. There is no CPU
fallback: without the CUDA library or a device, every call fails loudly.
"""

from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfmmx.so")
_lib = None


class FmmError(RuntimeError):
    """A failed engine call (status code and the engine's message)."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


STATUS_NAMES = {
    0: "ok",
    1: "invalid argument",
    2: "out of memory",
    3: "over budget",
    4: "leaf overflow",
    5: "device error",
    6: "timeout",
    7: "not built",
    8: "no CUDA device",
}

MAC_DEHNEN, MAC_THETA = 0, 1
CENTER_COM, CENTER_SPHERE = 0, 1
PLAIN_FP64, MIXED = 0, 1
M2L_AUTO, M2L_NAIVE, M2L_ROTATION = 0, 1, 2


class Config(C.Structure):
    _fields_ = [
        ("p", C.c_int),
        ("mac_mode", C.c_int),
        ("mac_eps", C.c_double),
        ("theta", C.c_double),
        ("softening", C.c_double),
        ("n_leaf", C.c_int),
        ("center_mode", C.c_int),
        ("precision", C.c_int),
        ("m2l_kernel", C.c_int),
        ("device", C.c_int),
        ("stream", C.c_void_p),
        ("p2p_tile", C.c_int),
        ("preemptible", C.c_int),
        ("soft_gap", C.c_double),
        ("use_graphs", C.c_int),
        ("overlap", C.c_int),
        ("device_budget_bytes", C.c_uint64),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("n", C.c_uint64),
        ("n_cells", C.c_uint64),
        ("n_leaves", C.c_uint64),
        ("n_levels", C.c_uint64),
        ("n_m2l", C.c_uint64),
        ("n_p2p", C.c_uint64),
        ("walk_pops", C.c_uint64),
        ("p2p_interactions", C.c_uint64),
        ("m2l_directed", C.c_uint64),
        ("ms_build", C.c_double),
        ("ms_upward", C.c_double),
        ("ms_walk", C.c_double),
        ("ms_lists", C.c_double),
        ("ms_m2l", C.c_double),
        ("ms_p2p", C.c_double),
        ("ms_l2l", C.c_double),
        ("ms_l2p", C.c_double),
        ("ms_evaluate", C.c_double),
        ("kernel_launches", C.c_uint64),
        ("walk_retries", C.c_uint64),
        ("device_bytes", C.c_uint64),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_dp = C.POINTER(C.c_double)
_u32p = C.POINTER(C.c_uint32)
_i32p = C.POINTER(C.c_int32)
_u64p = C.POINTER(C.c_uint64)
_vp = C.c_void_p
_sz = C.c_size_t
_st = C.c_int

# name -> (restype, argtypes); every symbol declared in include/fmmx.h
SIGNATURES = {
    "fmmx_config_default": (None, [C.POINTER(Config)]),
    "fmmx_create": (_st, [C.POINTER(Config), C.POINTER(_vp)]),
    "fmmx_destroy": (None, [_vp]),
    "fmmx_last_error": (C.c_char_p, [_vp]),
    "fmmx_status_string": (C.c_char_p, [_st]),
    "fmmx_build": (_st, [_vp, _sz, _dp, _dp]),
    "fmmx_evaluate": (_st, [_vp, _dp, _dp, _dp, _dp]),
    "fmmx_build_device": (_st, [_vp, _sz, _vp, _vp]),
    "fmmx_evaluate_device": (_st, [_vp, _vp, _vp, _vp, _vp]),
    "fmmx_synchronize": (_st, [_vp]),
    "fmmx_kdk_step_device": (_st, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _sz, _u64p, C.c_int]),
    "fmmx_leapfrog_device": (_st, [_vp, _vp, _vp, _vp, _vp, _vp, C.c_double, C.c_int, C.c_int, C.c_int]),
    "fmmx_build_ensemble": (_st, [_vp, _sz, _u64p, _dp, _dp]),
    "fmmx_build_ensemble_device": (_st, [_vp, _sz, _u64p, _vp, _vp]),
    "fmmx_get_stats": (_st, [_vp, C.POINTER(Stats)]),
    "fmmx_export_tree": (_st, [_vp, _u32p, _u64p, _u32p, _i32p, _dp, _dp, _dp]),
    "fmmx_export_lists": (_st, [_vp, _u32p, _u32p]),
    "fmmx_export_expansions": (_st, [_vp, _dp, _dp, _dp, _dp, _dp]),
    "fmmx_direct_targets": (_st, [C.c_int, _sz, _dp, _dp, C.c_double, _sz, _u32p, _dp, _dp, _dp]),
    "fmmx_probe_fma_peak": (_st, [C.c_int, C.c_int, _dp]),
    "fmmx_direct_targets_noalloc": (_st, [C.c_int, _vp, _sz, _vp, _vp, C.c_double, _sz, _vp, _vp, _vp, _vp]),
    "fmmx_gen_plummer": (None, [_sz, C.c_double, C.c_double, C.c_double, C.c_uint64, _dp, _dp]),
    "fmmx_gen_hernquist": (None, [_sz, C.c_double, C.c_double, C.c_double, C.c_uint64, _dp, _dp]),
    "fmmx_gen_plummer_ic": (None, [_sz, C.c_double, C.c_double, C.c_double, C.c_uint64, _dp, _dp, _dp]),
    "fmmx_gen_uniform_lognormal": (None, [_sz, C.c_double, C.c_uint64, _dp, _dp]),
    "fmmx_gen_clusters": (None, [_sz, C.c_int, C.c_double, C.c_double, C.c_uint64, _dp, _dp, _dp]),
}


def lib():
    """Load libfmmx.so (built in-tree by fmms_b200/build.py); raises if absent."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m fmms_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _ptr(a, t=_dp):
    return None if a is None else a.ctypes.data_as(t)


def _f64(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None and a.shape != shape:
        a = a.reshape(shape)
    return a


@dataclass
class Result:
    """fmm::Result (fmm.rs:17-21): accelerations and potentials in particle-id order."""

    accel: np.ndarray  # (n, 3)
    pot: np.ndarray  # (n,)
    n_cells: int


def dim(p: int) -> int:
    return (p + 1) * (p + 1)


class Fmm:
    """GPU counterpart of fmm::Fmm.

    ``Fmm(mass, pos, p, eps, n_leaf)`` builds the tree like ``Fmm::new``. The
    keyword arguments select the extensions: ``mac='theta'`` with ``theta``,
    ``softening``, ``precision='mixed'``, ``center='sphere'`` (as
    ``Fmm::with_center``), ``m2l='naive'|'rotation'``, ``soft_gap`` (M2L only
    between cells whose bodies are soft_gap * softening apart),
    ``device_budget_bytes`` (device memory the context may hold; beyond it a
    call raises FmmError with status "over budget").
    """

    def __init__(self, mass, pos, p: int = 8, eps: float = 1e-5, n_leaf: int = 16, *, mac: str = "dehnen",
                 theta: float = 0.5, softening: float = 0.0, precision: str = "plain", center: str = "com",
                 m2l: str = "auto", device: int = 0, stream: int | None = None, p2p_tile: int = 0,
                 preemptible: bool = False, soft_gap: float = 0.0, use_graphs: bool = True,
                 overlap: bool = True, device_budget_bytes: int = 0):
        cfg = Config()
        lib().fmmx_config_default(C.byref(cfg))
        cfg.p = int(p)
        cfg.mac_mode = {"dehnen": MAC_DEHNEN, "theta": MAC_THETA}[mac]
        cfg.mac_eps = float(eps)
        cfg.theta = float(theta)
        cfg.softening = float(softening)
        cfg.n_leaf = int(n_leaf)
        cfg.center_mode = {"com": CENTER_COM, "sphere": CENTER_SPHERE}[center]
        cfg.precision = {"plain": PLAIN_FP64, "mixed": MIXED}[precision]
        cfg.m2l_kernel = {"auto": M2L_AUTO, "naive": M2L_NAIVE, "rotation": M2L_ROTATION}[m2l]
        cfg.device = int(device)
        cfg.stream = stream
        cfg.p2p_tile = int(p2p_tile)
        cfg.preemptible = 1 if preemptible else 0
        cfg.soft_gap = float(soft_gap)
        cfg.use_graphs = 1 if use_graphs else 0
        cfg.overlap = 1 if overlap else 0
        cfg.device_budget_bytes = int(device_budget_bytes)
        self.cfg = cfg
        self.p = cfg.p
        h = _vp()
        st = lib().fmmx_create(C.byref(cfg), C.byref(h))
        if st != 0:
            raise FmmError(st, "fmmx_create failed")
        self._h = h
        self.n = 0
        if mass is not None:
            self.refresh(mass, pos)

    # --------------------------------------------------------------- lifecycle
    def close(self):
        h = getattr(self, "_h", None)
        if h:
            lib().fmmx_destroy(h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st != 0:
            msg = lib().fmmx_last_error(self._h)
            raise FmmError(st, msg.decode() if msg else "")

    # -------------------------------------------------------------- reference API
    @classmethod
    def new(cls, parts, p, eps, n_leaf, **kw):
        """Fmm::new(parts, p, eps, n_leaf) with parts = (mass, pos)."""
        mass, pos = parts
        return cls(mass, pos, p, eps, n_leaf, **kw)

    def refresh(self, mass, pos):
        """Fmm::refresh: rebuild the tree for new positions."""
        mass = _f64(mass)
        pos = _f64(pos)
        n = len(mass)
        if pos.shape != (n, 3):
            raise ValueError("pos must be (n, 3)")
        self._mass, self._pos = mass, pos
        self.n = n
        self._check(lib().fmmx_build(self._h, n, _ptr(pos), _ptr(mass)))

    def build_ensemble(self, offsets, mass, pos):
        """Forest of independent systems: system s is bodies offsets[s]:offsets[s+1]."""
        off = np.ascontiguousarray(offsets, dtype=np.uint64)
        mass = _f64(mass)
        pos = _f64(pos)
        self._mass, self._pos = mass, pos
        self.n = int(off[-1])
        self._check(lib().fmmx_build_ensemble(self._h, len(off) - 1, _ptr(off, _u64p), _ptr(pos), _ptr(mass)))

    def build_ensemble_device(self, offsets, pos_ptr: int, mass_ptr: int):
        off = np.ascontiguousarray(offsets, dtype=np.uint64)
        self.n = int(off[-1])
        self._check(lib().fmmx_build_ensemble_device(self._h, len(off) - 1, _ptr(off, _u64p), pos_ptr, mass_ptr))

    def run(self, mass=None, pos=None) -> Result:
        """Fmm::run: one force evaluation (bodies of the last build when None)."""
        n = self.n
        if mass is not None:
            mass = _f64(mass)
        if pos is not None:
            pos = _f64(pos)
            if pos.shape != (n, 3):
                raise ValueError("pos must be (n, 3) with the built n")
        acc = np.empty((n, 3))
        pot = np.empty(n)
        self._check(lib().fmmx_evaluate(self._h, _ptr(pos), _ptr(mass), _ptr(acc), _ptr(pot)))
        return Result(acc, pot, self.stats()["n_cells"])

    def run_threaded(self, mass=None, pos=None, nthreads: int = 1) -> Result:
        """Fmm::run_threaded: same result as run (threads are the GPU's)."""
        return self.run(mass, pos)

    # ------------------------------------------------------------ device-resident
    def build_device(self, pos_ptr: int, mass_ptr: int, n: int):
        self.n = n
        self._check(lib().fmmx_build_device(self._h, n, pos_ptr, mass_ptr))

    def evaluate_device(self, pos_ptr, mass_ptr, acc_ptr, pot_ptr):
        self._check(lib().fmmx_evaluate_device(self._h, pos_ptr, mass_ptr, acc_ptr, pot_ptr))

    def leapfrog_device(self, pos_ptr, vel_ptr, mass_ptr, acc_ptr, pot_ptr, dt, nsteps, scheme="kdk",
                        refresh_every=1):
        """Device-resident leapfrog; KDK needs acc at pos on entry."""
        sc = {"kdk": 0, "dkd": 1}[scheme]
        self._check(lib().fmmx_leapfrog_device(self._h, pos_ptr, vel_ptr, mass_ptr, acc_ptr, pot_ptr, float(dt),
                                               int(nsteps), sc, int(refresh_every)))

    def kdk_step_device(self, pos_ptr, vel_ptr, mass_ptr, acc_ptr, pot_ptr, dt_ptr, offsets=None,
                        rebuild=True):
        """One kick-drift-kick step with a time step per body (device array of
        n FP64; 0 keeps a body in place). With offsets the tree is rebuilt over
        those systems; without, rebuild=False reuses the last tree and lists."""
        off = None if offsets is None else np.ascontiguousarray(offsets, dtype=np.uint64)
        if off is not None:
            self.n = int(off[-1])
        self._check(lib().fmmx_kdk_step_device(self._h, pos_ptr, vel_ptr, mass_ptr, acc_ptr, pot_ptr, dt_ptr,
                                               0 if off is None else len(off) - 1,
                                               None if off is None else _ptr(off, _u64p), 1 if rebuild else 0))

    def synchronize(self):
        self._check(lib().fmmx_synchronize(self._h))

    # ------------------------------------------------------------------ reports
    def stats(self) -> dict:
        s = Stats()
        self._check(lib().fmmx_get_stats(self._h, C.byref(s)))
        return s.as_dict()

    @property
    def n_cells(self) -> int:
        return int(self.stats()["n_cells"])

    def export_tree(self):
        n, nc = self.n, self.n_cells
        order = np.empty(n, dtype=np.uint32)
        keys = np.empty(n, dtype=np.uint64)
        info = np.empty((nc, 4), dtype=np.uint32)
        ch = np.empty((nc, 8), dtype=np.int32)
        cen = np.empty((nc, 3))
        mass = np.empty(nc)
        rho = np.empty(nc)
        self._check(lib().fmmx_export_tree(self._h, _ptr(order, _u32p), _ptr(keys, _u64p), _ptr(info, _u32p),
                                           _ptr(ch, _i32p), _ptr(cen), _ptr(mass), _ptr(rho)))
        cells = dict(first=info[:, 0], count=info[:, 1], level=info[:, 2], leaf=info[:, 3].astype(bool),
                     children=ch, cen=cen, mass=mass, rho=rho)
        return order, keys, cells

    def export_lists(self):
        st = self.stats()
        m2l = np.empty((int(st["n_m2l"]), 2), dtype=np.uint32)
        p2p = np.empty((int(st["n_p2p"]), 2), dtype=np.uint32)
        self._check(lib().fmmx_export_lists(self._h, _ptr(m2l, _u32p), _ptr(p2p, _u32p)))
        return m2l, p2p

    def export_expansions(self):
        nc, d = self.n_cells, dim(self.p)
        mom = np.empty(2 * nc * d)
        loc = np.empty(2 * nc * d)
        pows = np.empty(nc * (self.p + 1))
        f = np.empty(self.n)
        fmin = np.empty(nc)
        self._check(lib().fmmx_export_expansions(self._h, _ptr(mom), _ptr(loc), _ptr(pows), _ptr(f), _ptr(fmin)))
        return dict(moments=mom.view(np.complex128).reshape(nc, d), locals=loc.view(np.complex128).reshape(nc, d),
                    pows=pows.reshape(nc, self.p + 1), f=f, fmin=fmin)


# --------------------------------------------------------------- free functions
def direct_targets(mass, pos, targets, softening=0.0, device=0):
    """FP64 direct sum on the device at `targets`: (acc[nt,3], pot[nt], f[nt])."""
    mass = _f64(mass)
    pos = _f64(pos)
    t = np.ascontiguousarray(targets, dtype=np.uint32)
    acc = np.empty((len(t), 3))
    pot = np.empty(len(t))
    f = np.empty(len(t))
    st = lib().fmmx_direct_targets(device, len(mass), _ptr(pos), _ptr(mass), float(softening), len(t),
                                   _ptr(t, _u32p), _ptr(acc), _ptr(pot), _ptr(f))
    if st != 0:
        raise FmmError(st, "fmmx_direct_targets failed")
    return acc, pot, f


def gen_plummer(n, center=(0.0, 0.0, 0.0), seed=42):
    """models::plummer (models.rs:35-58), bit for bit -> (mass, pos)."""
    mass = np.empty(n)
    pos = np.empty((n, 3))
    lib().fmmx_gen_plummer(n, center[0], center[1], center[2], seed, _ptr(mass), _ptr(pos))
    return mass, pos


def gen_hernquist(n, center=(0.0, 0.0, 0.0), seed=7):
    mass = np.empty(n)
    pos = np.empty((n, 3))
    lib().fmmx_gen_hernquist(n, center[0], center[1], center[2], seed, _ptr(mass), _ptr(pos))
    return mass, pos


def gen_plummer_ic(n, mtot=1.0, a=1.0, rmax=20.0, seed=1, velocities=True):
    """Truncated Plummer sphere with Plummer-DF velocities -> (mass, pos, vel)."""
    mass = np.empty(n)
    pos = np.empty((n, 3))
    vel = np.empty((n, 3)) if velocities else None
    lib().fmmx_gen_plummer_ic(n, mtot, a, rmax, seed, _ptr(mass), _ptr(pos), _ptr(vel))
    return mass, pos, vel


def gen_uniform_lognormal(n, sigma=0.5, seed=2):
    """Uniform unit cube, log-normal masses normalised to 1 -> (mass, pos)."""
    mass = np.empty(n)
    pos = np.empty((n, 3))
    lib().fmmx_gen_uniform_lognormal(n, sigma, seed, _ptr(mass), _ptr(pos))
    return mass, pos


def gen_clusters(n, nclust=64, amin=1e-3, amax=1e-1, seed=3, velocities=True):
    """nclust Plummer spheres (Dirichlet(1) sizes) -> (mass, pos, vel)."""
    mass = np.empty(n)
    pos = np.empty((n, 3))
    vel = np.empty((n, 3)) if velocities else None
    lib().fmmx_gen_clusters(n, nclust, amin, amax, seed, _ptr(mass), _ptr(pos), _ptr(vel))
    return mass, pos, vel


def probe_fma_peak(fp64: bool, device: int = 0) -> float:
    """Measured FMA throughput (TFLOP/s) of the device, FP64 or FP32."""
    out = C.c_double()
    st = lib().fmmx_probe_fma_peak(device, int(fp64), C.byref(out))
    if st != 0:
        raise FmmError(st, "fmmx_probe_fma_peak failed")
    return out.value


DIRECT_NOALLOC_MAX_TARGETS = 4096


def direct_targets_noalloc(n, d_pos, d_mass, nt, d_targets, d_acc, d_pot=None, d_fscale=None, softening=0.0,
                           device=0, stream=None):
    """Allocation-free direct sum on device buffers (integer device pointers);
    queued on `stream`, returns without waiting. See fmmx_direct_targets_noalloc."""
    st = lib().fmmx_direct_targets_noalloc(device, stream, n, d_pos, d_mass, float(softening), nt, d_targets,
                                           d_acc, d_pot, d_fscale)
    if st != 0:
        raise FmmError(st, "fmmx_direct_targets_noalloc failed")
