"""ctypes binding of the C ABI in ``include/pot_gpu.h``.

The reference's hot path is two C calls per step on a host ``Particle``
array (``build_tree`` pot.c:1457, ``move_particles`` pot.c:2330).  This
module exposes the library that replaces them -- ``libpotgpu.so``, CUDA
kernels for sm_100a -- with the same records (:data:`PARTICLE_DTYPE` is the
56-byte ``Particle`` of pot.c:295-303) and the same error behaviour (failures
become :class:`PotError` carrying the library's status code instead of the
reference's ``abort()``).

There is no CPU fallback: if the library cannot be loaded the import of a
:class:`Run` fails with an exception.
"""
from __future__ import annotations

import ctypes as C
import os
import re
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
HEADER = os.path.join(ROOT, "include", "pot_gpu.h")
LIB_PATH = os.path.join(PKG, "libpotgpu.so")

PARTICLE_DTYPE = np.dtype([("x", "<f8"), ("y", "<f8"), ("z", "<f8"),
                           ("vx", "<f8"), ("vy", "<f8"), ("vz", "<f8"),
                           ("species", "<i4"), ("_pad", "<i4")])
DUST, ION, ELECTRON = 0, 1, 2

POT_OK = 0
STATUS_NAMES = {0: "POT_OK", -1: "POT_E_ARG", -2: "POT_E_CUDA", -3: "POT_E_NOMEM", -4: "POT_E_DOMAIN",
                -5: "POT_E_COINCIDENT", -6: "POT_E_WALK", -7: "POT_E_NONFINITE", -8: "POT_E_ITER",
                -9: "POT_E_CAPACITY", -10: "POT_E_STATE", -11: "POT_E_LIMIT"}
NOALLOC_MAX_POINTS = 65536
FORM_PLAIN, FORM_FAST = 0, 1
STEP_EPE = 0x1
CFG_SCEPTIC, CFG_DISABLE_GRAIN, CFG_DIPOLES, CFG_POIS_IONS = 0x1, 0x2, 0x4, 0x8
INT_BORIS, INT_VERLET, INT_EULER_RICHARDSON = 0, 1, 2
OPT_TIMING = 0x1
OPT_CHI_CAP = 0x2
WARN_CHI_CAP = 512
BATCH_NO_PACK = 0x1


class PotError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str = ""):
        self.status = status
        super().__init__("%s failed: %s (%s)%s" % (where, STATUS_NAMES.get(status, status), msg,
                                                  "" if not msg else ""))


class _RunCfg(C.Structure):
    _fields_ = [("N", C.c_uint64), ("r", C.c_uint32), ("flags", C.c_uint32), ("dt", C.c_double),
                ("mpp", C.c_double), ("soft", C.c_double), ("Te", C.c_double), ("Ti", C.c_double),
                ("x_drift", C.c_double), ("a", C.c_double), ("settle", C.c_double), ("theta", C.c_double),
                ("B", C.c_double * 3), ("A", C.c_double), ("axis", C.c_double * 3), ("bounce", C.c_double),
                ("integrator", C.c_uint32), ("pad", C.c_uint32)]


class _Opts(C.Structure):
    _fields_ = [("form", C.c_uint32), ("leaf_size", C.c_uint32), ("group_size", C.c_uint32),
                ("flags", C.c_uint32), ("device", C.c_int32), ("chi_b_ranks", C.c_uint32), ("seed", C.c_uint64),
                ("stream", C.c_void_p)]


class _Grain(C.Structure):
    _fields_ = [("q", C.c_int64), ("m", C.c_double), ("x", C.c_double), ("y", C.c_double), ("z", C.c_double),
                ("vx", C.c_double), ("vy", C.c_double), ("vz", C.c_double), ("tot_absor_e", C.c_uint64),
                ("t_steps", C.c_uint64), ("chi_b", C.c_double)]


class _Stats(C.Structure):
    _fields_ = [("t_steps", C.c_uint64), ("grain_q", C.c_int64), ("dq", C.c_int64), ("de", C.c_uint64),
                ("n_absorbed", C.c_uint64), ("n_reinjected", C.c_uint64), ("n_pushed", C.c_uint64),
                ("interactions", C.c_uint64), ("n_nodes", C.c_uint64), ("chi_b", C.c_double),
                ("status", C.c_int32), ("stack_max", C.c_uint32), ("epe", C.c_double * 3),
                ("q_sum", C.c_int64), ("warn", C.c_uint32), ("n_collected", C.c_uint32),
                ("n_wall", C.c_uint32), ("n_bounced", C.c_uint32), ("n_groups", C.c_uint32), ("pad", C.c_uint32),
                ("far_cells", C.c_uint64)]


_LIB = None


def header_symbols() -> list:
    """Entry points declared in include/pot_gpu.h."""
    with open(HEADER) as f:
        text = f.read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_ ]*?\**\s*\b(pot_gpu_[a-z_]+)\s*\(",
                                 text, flags=re.M)))


def load_library(path: str = LIB_PATH, build_if_stale: bool = True):
    """Load libpotgpu.so (building it first if nvcc is present and the
    sources are newer).  Raises if the library cannot be loaded."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if build_if_stale and path == LIB_PATH:
        from . import build as _build
        try:
            if _build.stale():
                _build.build()
        except FileNotFoundError:
            pass  # no nvcc here: load what exists, fail below if nothing does
    if not os.path.exists(path):
        raise OSError("libpotgpu.so not found at %s (run python -m pot_b200.build)" % path)
    L = C.CDLL(path)
    vp, u64, u32, i32, dp = C.c_void_p, C.c_uint64, C.c_uint32, C.c_int32, C.c_void_p
    L.pot_gpu_create.argtypes = [C.POINTER(_RunCfg), C.POINTER(_Opts), C.POINTER(vp)]
    L.pot_gpu_destroy.argtypes = [vp]
    L.pot_gpu_destroy.restype = None
    L.pot_gpu_strerror.argtypes = [C.c_int]
    L.pot_gpu_strerror.restype = C.c_char_p
    L.pot_gpu_upload.argtypes = [vp, vp, u64, C.POINTER(_Grain)]
    L.pot_gpu_init_particles.argtypes = [vp]
    L.pot_gpu_step.argtypes = [vp, u32, u32, C.POINTER(_Stats)]
    L.pot_gpu_step_async.argtypes = [vp, u32, u32]
    L.pot_gpu_download.argtypes = [vp, vp, C.POINTER(_Grain)]
    L.pot_gpu_move_particles.argtypes = [vp, vp, u64, C.POINTER(_Grain), C.POINTER(_Stats)]
    L.pot_gpu_build_tree.argtypes = [vp, C.POINTER(u64)]
    L.pot_gpu_tree_dump.argtypes = [vp, u64, C.POINTER(u64), vp, vp, vp, vp, vp, vp, C.POINTER(u64), vp, vp, vp]
    L.pot_gpu_field_at.argtypes = [vp, u64, vp, vp, vp]
    L.pot_gpu_field_at_noalloc.argtypes = [vp, u64, vp, vp, vp]
    L.pot_gpu_phi_at.argtypes = [vp, u64, vp, vp]
    L.pot_gpu_kernel_times.argtypes = [vp, C.c_int, C.POINTER(C.c_char_p), C.POINTER(C.c_double),
                                       C.POINTER(u64)]
    L.pot_gpu_reset_kernel_times.argtypes = [vp]
    L.pot_gpu_sync.argtypes = [vp]
    L.pot_gpu_launch_count.argtypes = [vp, C.POINTER(u64)]
    L.pot_gpu_macro.argtypes = [vp, C.POINTER(_MacroSums)]
    L.pot_gpu_grain.argtypes = [vp, C.POINTER(_Grain)]
    L.pot_gpu_set_ion_temp.argtypes = [vp, C.c_double]
    L.pot_gpu_ion_temp.argtypes = [vp, C.POINTER(C.c_double)]
    L.pot_gpu_bytes_needed.argtypes = [C.POINTER(_RunCfg), C.POINTER(_Opts), C.POINTER(u64)]
    L.pot_gpu_tune.argtypes = [C.POINTER(_RunCfg), C.POINTER(_Opts), u32, C.POINTER(C.c_double)]
    L.pot_batch_create.argtypes = [C.POINTER(_BatchOpts), C.POINTER(vp)]
    L.pot_batch_destroy.argtypes = [vp]
    L.pot_batch_destroy.restype = None
    L.pot_batch_admit.argtypes = [vp, C.POINTER(_RunCfg), C.POINTER(_Opts), vp, C.POINTER(_Grain),
                                  C.POINTER(C.c_int32)]
    L.pot_batch_evict.argtypes = [vp, C.c_int32]
    L.pot_batch_step.argtypes = [vp, u32]
    L.pot_batch_sync.argtypes = [vp]
    L.pot_batch_summary.argtypes = [vp, u32, vp, C.POINTER(u32)]
    L.pot_batch_count.argtypes = [vp, C.POINTER(u32), C.POINTER(u64), C.POINTER(u64)]
    L.pot_batch_ctx.argtypes = [vp, C.c_int32, C.POINTER(vp)]
    for name in ("pot_batch_create", "pot_batch_admit", "pot_batch_evict", "pot_batch_step", "pot_batch_sync",
                 "pot_batch_summary", "pot_batch_count", "pot_batch_ctx"):
        getattr(L, name).restype = C.c_int
    for name in header_symbols():
        fn = getattr(L, name)
        if fn.restype is C.c_int or name not in ("pot_gpu_destroy", "pot_gpu_strerror"):
            if name not in ("pot_gpu_destroy", "pot_gpu_strerror"):
                fn.restype = C.c_int
    _LIB = L
    return L


class _MacroSums(C.Structure):
    _fields_ = [("n_e", C.c_double), ("n_i", C.c_double), ("K_e", C.c_double), ("s_e", C.c_double),
                ("s_i", C.c_double), ("v_e", C.c_double * 3), ("v_i", C.c_double * 3), ("am_e", C.c_double * 3),
                ("am_i", C.c_double * 3), ("pad1", C.c_double * 3), ("sumsq_K_e", C.c_double),
                ("sum_x_e", C.c_double), ("sumsq_x_e", C.c_double), ("K_e_c", C.c_double * 3),
                ("s_e_c", C.c_double * 3), ("T_e", C.c_double), ("sum_K_i", C.c_double), ("sumsq_K_i", C.c_double),
                ("s_i_c", C.c_double * 3), ("T_i", C.c_double), ("pad2", C.c_double * 2)]


class _BatchOpts(C.Structure):
    _fields_ = [("device", C.c_int32), ("steps_per_launch", C.c_uint32), ("reserve_bytes", C.c_uint64),
                ("flags", C.c_uint32), ("pad", C.c_uint32)]


BATCH_ROW_DTYPE = np.dtype([("slot", "<i4"), ("status", "<i4"), ("t_steps", "<u8"), ("grain_q", "<i8"),
                            ("q_sum", "<i8"), ("tot_absor_e", "<u8"), ("particles", "<u8"), ("warn", "<u4"),
                            ("pad", "<u4")])


@dataclass
class RunConfig:
    """Run settings with the reference's flag meanings (pot.c:4557-4850)."""
    N: int
    r: int
    dt: float
    mpp: float
    soft: float
    Te: float
    Ti: float
    x_drift: float = 0.0
    a: float = 2.5e-6
    settle: float = 0.0
    theta: float = 0.5
    B: Sequence[float] = field(default_factory=lambda: (0.0, 0.0, 0.0))
    A: float = 0.0
    sceptic: bool = True
    disable_grain: bool = False
    axis: Sequence[float] = field(default_factory=lambda: (0.0, 0.0, 0.0))
    # the reference's other compile-time variants (pot.c:99-133, 165-173)
    bounce: float = 0.0          # OUT_BOUNCE coefficient of restitution; 0 = reinjection
    integrator: int = INT_BORIS  # INT_BORIS, INT_VERLET or INT_EULER_RICHARDSON
    dipoles: bool = False        # DIPOLES (fast form: groups of at most 32)
    pois_ions: bool = False      # POIS_POS_COLLECTION

    def to_c(self) -> _RunCfg:
        c = _RunCfg()
        c.N, c.r = int(self.N), int(self.r)
        c.flags = ((CFG_SCEPTIC if self.sceptic else 0) | (CFG_DISABLE_GRAIN if self.disable_grain else 0)
                   | (CFG_DIPOLES if self.dipoles else 0) | (CFG_POIS_IONS if self.pois_ions else 0))
        c.bounce = float(self.bounce)
        c.integrator = int(self.integrator)
        c.dt, c.mpp, c.soft, c.Te, c.Ti = self.dt, self.mpp, self.soft, self.Te, self.Ti
        c.x_drift, c.a, c.settle, c.theta, c.A = self.x_drift, self.a, self.settle, self.theta, self.A
        for k in range(3):
            c.B[k] = float(self.B[k])
            c.axis[k] = float(self.axis[k])
        return c


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def _stats_dict(st: "_Stats") -> dict:
    d = {k: getattr(st, k) for k, _ in _Stats._fields_ if k not in ("pad", "pad2", "epe")}
    d["epe"] = np.array(list(st.epe))
    return d


def _grain_dict(g: _Grain) -> dict:
    return dict(q=g.q, m=g.m, pos=np.array([g.x, g.y, g.z]), vel=np.array([g.vx, g.vy, g.vz]),
                tot_absor_e=g.tot_absor_e, t_steps=g.t_steps, chi_b=g.chi_b)


def _grain_c(d: Optional[dict]) -> Optional[_Grain]:
    if d is None:
        return None
    g = _Grain()
    g.q = int(d.get("q", 0))
    g.m = float(d.get("m", 1.67e-12))
    pos = d.get("pos", (0.0, 0.0, 0.0))
    vel = d.get("vel", (0.0, 0.0, 0.0))
    g.x, g.y, g.z = (float(v) for v in pos)
    g.vx, g.vy, g.vz = (float(v) for v in vel)
    g.tot_absor_e = int(d.get("tot_absor_e", 0))
    g.t_steps = int(d.get("t_steps", 0))
    g.chi_b = float(d.get("chi_b", 0.0))
    return g


class Run:
    """One simulation run on one GPU (a ``pot_gpu_ctx``)."""

    def __init__(self, cfg: RunConfig, form: str = "plain", leaf_size: int = 0, group_size: int = 0,
                 seed: int = 1, device: int = 0, stream: Optional[int] = None, timing: bool = False,
                 chi_b_ranks: int = 0, chi_cap: bool = False):
        self.lib = load_library()
        self.cfg = cfg
        o = _Opts()
        o.form = FORM_PLAIN if form == "plain" else FORM_FAST
        o.leaf_size = int(leaf_size)
        o.group_size = int(group_size)
        o.flags = (OPT_TIMING if timing else 0) | (OPT_CHI_CAP if chi_cap else 0)
        o.device = int(device)
        o.seed = int(seed) & ((1 << 64) - 1)
        o.stream = stream
        o.chi_b_ranks = int(chi_b_ranks)
        self.form = form
        self.h = C.c_void_p()
        self._check(self.lib.pot_gpu_create(C.byref(cfg.to_c()), C.byref(o), C.byref(self.h)), "pot_gpu_create")

    def _check(self, rc: int, where: str):
        if rc != POT_OK:
            msg = self.lib.pot_gpu_strerror(rc).decode()
            raise PotError(rc, where, msg)
        return rc

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            self.lib.pot_gpu_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- state ------------------------------------------------------------------
    def upload(self, parts: np.ndarray, grain: Optional[dict] = None):
        parts = np.ascontiguousarray(parts, dtype=PARTICLE_DTYPE)
        g = _grain_c(grain)
        self._check(self.lib.pot_gpu_upload(self.h, _ptr(parts), len(parts), C.byref(g) if g else None),
                    "pot_gpu_upload")

    def init_particles(self):
        self._check(self.lib.pot_gpu_init_particles(self.h), "pot_gpu_init_particles")

    def step(self, n: int = 1, epe: bool = False) -> dict:
        """Run n steps; epe=True also computes the potential energies."""
        st = _Stats()
        rc = self.lib.pot_gpu_step(self.h, int(n), STEP_EPE if epe else 0, C.byref(st))
        if rc != POT_OK:
            e = PotError(rc, "pot_gpu_step", self.lib.pot_gpu_strerror(rc).decode())
            e.stats = _stats_dict(st)  # the run record at the failure (the library fills it)
            raise e
        return _stats_dict(st)

    def step_async(self, n: int = 1, epe: bool = False):
        """Enqueue n steps without waiting (errors surface at the next sync)."""
        self._check(self.lib.pot_gpu_step_async(self.h, int(n), STEP_EPE if epe else 0), "pot_gpu_step_async")

    def download(self):
        out = np.zeros(self.cfg.N, PARTICLE_DTYPE)
        g = _Grain()
        self._check(self.lib.pot_gpu_download(self.h, _ptr(out), C.byref(g)), "pot_gpu_download")
        return out, _grain_dict(g)

    def move_particles(self, parts: np.ndarray, grain: Optional[dict] = None):
        """Drop-in for one run() iteration: in-place on ``parts``."""
        assert parts.dtype == PARTICLE_DTYPE and parts.flags.c_contiguous
        g = _grain_c(grain) or _grain_c(dict(pos=(parts[0]["x"], parts[0]["y"], parts[0]["z"])))
        st = _Stats()
        self._check(self.lib.pot_gpu_move_particles(self.h, _ptr(parts), len(parts), C.byref(g), C.byref(st)),
                    "pot_gpu_move_particles")
        return _grain_dict(g), _stats_dict(st)

    def macro(self) -> dict:
        """The macroscopic-summary sums of the current state, on the device."""
        m = _MacroSums()
        self._check(self.lib.pot_gpu_macro(self.h, C.byref(m)), "pot_gpu_macro")
        out = {}
        for k, t in _MacroSums._fields_:
            if k.startswith("pad"):
                continue
            v = getattr(m, k)
            out[k] = np.array(list(v)) if hasattr(v, "__len__") else v
        return out

    def grain(self) -> dict:
        g = _Grain()
        self._check(self.lib.pot_gpu_grain(self.h, C.byref(g)), "pot_gpu_grain")
        return _grain_dict(g)

    def set_ion_temp(self, Ti: float):
        """The cached ion temperature of the Poisson ion collection."""
        self._check(self.lib.pot_gpu_set_ion_temp(self.h, float(Ti)), "pot_gpu_set_ion_temp")

    def ion_temp(self) -> float:
        t = C.c_double()
        self._check(self.lib.pot_gpu_ion_temp(self.h, C.byref(t)), "pot_gpu_ion_temp")
        return t.value

    # -- inspection ---------------------------------------------------------------
    def build_tree(self) -> int:
        n = C.c_uint64()
        self._check(self.lib.pot_gpu_build_tree(self.h, C.byref(n)), "pot_gpu_build_tree")
        return n.value

    def tree_dump(self) -> dict:
        mx = 9 * self.cfg.N + 16
        ni, nl = C.c_uint64(), C.c_uint64()
        il = np.zeros(mx, np.int32)
        ip = np.zeros(mx, np.uint64)
        iq = np.zeros(mx, np.int32)
        iaq = np.zeros(mx, np.uint32)
        ic = np.zeros((mx, 3), np.float64)
        iw = np.zeros(mx, np.float64)
        lp = np.zeros(mx, np.uint32)
        ll = np.zeros(mx, np.int32)
        lpa = np.zeros(mx, np.uint64)
        self._check(self.lib.pot_gpu_tree_dump(self.h, mx, C.byref(ni), _ptr(il), _ptr(ip), _ptr(iq), _ptr(iaq),
                                               _ptr(ic), _ptr(iw), C.byref(nl), _ptr(lp), _ptr(ll), _ptr(lpa)),
                    "pot_gpu_tree_dump")
        a, b = ni.value, nl.value
        return dict(int_level=il[:a], int_path=ip[:a], int_q=iq[:a], int_aq=iaq[:a], int_c=ic[:a],
                    int_w=iw[:a], leaf_part=lp[:b], leaf_level=ll[:b], leaf_path=lpa[:b])

    def field_at(self, idx, xyz) -> np.ndarray:
        idx = np.ascontiguousarray(idx, np.uint32)
        xyz = np.ascontiguousarray(xyz, np.float64).reshape(-1, 3)
        out = np.zeros_like(xyz)
        self._check(self.lib.pot_gpu_field_at(self.h, len(idx), _ptr(idx), _ptr(xyz), _ptr(out)),
                    "pot_gpu_field_at")
        return out

    def field_at_noalloc(self, idx, xyz) -> np.ndarray:
        """field_at through the entry point that allocates no device memory
        (at most NOALLOC_MAX_POINTS points per call)."""
        idx = np.ascontiguousarray(idx, np.uint32)
        xyz = np.ascontiguousarray(xyz, np.float64).reshape(-1, 3)
        out = np.zeros_like(xyz)
        self._check(self.lib.pot_gpu_field_at_noalloc(self.h, len(idx), _ptr(idx), _ptr(xyz), _ptr(out)),
                    "pot_gpu_field_at_noalloc")
        return out

    def phi_at(self, xyz) -> np.ndarray:
        xyz = np.ascontiguousarray(xyz, np.float64).reshape(-1, 3)
        out = np.zeros(len(xyz))
        self._check(self.lib.pot_gpu_phi_at(self.h, len(xyz), _ptr(xyz), _ptr(out)), "pot_gpu_phi_at")
        return out

    def kernel_times(self) -> dict:
        n = 64
        names = (C.c_char_p * n)()
        ms = (C.c_double * n)()
        cnt = (C.c_uint64 * n)()
        k = self.lib.pot_gpu_kernel_times(self.h, n, names, ms, cnt)
        return {names[i].decode(): (ms[i], cnt[i]) for i in range(min(k, n))}

    def reset_kernel_times(self):
        self._check(self.lib.pot_gpu_reset_kernel_times(self.h), "pot_gpu_reset_kernel_times")

    def launch_count(self) -> int:
        n = C.c_uint64()
        self._check(self.lib.pot_gpu_launch_count(self.h, C.byref(n)), "pot_gpu_launch_count")
        return n.value

    def sync(self):
        self._check(self.lib.pot_gpu_sync(self.h), "pot_gpu_sync")


def _opts(form="fast", leaf_size=0, group_size=0, seed=1, device=0, chi_cap=False) -> _Opts:
    o = _Opts()
    o.flags = OPT_CHI_CAP if chi_cap else 0
    o.form = FORM_PLAIN if form == "plain" else FORM_FAST
    o.leaf_size = int(leaf_size)
    o.group_size = int(group_size)
    o.device = int(device)
    o.seed = int(seed) & ((1 << 64) - 1)
    return o


def bytes_needed(cfg: RunConfig, form="fast", leaf_size=0, group_size=0) -> int:
    """Device bytes a run with these settings allocates."""
    L = load_library()
    b = C.c_uint64()
    rc = L.pot_gpu_bytes_needed(C.byref(cfg.to_c()), C.byref(_opts(form, leaf_size, group_size)), C.byref(b))
    if rc != POT_OK:
        raise PotError(rc, "pot_gpu_bytes_needed", L.pot_gpu_strerror(rc).decode())
    return b.value


def tune(cfg: RunConfig, steps: int = 6, seed: int = 1, device: int = 0):
    """Autotuner: the fastest (leaf size, group size) of the fast form for
    this run, and its ms per step."""
    L = load_library()
    o = _opts("fast", seed=seed, device=device)
    ms = C.c_double()
    rc = L.pot_gpu_tune(C.byref(cfg.to_c()), C.byref(o), int(steps), C.byref(ms))
    if rc != POT_OK:
        raise PotError(rc, "pot_gpu_tune", L.pot_gpu_strerror(rc).decode())
    return dict(leaf_size=o.leaf_size, group_size=o.group_size, ms_per_step=ms.value)


class Batch:
    """Many independent runs stepped by one CUDA-graph launch
    (``pot_batch``)."""

    def __init__(self, device: int = 0, steps_per_launch: int = 2, reserve_bytes: int = 0, pack: bool = True):
        self.lib = load_library()
        o = _BatchOpts()
        o.device, o.steps_per_launch, o.reserve_bytes = int(device), int(steps_per_launch), int(reserve_bytes)
        o.flags = 0 if pack else BATCH_NO_PACK
        self.h = C.c_void_p()
        self.cfgs = {}
        self._check(self.lib.pot_batch_create(C.byref(o), C.byref(self.h)), "pot_batch_create")

    def _check(self, rc, where):
        if rc != POT_OK:
            raise PotError(rc, where, self.lib.pot_gpu_strerror(rc).decode())
        return rc

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            self.lib.pot_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def admit(self, cfg: RunConfig, form="fast", leaf_size=0, group_size=0, seed=1, parts=None, grain=None,
              chi_cap=False) -> int:
        slot = C.c_int32(-1)
        o = _opts(form, leaf_size, group_size, seed, chi_cap=chi_cap)
        pp = None
        if parts is not None:
            parts = np.ascontiguousarray(parts, dtype=PARTICLE_DTYPE)
            pp = _ptr(parts)
        g = _grain_c(grain)
        self._check(self.lib.pot_batch_admit(self.h, C.byref(cfg.to_c()), C.byref(o), pp, C.byref(g) if g else None,
                                             C.byref(slot)), "pot_batch_admit")
        self.cfgs[slot.value] = cfg
        return slot.value

    def try_admit(self, *a, **k):
        """admit, or None when the run does not fit in free HBM."""
        try:
            return self.admit(*a, **k)
        except PotError as e:
            if e.status == -3:
                return None
            raise

    def evict(self, slot: int):
        self._check(self.lib.pot_batch_evict(self.h, int(slot)), "pot_batch_evict")
        self.cfgs.pop(slot, None)

    def step(self, n: int = 2):
        self._check(self.lib.pot_batch_step(self.h, int(n)), "pot_batch_step")

    def sync(self):
        self._check(self.lib.pot_batch_sync(self.h), "pot_batch_sync")

    def summary(self) -> np.ndarray:
        cap = max(1, len(self.cfgs))
        rows = np.zeros(cap, BATCH_ROW_DTYPE)
        n = C.c_uint32()
        self._check(self.lib.pot_batch_summary(self.h, cap, _ptr(rows), C.byref(n)), "pot_batch_summary")
        return rows[:n.value]

    def count(self):
        r, p, b = C.c_uint32(), C.c_uint64(), C.c_uint64()
        self._check(self.lib.pot_batch_count(self.h, C.byref(r), C.byref(p), C.byref(b)), "pot_batch_count")
        return dict(runs=r.value, particles=p.value, bytes=b.value)

    def download(self, slot: int):
        h = C.c_void_p()
        self._check(self.lib.pot_batch_ctx(self.h, int(slot), C.byref(h)), "pot_batch_ctx")
        cfg = self.cfgs[slot]
        out = np.zeros(cfg.N, PARTICLE_DTYPE)
        g = _Grain()
        self._check(self.lib.pot_gpu_download(h, _ptr(out), C.byref(g)), "pot_gpu_download")
        return out, _grain_dict(g)
