"""ctypes loaders for the CPU oracle (test infrastructure only).

* :class:`Ref` wraps ``oracle/_ref/libpotref_<variant>.so`` -- the reference
  program itself, compiled by ``oracle/build.py`` from the reference tree
  (present only where that tree is; never on a GPU box unless prebuilt).
* :class:`Oracle` wraps ``oracle/libpotoracle.so`` -- the project's own C
  restatement of the reference's per-step loop (``oracle/pot_oracle.c``).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this module; the GPU product path never does.
"""
from __future__ import annotations

import ctypes as C
import os
import struct

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# Particle record of pot.c:295-303: six doubles + enum Species, padded to 56 B.
PARTICLE_DTYPE = np.dtype([("x", "<f8"), ("y", "<f8"), ("z", "<f8"),
                           ("vx", "<f8"), ("vy", "<f8"), ("vz", "<f8"),
                           ("species", "<i4"), ("_pad", "<i4")])
assert PARTICLE_DTYPE.itemsize == 56
DUST, ION, ELECTRON = 0, 1, 2

_u64 = (1 << 64) - 1


def splitmix64_words(seed: int, n: int = 16):
    """n uint32 words from the splitmix64 stream seeded with ``seed``.

    This is the project's convention for turning an integer seed into the
    reference's 512-bit WELL512 seed (pot.c:5168-5179 reads 16 uint32 words
    from its randomness source)."""
    out = []
    x = seed & _u64
    while len(out) < n:
        x = (x + 0x9E3779B97F4A7C15) & _u64
        z = x
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _u64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _u64
        z ^= z >> 31
        out.append(z & 0xFFFFFFFF)
        out.append(z >> 32)
    return np.array(out[:n], dtype=np.uint32)


def shape_of(A: float) -> int:
    """Grain shape code: 0 sphere (pot.c), 1 prolate (A > 1), 2 oblate
    (0 < A < 1) -- pot-spheroid.c's PROLATE / OBLATE programs."""
    if not A:
        return 0
    if A > 1.0:
        return 1
    if 0.0 < A < 1.0:
        return 2
    raise ValueError("aspect ratio must be 0 (sphere), > 1 (prolate) or in (0, 1) (oblate)")


class RunParams:
    """The reference's Run settings (pot.c:335-358) for a spherical domain.
    ``A`` is pot-spheroid.c's aspect ratio (Run.A, pot-spheroid.c:376-378;
    0 = the spherical grain of pot.c) and ``axis`` the spheroid's symmetry
    axis (x in the reference; any other unit vector is this project's
    extension, unpinned).  The reference's other compile-time variants:
    ``bounce`` (OUT_BOUNCE, the wall's coefficient of restitution; 0 =
    reinjection), ``integrator`` (0 Boris, 1 velocity Verlet, 2
    Euler-Richardson), ``dipoles`` (DIPOLES) and ``pois_ions``
    (POIS_POS_COLLECTION)."""

    def __init__(self, N, r, dt, mpp, soft, Te, Ti, x_drift=0.0, a=2.5e-6, settle=0.0,
                 theta=0.5, B=(0.0, 0.0, 0.0), A=0.0, axis=(1.0, 0.0, 0.0), bounce=0.0, integrator=0,
                 dipoles=False, pois_ions=False):
        self.N = int(N)
        self.r = int(r)
        self.dt = float(dt)
        self.mpp = float(mpp)
        self.soft = float(soft)
        self.Te = float(Te)
        self.Ti = float(Ti)
        self.x_drift = float(x_drift)
        self.a = float(a)
        self.settle = float(settle)
        self.theta = float(theta)
        self.B = tuple(float(b) for b in B)
        self.A = float(A)
        self.axis = tuple(float(u) for u in axis)
        self.shape = shape_of(self.A)
        self.bounce = float(bounce)
        self.integrator = int(integrator)
        self.dipoles = bool(dipoles)
        self.pois_ions = bool(pois_ions)

    def as_dict(self):
        return dict(N=self.N, r=self.r, dt=self.dt, mpp=self.mpp, soft=self.soft, Te=self.Te,
                    Ti=self.Ti, x_drift=self.x_drift, a=self.a, settle=self.settle,
                    theta=self.theta, B=list(self.B), A=self.A, axis=list(self.axis), bounce=self.bounce,
                    integrator=self.integrator, dipoles=self.dipoles, pois_ions=self.pois_ions)

    def variant_flags(self) -> int:
        """The bits of the reference harness's potref_variant_flags."""
        return ((1 if self.dipoles else 0) | (2 if self.bounce else 0) | (4 if self.pois_ions else 0)
                | (8 if self.integrator else 0) | (16 if self.integrator == 2 else 0))


def _ptr(a, t=C.c_void_p):
    return a.ctypes.data_as(t)


def _load(path):
    lib = C.CDLL(path)
    return lib


class RefLib:
    """The compiled reference (one library per variant, one run per process)."""

    def __init__(self, variant: str = "sceptic", build: bool = True):
        import importlib.util
        spec = importlib.util.spec_from_file_location("_oracle_build", os.path.join(HERE, "build.py"))
        b = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(b)
        path = b.ref_lib_path(variant)
        if build:
            b.build_ref(variants=(variant,))
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.variant = variant
        self.lib = _load(path)
        L = self.lib
        L.potref_setup.argtypes = [C.c_ulong, C.c_uint, C.c_double, C.c_double, C.c_double,
                                   C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                   C.c_double, C.c_double, C.c_double, C.c_double,
                                   C.c_void_p, C.c_int, C.c_int, C.c_int]
        L.potref_setup.restype = C.c_int
        L.potref_build_tree.restype = C.c_int
        L.potref_step.argtypes = [C.c_int]
        L.potref_step.restype = C.c_int
        L.potref_run_steps.argtypes = [C.c_ulong, C.c_int]
        L.potref_run_steps.restype = C.c_int
        L.potref_move.argtypes = [C.c_ulong, C.c_int]
        L.potref_get_particles.argtypes = [C.c_void_p]
        L.potref_set_particles.argtypes = [C.c_void_p]
        L.potref_get_grain.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_uint),
                                       C.POINTER(C.c_ulong), C.POINTER(C.c_double)]
        L.potref_set_grain.argtypes = [C.c_int, C.c_double, C.c_uint, C.c_ulong, C.c_double]
        L.potref_get_prng.argtypes = [C.c_void_p]
        L.potref_set_prng.argtypes = [C.c_void_p]
        L.potref_get_tss.argtypes = [C.c_void_p]
        L.potref_tree_dump.argtypes = [C.c_ulong, C.POINTER(C.c_ulong), C.c_void_p, C.c_void_p,
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.POINTER(C.c_ulong), C.c_void_p, C.c_void_p, C.c_void_p]
        L.potref_tree_dump.restype = C.c_int
        L.potref_field_many.argtypes = [C.c_ulong, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        self.has_phi_at = bool(L.potref_has_phi_at())
        if self.has_phi_at:
            L.potref_phi_at.argtypes = [C.c_double, C.c_double, C.c_double]
            L.potref_phi_at.restype = C.c_double
        L.potref_phi_particle_feels.argtypes = [C.c_uint, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.potref_cross_grain.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double]
        L.potref_cross_grain.restype = C.c_int
        L.potref_inject.argtypes = [C.c_void_p, C.c_int]
        L.potref_get_epe.argtypes = [C.c_void_p]
        L.potref_set_aspect.argtypes = [C.c_double]
        L.potref_set_aspect.restype = None
        self.variant_flags = int(L.potref_variant_flags())
        L.potref_bounce.restype = C.c_double
        self.bounce = float(L.potref_bounce())
        if self.variant_flags & 4:
            L.potref_set_ion_temp.argtypes = [C.c_double]
            L.potref_ion_temp.restype = C.c_double
            L.potref_pos_rate_const.restype = C.c_double
        if self.variant_flags & 1:
            L.potref_tree_dipoles.argtypes = [C.c_ulong, C.c_void_p]
            L.potref_tree_dipoles.restype = C.c_long
        L.potref_write_state.argtypes = [C.c_char_p]
        L.potref_read_state.argtypes = [C.c_char_p]
        L.potref_read_state.restype = C.c_int
        self.has_write_phi = bool(L.potref_has_write_phi())
        if self.has_write_phi:
            L.potref_write_phi.argtypes = [C.c_char_p, C.c_ulong]
        self.shape = int(L.potref_shape())
        self.grain_enabled = bool(L.potref_grain_enabled())
        self.sceptic = bool(L.potref_has_sceptic())
        if self.sceptic:
            L.potref_measure_chi_b.restype = C.c_double
            for fn in ("potref_u_icdf", "potref_integrate_for_alpha"):
                getattr(L, fn).restype = C.c_double
            L.potref_u_icdf.argtypes = [C.c_double] * 3
            L.potref_u_no_flow_icdf.argtypes = [C.c_double] * 2
            L.potref_u_no_flow_icdf.restype = C.c_double
            L.potref_integrate_for_alpha.argtypes = [C.c_double] * 4
        self.N = 0
        self.prng_size = L.potref_sizeof_prng()
        assert L.potref_sizeof_particle() == 56

    # -- set-up ---------------------------------------------------------------
    def setup(self, p: RunParams, seed: int = 1, init: bool = True, nprocs: int = 1, rank: int = 0):
        """Set up a run; with nprocs > 1 this process plays MPI rank `rank`
        (it builds the whole tree and steps only its own block)."""
        words = splitmix64_words(seed)
        if p.shape != self.shape:
            raise ValueError("run shape %d does not match the %s program" % (p.shape, self.variant))
        if p.variant_flags() != self.variant_flags or (p.bounce and p.bounce != self.bounce):
            raise ValueError("run variants do not match the %s program" % self.variant)
        if self.shape:
            if p.axis != (1.0, 0.0, 0.0):
                raise ValueError("the reference's spheroid axis is x")
            self.lib.potref_set_aspect(p.A)
        rc = self.lib.potref_setup(p.N, p.r, p.dt, p.mpp, p.soft, p.Te, p.Ti, p.x_drift, p.a,
                                   p.settle, p.theta, p.B[0], p.B[1], p.B[2], _ptr(words),
                                   1 if init else 0, int(nprocs), int(rank))
        if rc != 0:
            raise RuntimeError("potref_setup failed: %d" % rc)
        self.N = p.N
        self.params = p
        return self

    def tss(self):
        out = np.zeros(3, np.uint32)
        self.lib.potref_get_tss(_ptr(out))
        return out

    def particles(self):
        out = np.zeros(self.N, PARTICLE_DTYPE)
        self.lib.potref_get_particles(_ptr(out))
        return out

    def set_particles(self, parts):
        parts = np.ascontiguousarray(parts, dtype=PARTICLE_DTYPE)
        assert parts.shape[0] == self.N
        self.lib.potref_set_particles(_ptr(parts))

    def grain(self):
        q, m, e, t, chi = C.c_int(), C.c_double(), C.c_uint(), C.c_ulong(), C.c_double()
        self.lib.potref_get_grain(C.byref(q), C.byref(m), C.byref(e), C.byref(t), C.byref(chi))
        return dict(q=q.value, m=m.value, tot_absor_e=e.value, t_steps=t.value, chi_b=chi.value)

    def set_grain(self, q=0, m=1.67e-12, tot_absor_e=0, t_steps=0, chi_b=0.0):
        self.lib.potref_set_grain(int(q), float(m), int(tot_absor_e), int(t_steps), float(chi_b))

    def prng(self) -> bytes:
        buf = (C.c_char * self.prng_size)()
        self.lib.potref_get_prng(buf)
        return bytes(buf)

    def write_state(self, path: str):
        """The reference's write_sim_state_to_file (format C, pot.c:3816-3901)."""
        self.lib.potref_write_state(os.fsencode(path))

    def read_state(self, path: str):
        """The reference's read_sim_state_from_file (pot.c:3904-4019)."""
        if self.lib.potref_read_state(os.fsencode(path)) != 0:
            raise RuntimeError("the reference failed to read the state file %s" % path)

    def write_phi(self, path: str, time_step: int):
        """The reference's write_phi_data_to_file (pot.c:3001-3042) over the
        tree last built, rows appended to path."""
        self.lib.potref_write_phi(os.fsencode(path), int(time_step))

    def set_prng(self, blob: bytes):
        buf = (C.c_char * self.prng_size).from_buffer_copy(blob)
        self.lib.potref_set_prng(buf)

    # -- hot path -------------------------------------------------------------
    def build_tree(self):
        if self.lib.potref_build_tree() != 0:
            raise RuntimeError("reference build_tree returned NULL")

    def tree_dump(self):
        mx = 9 * self.N + 16
        ni, nl = C.c_ulong(), C.c_ulong()
        il = np.zeros(mx, np.int32)
        ip = np.zeros(mx, np.uint64)
        iq = np.zeros(mx, np.int32)
        iaq = np.zeros(mx, np.uint32)
        ic = np.zeros((mx, 3), np.float64)
        iw = np.zeros(mx, np.float64)
        lp = np.zeros(mx, np.uint32)
        ll = np.zeros(mx, np.int32)
        lpa = np.zeros(mx, np.uint64)
        rc = self.lib.potref_tree_dump(mx, C.byref(ni), _ptr(il), _ptr(ip), _ptr(iq), _ptr(iaq),
                                       _ptr(ic), _ptr(iw), C.byref(nl), _ptr(lp), _ptr(ll), _ptr(lpa))
        if rc != 0:
            raise RuntimeError("tree dump overflow")
        a, b = ni.value, nl.value
        return dict(int_level=il[:a], int_path=ip[:a], int_q=iq[:a], int_aq=iaq[:a],
                    int_c=ic[:a], int_w=iw[:a], leaf_part=lp[:b], leaf_level=ll[:b],
                    leaf_path=lpa[:b])

    def field_many(self, idx, xyz):
        idx = np.ascontiguousarray(idx, np.uint32)
        xyz = np.ascontiguousarray(xyz, np.float64).reshape(-1, 3)
        hi = np.zeros_like(xyz)
        lo = np.zeros_like(xyz)
        self.lib.potref_field_many(len(idx), _ptr(idx), _ptr(xyz), _ptr(hi), _ptr(lo))
        return hi, lo

    def phi_at(self, x, y, z):
        return self.lib.potref_phi_at(x, y, z)

    def phi_particle_feels(self, i):
        hi, lo = C.c_double(), C.c_double()
        self.lib.potref_phi_particle_feels(int(i), C.byref(hi), C.byref(lo))
        return hi.value, lo.value

    def cross_grain(self, p, d_pos, gr, a):
        p = np.ascontiguousarray(p, PARTICLE_DTYPE).reshape(1)
        gr = np.ascontiguousarray(gr, PARTICLE_DTYPE).reshape(1)
        d = np.ascontiguousarray(d_pos, np.float64)
        return bool(self.lib.potref_cross_grain(_ptr(p), _ptr(d), _ptr(gr), float(a)))

    def inject(self, p, reinjection=True):
        p = np.ascontiguousarray(p, PARTICLE_DTYPE).reshape(1).copy()
        self.lib.potref_inject(_ptr(p), 1 if reinjection else 0)
        return p[0]

    def step(self, compute_epe=False):
        if self.lib.potref_step(1 if compute_epe else 0) != 0:
            raise RuntimeError("reference step failed (build_tree NULL)")

    def run_steps(self, n, compute_epe=False):
        if self.lib.potref_run_steps(int(n), 1 if compute_epe else 0) != 0:
            raise RuntimeError("reference run failed")

    def move(self, time_steps, compute_epe=False):
        self.lib.potref_move(int(time_steps), 1 if compute_epe else 0)

    def epe(self):
        out = np.zeros(3, np.float64)
        self.lib.potref_get_epe(_ptr(out))
        return out

    def measure_chi_b(self):
        return self.lib.potref_measure_chi_b()

    def set_ion_temp(self, Ti):
        self.lib.potref_set_ion_temp(float(Ti))

    def ion_temp(self):
        return self.lib.potref_ion_temp()

    def pos_rate_const(self):
        return self.lib.potref_pos_rate_const()

    def tree_dipoles(self):
        mx = 9 * self.N + 16
        out = np.zeros((mx, 3))
        n = self.lib.potref_tree_dipoles(mx, _ptr(out))
        if n < 0:
            raise RuntimeError("tree dump overflow")
        return out[:n]


class _PtoCfg(C.Structure):
    _fields_ = [("N", C.c_uint64), ("r", C.c_uint32), ("dt", C.c_double), ("mpp", C.c_double),
                ("soft", C.c_double), ("Te", C.c_double), ("Ti", C.c_double),
                ("x_drift", C.c_double), ("a", C.c_double), ("settle", C.c_double),
                ("theta", C.c_double), ("B", C.c_double * 3), ("sceptic", C.c_int32),
                ("quirk", C.c_int32), ("rng", C.c_int32), ("pad", C.c_int32), ("seed", C.c_uint64),
                ("shape", C.c_int32), ("chi_ranks", C.c_int32), ("A", C.c_double), ("axis", C.c_double * 3),
                ("bounce", C.c_double), ("integrator", C.c_int32), ("dipoles", C.c_int32),
                ("pois_ions", C.c_int32), ("pad2", C.c_int32)]


WELL_DTYPE = np.dtype([("abcd", "<u4", 4), ("index", "<u4"), ("state", "<u4", 16)])


class Oracle:
    """The C restatement (``oracle/pot_oracle.c``), one run per instance.

    ``mode="reference"``: the reference's in-place half-drift ordering and a
    WELL512 stream seeded like pot.c (bit-for-bit the reference program).
    ``mode="gpu"``: pre-step sources for every target and the Philox counter
    stream of the CUDA kernels (what the GPU path computes)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            import importlib.util
            spec = importlib.util.spec_from_file_location("_oracle_build", os.path.join(HERE, "build.py"))
            b = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(b)
            L = C.CDLL(b.build_oracle())
            vp, u64, i32, u32, d = C.c_void_p, C.c_uint64, C.c_int32, C.c_uint32, C.c_double
            L.pto_create.argtypes = [vp]
            L.pto_create.restype = vp
            L.pto_destroy.argtypes = [vp]
            for fn in ("pto_set_particles", "pto_get_particles", "pto_set_well", "pto_get_well",
                       "pto_seed_well", "pto_get_tss"):
                getattr(L, fn).argtypes = [vp, vp]
            L.pto_set_grain.argtypes = [vp, i32, d, u32, u64, d]
            L.pto_get_grain.argtypes = [vp, vp, vp, vp, vp, vp, vp]
            L.pto_init_particles.argtypes = [vp]
            L.pto_build_tree.argtypes = [vp]
            L.pto_tree_dump.argtypes = [vp, u64, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]
            L.pto_field_many.argtypes = [vp, u64, vp, vp, vp, vp]
            L.pto_field_direct_many.argtypes = [vp, u64, vp, vp, i32, vp, vp]
            L.pto_phi_at.argtypes = [vp, d, d, d]
            L.pto_phi_at.restype = d
            L.pto_phi_particle_feels.argtypes = [vp, u32]
            L.pto_phi_particle_feels.restype = d
            L.pto_cross_grain.argtypes = [vp, vp, vp, d]
            L.pto_cross_grain_run.argtypes = [vp, vp, vp, vp]
            L.pto_grain_field.argtypes = [vp, d, d, d, vp]
            L.pto_grain_field.restype = None
            L.pto_grain_phi.argtypes = [vp, d, d, d]
            L.pto_grain_phi.restype = d
            L.pto_integrate_for_alpha_dev.argtypes = [d, d, d, d, d]
            L.pto_integrate_for_alpha_dev.restype = d
            L.pto_measure_chi_b.argtypes = [vp]
            L.pto_measure_chi_b.restype = d
            L.pto_measure_chi_b_ranks.argtypes = [vp, i32]
            L.pto_measure_chi_b_ranks.restype = d
            L.pto_step.argtypes = [vp, i32]
            L.pto_run_steps.argtypes = [vp, u64, i32]
            L.pto_last_step_stats.argtypes = [vp, vp, vp, vp, vp, vp, vp]
            L.pto_sample_reinject.argtypes = [vp, u64, i32, vp]
            L.pto_u_icdf.argtypes = [d, d, d]
            L.pto_u_icdf.restype = d
            L.pto_u_no_flow_icdf.argtypes = [d, d]
            L.pto_u_no_flow_icdf.restype = d
            L.pto_integrate_for_alpha.argtypes = [d, d, d, d]
            L.pto_integrate_for_alpha.restype = d
            L.pto_philox4x32.argtypes = [vp, vp, vp]
            L.pto_set_ion_temp.argtypes = [vp, d]
            L.pto_ion_temp.argtypes = [vp]
            L.pto_ion_temp.restype = d
            L.pto_poisson.argtypes = [vp, d]
            L.pto_poisson.restype = u32
            L.pto_tree_dipoles.argtypes = [vp, u64, vp]
            L.pto_tree_dipoles.restype = C.c_int64
            L.pto_last_step_variant_stats.argtypes = [vp, vp, vp]
            assert L.pto_sizeof_particle() == 56
            cls._lib = L
        return cls._lib

    def __init__(self, p: RunParams, mode: str = "reference", sceptic: bool = True, seed: int = 1,
                 init: bool = True, chi_ranks: int = 0):
        L = self.lib()
        cfg = _PtoCfg()
        cfg.N, cfg.r, cfg.dt, cfg.mpp, cfg.soft = p.N, p.r, p.dt, p.mpp, p.soft
        cfg.Te, cfg.Ti, cfg.x_drift, cfg.a, cfg.settle, cfg.theta = p.Te, p.Ti, p.x_drift, p.a, p.settle, p.theta
        for k in range(3):
            cfg.B[k] = p.B[k]
        cfg.sceptic = 1 if sceptic else 0
        cfg.quirk = 1 if mode == "reference" else 0
        cfg.rng = 0 if mode == "reference" else 1
        cfg.seed = seed & ((1 << 64) - 1)
        cfg.shape = p.shape
        cfg.chi_ranks = int(chi_ranks)
        cfg.A = p.A
        for k in range(3):
            cfg.axis[k] = p.axis[k]
        cfg.bounce = p.bounce
        cfg.integrator = p.integrator
        cfg.dipoles = 1 if p.dipoles else 0
        cfg.pois_ions = 1 if p.pois_ions else 0
        self.cfg = cfg
        self.params = p
        self.mode = mode
        self.seed = seed
        self.sceptic = sceptic
        self.N = p.N
        self.h = L.pto_create(C.byref(cfg))
        if not self.h:
            raise MemoryError("pto_create failed")
        words = splitmix64_words(seed)
        L.pto_seed_well(self.h, _ptr(words))
        if init:
            L.pto_init_particles(self.h)

    def __del__(self):
        try:
            if self.h:
                self.lib().pto_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def tss(self):
        out = np.zeros(3, np.uint32)
        self.lib().pto_get_tss(self.h, _ptr(out))
        return out

    def particles(self):
        out = np.zeros(self.N, PARTICLE_DTYPE)
        self.lib().pto_get_particles(self.h, _ptr(out))
        return out

    def set_particles(self, parts):
        parts = np.ascontiguousarray(parts, dtype=PARTICLE_DTYPE)
        assert parts.shape[0] == self.N
        self.lib().pto_set_particles(self.h, _ptr(parts))

    def well(self) -> bytes:
        w = np.zeros(1, WELL_DTYPE)
        self.lib().pto_get_well(self.h, _ptr(w))
        return w.tobytes()

    def set_well(self, blob: bytes):
        w = np.frombuffer(blob, WELL_DTYPE).copy()
        self.lib().pto_set_well(self.h, _ptr(w))

    def grain(self):
        q, m, e, t, chi = C.c_int32(), C.c_double(), C.c_uint32(), C.c_uint64(), C.c_double()
        v = np.zeros(3)
        self.lib().pto_get_grain(self.h, C.byref(q), C.byref(m), C.byref(e), C.byref(t), C.byref(chi), _ptr(v))
        return dict(q=q.value, m=m.value, tot_absor_e=e.value, t_steps=t.value, chi_b=chi.value, v=v)

    def set_grain(self, q=0, m=1.67e-12, tot_absor_e=0, t_steps=0, chi_b=0.0):
        self.lib().pto_set_grain(self.h, int(q), float(m), int(tot_absor_e), int(t_steps), float(chi_b))

    def build_tree(self):
        rc = self.lib().pto_build_tree(self.h)
        if rc != 0:
            raise RuntimeError("oracle build_tree failed: %d" % rc)

    def tree_dump(self):
        mx = 9 * self.N + 16
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
        rc = self.lib().pto_tree_dump(self.h, mx, C.byref(ni), _ptr(il), _ptr(ip), _ptr(iq), _ptr(iaq),
                                      _ptr(ic), _ptr(iw), C.byref(nl), _ptr(lp), _ptr(ll), _ptr(lpa))
        if rc != 0:
            raise RuntimeError("tree dump overflow")
        a, b = ni.value, nl.value
        return dict(int_level=il[:a], int_path=ip[:a], int_q=iq[:a], int_aq=iaq[:a],
                    int_c=ic[:a], int_w=iw[:a], leaf_part=lp[:b], leaf_level=ll[:b],
                    leaf_path=lpa[:b])

    def field_many(self, idx, xyz):
        idx = np.ascontiguousarray(idx, np.uint32)
        xyz = np.ascontiguousarray(xyz, np.float64).reshape(-1, 3)
        hi = np.zeros_like(xyz)
        lo = np.zeros_like(xyz)
        self.lib().pto_field_many(self.h, len(idx), _ptr(idx), _ptr(xyz), _ptr(hi), _ptr(lo))
        return hi, lo

    def field_direct_many(self, idx, xyz, soften_all=False):
        idx = np.ascontiguousarray(idx, np.uint32)
        xyz = np.ascontiguousarray(xyz, np.float64).reshape(-1, 3)
        hi = np.zeros_like(xyz)
        lo = np.zeros_like(xyz)
        self.lib().pto_field_direct_many(self.h, len(idx), _ptr(idx), _ptr(xyz), 1 if soften_all else 0,
                                         _ptr(hi), _ptr(lo))
        return hi, lo

    def phi_at(self, x, y, z):
        return self.lib().pto_phi_at(self.h, x, y, z)

    def phi_particle_feels(self, i):
        return self.lib().pto_phi_particle_feels(self.h, int(i))

    def measure_chi_b(self):
        return self.lib().pto_measure_chi_b(self.h)

    def cross_grain(self, p, d_pos, gr, a):
        p = np.ascontiguousarray(p, PARTICLE_DTYPE).reshape(1)
        gr = np.ascontiguousarray(gr, PARTICLE_DTYPE).reshape(1)
        d = np.ascontiguousarray(d_pos, np.float64)
        return bool(self.lib().pto_cross_grain(_ptr(p), _ptr(d), _ptr(gr), float(a)))

    def cross_grain_run(self, p, d_pos, gr):
        """The run's absorption test (sphere or spheroid)."""
        p = np.ascontiguousarray(p, PARTICLE_DTYPE).reshape(1)
        gr = np.ascontiguousarray(gr, PARTICLE_DTYPE).reshape(1)
        d = np.ascontiguousarray(d_pos, np.float64)
        return bool(self.lib().pto_cross_grain_run(self.h, _ptr(p), _ptr(d), _ptr(gr)))

    def grain_field(self, x, y, z):
        out = np.zeros(3)
        self.lib().pto_grain_field(self.h, x, y, z, _ptr(out))
        return out

    def grain_phi(self, x, y, z):
        return self.lib().pto_grain_phi(self.h, x, y, z)

    def step(self, compute_epe=False):
        rc = self.lib().pto_step(self.h, 1 if compute_epe else 0)
        if rc != 0:
            raise RuntimeError("oracle step failed: %d" % rc)

    def run_steps(self, n, compute_epe=False):
        rc = self.lib().pto_run_steps(self.h, int(n), 1 if compute_epe else 0)
        if rc != 0:
            raise RuntimeError("oracle run failed: %d" % rc)

    def last_step_stats(self):
        dq, de, na, nr, npush = C.c_int64(), C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint64()
        epe = np.zeros(3)
        self.lib().pto_last_step_stats(self.h, C.byref(dq), C.byref(de), C.byref(na), C.byref(nr),
                                       C.byref(npush), _ptr(epe))
        return dict(dq=dq.value, de=de.value, n_absorbed=na.value, n_reinjected=nr.value,
                    n_pushed=npush.value, epe=epe)

    def variant_stats(self):
        """Charges the Poisson ion collection added, and particles found in
        the wall moving inwards (OUT_BOUNCE), in the last step."""
        a, b = C.c_uint32(), C.c_uint32()
        self.lib().pto_last_step_variant_stats(self.h, C.byref(a), C.byref(b))
        return dict(n_pois=a.value, n_wall=b.value)

    def set_ion_temp(self, Ti):
        self.lib().pto_set_ion_temp(self.h, float(Ti))

    def ion_temp(self):
        return self.lib().pto_ion_temp(self.h)

    def poisson(self, lam):
        return self.lib().pto_poisson(self.h, float(lam))

    def tree_dipoles(self):
        mx = 9 * self.N + 16
        out = np.zeros((mx, 3))
        n = self.lib().pto_tree_dipoles(self.h, mx, _ptr(out))
        if n < 0:
            raise RuntimeError("tree dump overflow")
        return out[:n]

    def sample_reinject(self, n, species):
        out = np.zeros(int(n), PARTICLE_DTYPE)
        self.lib().pto_sample_reinject(self.h, int(n), int(species), _ptr(out))
        return out


def philox4x32(ctr, key):
    """Philox4x32-10 block (test helper)."""
    L = Oracle.lib()
    c = np.ascontiguousarray(ctr, np.uint32)
    k = np.ascontiguousarray(key, np.uint32)
    out = np.zeros(4, np.uint32)
    L.pto_philox4x32(_ptr(c), _ptr(k), _ptr(out))
    return out
