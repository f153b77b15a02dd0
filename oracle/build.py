"""Build recipe for the CPU oracle (test infrastructure only).

Two things are built here, both with gcc, both outside the GPU product path:

1. ``oracle/libpotoracle.so`` -- the project's own C restatement of the
   reference's per-step particle loop (``oracle/pot_oracle.c``).  Needs only
   gcc; it is rebuilt on demand on any machine (including a GPU box, from the
   committed source).

2. ``oracle/_ref/libpotref_<variant>.so`` -- the *reference itself*, compiled
   from the sources where they lie under the reference tree.  The reference
   selects its physics with unconditional ``#define`` lines (pot.c:25-196), so
   one file has to be patched: a copy of ``pot.c`` with those switches set is
   written to ``oracle/_ref/src_<variant>/pot.c`` (an output, git-ignored,
   never committed).  ``prng.c``, ``prng.h``, ``coord.c`` and ``coord.h`` are
   used unmodified from the reference tree.  The single-rank ``mpi.h`` stand-in
   in ``oracle/mpi_stub`` replaces MPI, which is not installed.

   Variants:
     ``sphere``   SPHERICAL on, DISABLE_GRAIN/DEBUG_LANGMUIR off, default
                  (non flux-weighted) reinjection, Boris, monopole cells;
     ``sceptic``  as ``sphere`` plus SCEPTIC_REINJECTION (the flux-weighted
                  drifting-Maxwellian reinjection, pot.c:496-652);
     ``prolate``, ``prolate_sceptic``, ``oblate``, ``oblate_sceptic``
                  the spheroidal-grain program pot-spheroid.c the same way
                  (its CR line ends stripped, its GLFW/GLU includes and
                  ``#define GL`` taken out -- no graphics stack is needed or
                  used -- PROLATE or OBLATE selected, SCEPTIC_REINJECTION on
                  or off); the aspect ratio A is set at run time.
   Feature suffixes switch on the reference's other variants, on either
   program: ``_dip`` DIPOLES, ``_bounce`` OUT_BOUNCE 0.95, ``_pois``
   POIS_POS_COLLECTION, ``_verlet`` BORIS off (velocity Verlet), ``_er``
   BORIS off and EULER_RICHARDSON on -- e.g. ``sceptic_dip``.
   In all, OAP and EXTERNAL_B_{X,Y,Z} become run-time globals
   (``pot_ref_oap``, ``pot_ref_b{x,y,z}``) so one library serves every
   opening angle and field; C evaluates ``OAP * OAP * dist2`` identically for
   a literal and for a variable holding the same double.

Usage: ``python oracle/build.py [--ref-root PATH] [--force]``.  The reference
checkout is ``$POT_REFERENCE_ROOT`` if set, else ``--ref-root``, else a
directory named ``reference`` beside this repository's own directory.
"""
from __future__ import annotations

import argparse
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_OUT = os.path.join(HERE, "_ref")
# The reference checkout: $POT_REFERENCE_ROOT, else --ref-root, else a
# directory named "reference" beside this repository.
DEFAULT_REF_ROOT = os.environ.get("POT_REFERENCE_ROOT") or \
    os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")

VARIANTS = ("sphere", "sceptic")
SPHEROID_VARIANTS = ("prolate", "prolate_sceptic", "oblate", "oblate_sceptic")
FEATURES = ("dip", "bounce", "pois", "verlet", "er")
FEATURE_VARIANTS = tuple("sceptic_" + f for f in FEATURES)


def split_variant(variant: str):
    """(program variant, feature list): 'sceptic_dip' -> ('sceptic', ['dip'])."""
    parts = variant.split("_")
    feats = []
    while parts and parts[-1] in FEATURES:
        feats.insert(0, parts.pop())
    return "_".join(parts), feats


def _patch_features(t: str, feats, sub1) -> str:
    """Switch on the commented-out variant defines (pot.c:99-133, 165-173;
    pot-spheroid.c:97-180 has the same lines)."""
    for f in feats:
        if f == "dip":
            t = sub1(r"^(/\*\n#define DIPOLES\n\*/)$", r"\1\n#define DIPOLES", t)
        elif f == "bounce":
            t = sub1(r"^(/\*\n#define OUT_BOUNCE 0\.95\n\*/)$", r"\1\n#define OUT_BOUNCE 0.95", t)
        elif f == "pois":
            t = sub1(r"^(/\*\n#define POIS_POS_COLLECTION\n\*/)$", r"\1\n#define POIS_POS_COLLECTION", t)
        elif f in ("verlet", "er"):
            t = sub1(r"^#define BORIS\s*$", "/* BORIS switched off by the oracle recipe */", t)
            if f == "er":
                t = sub1(r"^(/\*\n#define EULER_RICHARDSON\n\*/)$", r"\1\n#define EULER_RICHARDSON", t)
    return t

CFLAGS = ["-O2", "-std=c99", "-fPIC", "-shared", "-Wall", "-Wno-unused-function",
          "-Wno-unused-variable", "-Wno-unused-but-set-variable", "-Wno-format",
          "-Wno-unused-result", "-Wno-maybe-uninitialized"]


def _run(cmd):
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError("command failed: %s\n%s%s" % (" ".join(cmd), proc.stdout, proc.stderr))
    return proc


def oracle_lib_path() -> str:
    return os.path.join(HERE, "libpotoracle.so")


def ref_lib_path(variant: str) -> str:
    return os.path.join(REF_OUT, "libpotref_%s.so" % variant)


def _stale(target: str, sources) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources if os.path.exists(s))


def build_oracle(force: bool = False) -> str:
    """Compile the C restatement into oracle/libpotoracle.so."""
    src = os.path.join(HERE, "pot_oracle.c")
    hdr = os.path.join(HERE, "pot_oracle.h")
    out = oracle_lib_path()
    if force or _stale(out, [src, hdr, __file__]):
        tmp = out + ".tmp%d" % os.getpid()
        _run(["gcc"] + CFLAGS + ["-I", HERE, src, "-o", tmp, "-lm"])
        os.replace(tmp, out)
    return out


def _patch_pot_c(text: str, variant: str) -> str:
    """Return pot.c with the hot-path switches set for ``variant``."""
    def sub1(pattern, repl, s):
        s2, n = re.subn(pattern, repl, s, count=1, flags=re.M)
        if n != 1:
            raise RuntimeError("patch pattern not found: %r" % pattern)
        return s2

    t = text.replace("\r\n", "\n")
    t = sub1(r"^#define DISABLE_GRAIN\s*$", "/* DISABLE_GRAIN switched off by the oracle recipe */", t)
    t = sub1(r"^#define DEBUG_LANGMUIR 0\.1\s*$", "/* DEBUG_LANGMUIR switched off by the oracle recipe */", t)
    t = sub1(r"^#define OAP 0\.8\s*$", "#define OAP pot_ref_oap", t)
    t = sub1(r"^#define EXTERNAL_B_X 0\.0\s*$", "#define EXTERNAL_B_X pot_ref_bx", t)
    t = sub1(r"^#define EXTERNAL_B_Y 0\.0\s*$", "#define EXTERNAL_B_Y pot_ref_by", t)
    t = sub1(r"^#define EXTERNAL_B_Z 0\.0\s*$", "#define EXTERNAL_B_Z pot_ref_bz", t)
    # SPHERICAL sits commented out (pot.c:109-111); define it right after.
    t = sub1(r"^(/\*\n#define SPHERICAL\n\*/)$", r"\1\n#define SPHERICAL", t)
    base, feats = split_variant(variant)
    if base == "sceptic":
        t = sub1(r"^(/\*\n#define SCEPTIC_REINJECTION\n\*/)$", r"\1\n#define SCEPTIC_REINJECTION", t)
    t = _patch_features(t, feats, sub1)
    header = ("/* Generated by oracle/build.py from the reference pot.c; variant %s. */\n"
              "extern double pot_ref_oap, pot_ref_bx, pot_ref_by, pot_ref_bz;\n" % variant)
    return header + t


def _patch_spheroid_c(text: str, variant: str) -> str:
    """Return pot-spheroid.c with the hot-path switches set for ``variant``."""
    def sub1(pattern, repl, s):
        s2, n = re.subn(pattern, repl, s, count=1, flags=re.M)
        if n != 1:
            raise RuntimeError("patch pattern not found: %r" % pattern)
        return s2

    t = text.replace("\r\n", "\n").replace("\r", "")
    t = sub1(r"^#define GLFW_INCLUDE_GLU\s*$", "/* graphics include removed by the oracle recipe */", t)
    t = sub1(r"^#include <GLFW/glfw.h>\s*$", "", t)
    t = sub1(r"^#include <GL/glu.h>\s*$", "", t)
    t = sub1(r"^#define GL\s*$", "/* GL switched off by the oracle recipe */", t)
    t = sub1(r"^#define OAP 1\.0\s*$", "#define OAP pot_ref_oap", t)
    t = sub1(r"^#define EXTERNAL_B_X 0\.0\s*$", "#define EXTERNAL_B_X pot_ref_bx", t)
    t = sub1(r"^#define EXTERNAL_B_Y 0\.0\s*$", "#define EXTERNAL_B_Y pot_ref_by", t)
    t = sub1(r"^#define EXTERNAL_B_Z 0\.0\s*$", "#define EXTERNAL_B_Z pot_ref_bz", t)
    base, feats = split_variant(variant)
    if not base.endswith("_sceptic"):
        t = sub1(r"^#define SCEPTIC_REINJECTION\s*$", "/* SCEPTIC_REINJECTION switched off by the oracle recipe */", t)
    t = _patch_features(t, feats, sub1)
    if variant.startswith("oblate"):
        t = sub1(r"^#define PROLATE\s*$", "/* PROLATE switched off by the oracle recipe */\n#define OBLATE", t)
    header = ("/* Generated by oracle/build.py from the reference pot-spheroid.c; variant %s. */\n"
              "extern double pot_ref_oap, pot_ref_bx, pot_ref_by, pot_ref_bz;\n" % variant)
    return header + t


def build_ref(ref_root: str = DEFAULT_REF_ROOT, force: bool = False, variants=VARIANTS):
    """Compile the reference (patched copy of pot.c + its own prng.c) per variant.

    Returns a dict variant -> library path.  Raises FileNotFoundError when the
    reference tree is absent (it never travels to a GPU box)."""
    prng_c = os.path.join(ref_root, "prng.c")
    if not (os.path.exists(os.path.join(ref_root, "pot.c")) and os.path.exists(prng_c)):
        raise FileNotFoundError("reference sources not found under %s" % ref_root)
    os.makedirs(REF_OUT, exist_ok=True)
    harness = os.path.join(HERE, "ref_harness.c")
    stub = os.path.join(HERE, "mpi_stub", "mpi.h")
    out = {}
    for v in variants:
        srcdir = os.path.join(REF_OUT, "src_" + v)
        os.makedirs(srcdir, exist_ok=True)
        patched = os.path.join(srcdir, "pot.c")
        lib = ref_lib_path(v)
        spheroid = split_variant(v)[0] in SPHEROID_VARIANTS
        pot_c = os.path.join(ref_root, "pot-spheroid.c" if spheroid else "pot.c")
        deps = [pot_c, prng_c, harness, stub, __file__]
        if force or _stale(lib, deps) or not os.path.exists(patched):
            with open(pot_c, "r", encoding="latin-1") as f:
                text = f.read()
            with open(patched, "w", encoding="latin-1") as f:
                f.write(_patch_spheroid_c(text, v) if spheroid else _patch_pot_c(text, v))
            tmp = lib + ".tmp%d" % os.getpid()
            # -iquote order: the patched pot.c is found before the reference's
            # own; prng.h / coord.c / coord.h come from the reference tree.
            _run(["gcc"] + CFLAGS + ["-iquote", srcdir, "-iquote", ref_root,
                                     "-I", os.path.join(HERE, "mpi_stub"),
                                     "-Dmain=pot_ref_main", harness, prng_c, "-o", tmp, "-lm"])
            os.replace(tmp, lib)
        out[v] = lib
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--ref-root", default=DEFAULT_REF_ROOT)
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args(argv)
    print(build_oracle(force=args.force))
    try:
        for v, p in build_ref(args.ref_root, force=args.force).items():
            print(v, p)
    except FileNotFoundError as e:
        print("reference not built:", e, file=sys.stderr)
    return 0


if __name__ == "__main__":
    sys.exit(main())
