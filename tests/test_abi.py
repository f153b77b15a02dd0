"""C ABI: the library loads, exports every entry point include/pot_gpu.h
declares, and the records have the reference's layout.  No compute calls."""
import ctypes as C

import numpy as np

from oracle.oracle import PARTICLE_DTYPE as ORACLE_PARTICLE
from pot_b200 import gpu


def test_library_exports_header_symbols():
    L = gpu.load_library()
    names = gpu.header_symbols()
    assert len(names) >= 15
    for n in names:
        assert hasattr(L, n), n


def test_particle_record_is_the_reference_layout():
    # pot.c:295-303 on x86-64: six doubles, an enum, padding -> 56 bytes
    assert gpu.PARTICLE_DTYPE.itemsize == 56
    assert gpu.PARTICLE_DTYPE == ORACLE_PARTICLE
    assert [gpu.PARTICLE_DTYPE.fields[k][1] for k in ("x", "vz", "species")] == [0, 40, 48]


def test_struct_sizes():
    assert C.sizeof(gpu._RunCfg) == 8 + 4 + 4 + 8 * 9 + 24 + 8 + 24 + 8 + 4 + 4
    assert C.sizeof(gpu._Opts) == 40
    assert C.sizeof(gpu._Grain) == 88
    assert C.sizeof(gpu._Stats) == 88 + 24 + 8 + 16 + 8 + 8


def test_strerror_covers_every_status():
    L = gpu.load_library()
    for code, name in gpu.STATUS_NAMES.items():
        msg = L.pot_gpu_strerror(code).decode()
        assert msg and msg != "unknown status", (code, name)


def test_create_rejects_bad_arguments_before_touching_a_device():
    L = gpu.load_library()
    h = C.c_void_p()
    cfg = gpu.RunConfig(N=1, r=1000, dt=1e-15, mpp=1e-9, soft=1e-9, Te=1e4, Ti=1e4).to_c()
    opts = gpu._Opts()
    assert L.pot_gpu_create(C.byref(cfg), C.byref(opts), C.byref(h)) == -1  # N < 2
    for A in (1.0, -2.0, float("nan")):  # neither sphere (0), prolate (> 1) nor oblate (0, 1)
        cfg = gpu.RunConfig(N=100, r=1000, dt=1e-15, mpp=1e-9, soft=1e-9, Te=1e4, Ti=1e4, A=A).to_c()
        assert L.pot_gpu_create(C.byref(cfg), C.byref(opts), C.byref(h)) == -1
    opts.form = 0
    opts.leaf_size = 8  # plain form is leaf size 1
    cfg = gpu.RunConfig(N=100, r=1000, dt=1e-15, mpp=1e-9, soft=1e-9, Te=1e4, Ti=1e4).to_c()
    assert L.pot_gpu_create(C.byref(cfg), C.byref(opts), C.byref(h)) == -1


def test_no_cpu_fallback_without_device():
    """With no CUDA device the library refuses (POT_E_CUDA), it never
    computes on the host."""
    import torch
    if torch.cuda.is_available():
        return
    L = gpu.load_library()
    h = C.c_void_p()
    cfg = gpu.RunConfig(N=100, r=1000, dt=1e-15, mpp=1e-9, soft=1e-9, Te=1e4, Ti=1e4).to_c()
    opts = gpu._Opts()
    assert L.pot_gpu_create(C.byref(cfg), C.byref(opts), C.byref(h)) == -2


def test_python_mirror_matches_the_c_header(tmp_path):
    """Every field offset and record size of the ctypes mirror against the
    header as gcc lays it out."""
    import os
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        import pytest
        pytest.skip("no C compiler")
    mirrors = {"pot_run_cfg": gpu._RunCfg, "pot_gpu_opts": gpu._Opts, "pot_grain_state": gpu._Grain,
               "pot_step_stats": gpu._Stats, "pot_macro_sums": gpu._MacroSums, "pot_batch_opts": gpu._BatchOpts}
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "pot_gpu.h"', "int main(void) {"]
    for cname, cls in mirrors.items():
        lines.append('printf("%s %%zu\\n", sizeof(%s));' % (cname, cname))
        for f, _ in cls._fields_:
            lines.append('printf("%s.%s %%zu\\n", offsetof(%s, %s));' % (cname, f, cname, f))
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    subprocess.run([cc, "-I", inc, str(src), "-o", str(exe)], check=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                         check=True).stdout.splitlines())
    for cname, cls in mirrors.items():
        assert int(got[cname]) == C.sizeof(cls), cname
        for f, _ in cls._fields_:
            assert int(got["%s.%s" % (cname, f)]) == getattr(cls, f).offset, (cname, f)
