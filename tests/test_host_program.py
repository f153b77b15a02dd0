"""The C host program (pot_b200/host/potgpu.c): pot.c's command line,
its state files and output files.  CPU tests cover argument handling and
the state-file reader (``-R`` exits before any device is touched); GPU
tests run the program and check what it writes."""
import os
import struct
import subprocess

import numpy as np
import pytest

from oracle.oracle import PARTICLE_DTYPE

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "pot_b200", "potgpu")

SMALL_FLAGS = ["-N", "8193", "-r", "1000", "-m", "7.08046e-10", "-a", "1.41609e-08", "-s", "1.41609e-09",
               "-d", "3.37727e-15", "-E", "11600", "-I", "11600", "-x", "0", "-e", "0"]


@pytest.fixture(scope="module")
def potgpu():
    from pot_b200 import build
    try:
        return build.build_host()
    except FileNotFoundError as e:  # no nvcc: use what exists
        if os.path.exists(BIN):
            return BIN
        pytest.skip(str(e))


def run(args, cwd=None, timeout=600):
    return subprocess.run([BIN] + args, capture_output=True, text=True, cwd=cwd, timeout=timeout)


def test_list_settings_and_defaults(potgpu):
    p = run(["-l"])
    assert p.returncode == 0
    # pot.c:199-217 defaults
    assert "-N 150001 -r 1000 -d 1e-12 -m 4e-07 -s 2e-08 -E 220 -I 220 -x 0 -a 2.5e-06 -e 5e-07" in p.stdout
    p = run(["-l", "--prolate"])
    # pot-spheroid.c defaults (radius 654 px, 4e-10 m softening, 11600 K, no settling, A = 5)
    assert "-r 654" in p.stdout and "-s 4e-10" in p.stdout and "-E 11600" in p.stdout and "-A 5" in p.stdout
    p = run(["-l"] + SMALL_FLAGS + ["-i", "40"])
    assert "-N 8193" in p.stdout and "-i 40" in p.stdout


@pytest.mark.parametrize("args,msg", [(["-a", "-1"], "Grain radius must be positive."),
                                      (["-d", "0"], "Time step must be positive."),
                                      (["-i", "0"], "Number of time steps to run for must be a valid nonzero integer."),
                                      (["-N", "x"], "Number of particles must be a valid nonzero integer."),
                                      (["-A", "3"], "Aspect ratio is not a parameter for a sphere."),
                                      (["--prolate", "-A", "0.5"], "Prolate aspect ratio must be greater than 1."),
                                      (["-a", "1e-3", "-r", "10", "-m", "1e-5"], "Grain radius")])
def test_rejects_bad_settings(potgpu, args, msg):
    p = run(args)
    assert p.returncode != 0
    assert msg in p.stderr


def test_usage_on_unknown_flag(potgpu):
    p = run(["-Q"])
    assert p.returncode != 0 and "Usage:" in p.stderr


def _state_file(path, parts, fmt="C", workers=1, q=-37, m=1.67e-12, t=1234, tae=99, chi=-2.5):
    with open(path, "wb") as f:
        if fmt == "C":
            f.write(("C %u %i %g %lu %g %g %g %u %g\n" % (workers, q, m, t, 1e-20, 2e-20, 3e-20, tae, chi)).encode())
        elif fmt == "B":
            f.write(("B %u %i %lu %g %g %g %u\n" % (workers, q, t, 1e-20, 2e-20, 3e-20, tae)).encode())
        else:
            f.write(("%u %i %lu %g %g %g\n" % (workers, q, t, 1e-20, 2e-20, 3e-20)).encode())
        for w in range(workers):
            f.write(struct.pack("<21I", *([0] * 5 + list(range(w, w + 16)))))
        f.write(parts.tobytes())


@pytest.mark.parametrize("fmt,workers", [("C", 1), ("C", 3), ("B", 2), ("A", 1)])
def test_read_out_state_file(potgpu, tmp_path, fmt, workers):
    """-R prints the state file's particles as pot.c:4948-4961 does, for the
    reference's three state formats and any worker count."""
    rng = np.random.default_rng(3)
    P = np.zeros(7, PARTICLE_DTYPE)
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        P[k] = rng.normal(size=7)
    P["species"] = [0, 1, 1, 1, 2, 2, 2]
    path = tmp_path / "state"
    _state_file(path, P, fmt=fmt, workers=workers)
    p = run(["-N", "7", "-r", "1000", "-R", str(path)])
    assert p.returncode == 0, p.stderr
    lines = p.stdout.strip().splitlines()
    assert lines[0] == "NO S X Y Z VX VY VZ"
    assert len(lines) == 8
    for i, line in enumerate(lines[1:]):
        f = line.split()
        assert int(f[0]) == i and f[1] == '"%s"' % "die"[P["species"][i]]
        assert np.allclose([float(v) for v in f[2:]], [P[k][i] for k in ("x", "y", "z", "vx", "vy", "vz")],
                           rtol=1e-5)


def test_truncated_state_file_fails(potgpu, tmp_path):
    P = np.zeros(7, PARTICLE_DTYPE)
    path = tmp_path / "state"
    _state_file(path, P[:3])
    p = run(["-N", "7", "-R", str(path)])
    assert p.returncode != 0 and "failed to read particle states" in p.stderr


@pytest.mark.gpu
def test_run_writes_reference_outputs_and_resumes(potgpu, tmp_path):
    """A 240-step run writes pot-run-descrip.txt, pot-run-init-info.txt,
    pot-macroscopic.dat (header + a row per record step: every step up to
    200, then every 200th while t dt <= 2 settle, pot.c:4364-4369) and a
    format C state file; -g resumes from it with the same seed."""
    out = tmp_path / "output"
    out.mkdir()
    state = tmp_path / "state.dat"
    args = SMALL_FLAGS + ["-i", "240", "--seed", "5", "--output-dir", str(out), "-f", str(state)]
    p = run(args)
    assert p.returncode == 0, p.stderr
    descrip = (out / "pot-run-descrip.txt").read_text()
    assert "total particle count:          8193" in descrip and "Debye length (m):" in descrip
    assert "containment:          reinjection (SCEPTIC-style)" in descrip
    macro = (out / "pot-macroscopic.dat").read_text().splitlines()
    assert macro[0].split()[0] == "TIME" and len(macro[0].split()) == 35
    rows = [r.split() for r in macro[1:]]
    assert len(rows) == 201  # steps 1..200 and the last step (240), not a record step
    assert all(len(r) == 35 for r in rows)
    times = [float(r[0]) for r in rows]
    assert times == sorted(times)
    assert abs(times[-1] - 240 * 3.37727e-15) < 1e-20
    tote = [int(r[34]) for r in rows]
    assert tote == sorted(tote)
    assert all(r[2] != "NA" and r[4] != "NA" for r in rows[:200])  # potential energies on record steps
    with open(state, "rb") as f:
        head = f.readline().split()
        blob = f.read()
    assert head[0] == b"C" and int(head[1]) == 1 and int(head[4]) == 240
    assert len(blob) == 84 + 56 * 8193
    P = np.frombuffer(blob[84:], PARTICLE_DTYPE)
    assert P["species"][0] == 0 and (P["species"] == 1).sum() == 4096
    assert int(head[2]) == int(rows[-1][9])  # grain charge
    # resume for 10 more steps
    out2 = tmp_path / "output2"
    out2.mkdir()
    state2 = tmp_path / "state2.dat"
    p = run(SMALL_FLAGS + ["-i", "250", "-g", str(state), "--output-dir", str(out2), "-f", str(state2)])
    assert p.returncode == 0, p.stderr
    with open(state2, "rb") as f:
        head2 = f.readline().split()
    assert int(head2[4]) == 250
    rows2 = [r.split() for r in (out2 / "pot-macroscopic.dat").read_text().splitlines()[1:]]
    assert len(rows2) == 1 and abs(float(rows2[0][0]) - 250 * 3.37727e-15) < 1e-20
    # -g of a run that already reached -i stops at once
    p = run(SMALL_FLAGS + ["-i", "240", "-g", str(state), "--output-dir", str(out2)])
    assert p.returncode == 0 and "already run for 240 steps" in p.stdout


@pytest.mark.gpu
def test_spheroid_program_flags(potgpu, tmp_path):
    out = tmp_path / "o"
    out.mkdir()
    p = run(["--prolate", "-A", "3", "-N", "4097", "-r", "1000", "-m", "7.08046e-10", "-a", "3e-7", "-s",
             "1.41609e-09", "-d", "3.37727e-14", "-E", "11600", "-I", "1160", "-x", "30000", "-i", "30",
             "--seed", "2", "--bz", "0.5", "--output-dir", str(out)])
    assert p.returncode == 0, p.stderr
    d = (out / "pot-run-descrip.txt").read_text()
    assert "Grain shape:          prolate spheroid" in d and "aspect ratio:                  3" in d
    assert "ion/electron mass ratio: 1836.15" in d
    rows = (out / "pot-macroscopic.dat").read_text().splitlines()[1:]
    assert len(rows) == 30


def test_variant_switches_listed(potgpu):
    p = run(["-l", "--dipoles", "--bounce", "0.9", "--integrator", "euler-richardson", "--pois-ions"])
    assert p.returncode == 0
    assert "--dipoles --bounce 0.9 --integrator euler-richardson --pois-ions" in p.stdout
    p = run(["--integrator", "leapfrog"])
    assert p.returncode != 0
    p = run(["--bounce", "-1"])
    assert p.returncode != 0 and "restitution" in p.stderr


@pytest.mark.gpu
def test_variant_program_run(potgpu, tmp_path):
    """A run with every variant of pot.c's switches (plain form, since the
    dipole moments are plain-form): the description names them and the
    summary rows are written."""
    out = tmp_path / "v"
    out.mkdir()
    p = run(SMALL_FLAGS + ["-i", "12", "--seed", "3", "--form", "plain", "--dipoles", "--bounce", "0.95",
                           "--integrator", "verlet", "--pois-ions", "--output-dir", str(out)])
    assert p.returncode == 0, p.stderr
    d = (out / "pot-run-descrip.txt").read_text()
    assert "multipole expansion:  dipole" in d and "numerical integrator: velocity Verlet" in d
    assert "pos. Pois. collec'n:  yes" in d and "containment:          bouncing (c.o.e. 0.95)" in d
    rows = (out / "pot-macroscopic.dat").read_text().splitlines()[1:]
    assert len(rows) == 12


def _reference_state(path, steps=5, seed=1):
    """The reference itself (oracle/_ref, SCEPTIC) runs the small plasma
    `steps` steps and writes its format C state file (pot.c:3816-3901)."""
    from oracle.oracle import RefLib, RunParams
    from common import SMALL
    ref = RefLib("sceptic", build=False)
    ref.setup(RunParams(**SMALL), seed=seed)
    ref.set_grain(q=-40)
    ref.run_steps(steps)
    ref.write_state(str(path))
    return ref


def _parse_state_c(path, N):
    """Header fields, PRNG blocks and particles of a one-worker format C file."""
    raw = open(path, "rb").read()
    nl = raw.index(b"\n")
    head = raw[:nl].split()
    assert head[0] == b"C" and int(head[1]) == 1
    parts = np.frombuffer(raw[nl + 1 + 84:], PARTICLE_DTYPE)
    assert len(parts) == N
    return dict(q=int(head[2]), m=float(head[3]), t_steps=int(head[4]), tot_absor_e=int(head[8]),
                chi_b=float(head[9])), parts


def test_read_out_reference_state_file(potgpu, tmp_path):
    """-R reads a state file the reference program itself wrote."""
    path = tmp_path / "ref_state"
    ref = _reference_state(path)
    P = ref.particles()
    p = run(SMALL_FLAGS + ["-R", str(path)])
    assert p.returncode == 0, p.stderr
    lines = p.stdout.strip().splitlines()
    assert lines[0] == "NO S X Y Z VX VY VZ" and len(lines) == 8193 + 1
    for i in (0, 1, 4096, 4097, 8192):
        f = lines[1 + i].split()
        assert int(f[0]) == i and f[1] == '"%s"' % "die"[P["species"][i]]
        assert np.allclose([float(v) for v in f[2:]], [P[k][i] for k in ("x", "y", "z", "vx", "vy", "vz")],
                           rtol=1e-5)


@pytest.mark.gpu
def test_state_files_and_phi_exchange_with_reference(potgpu, tmp_path):
    """The reference writes a state file after 30 steps; potgpu -g resumes
    from it (plain form, theta 0.5) and writes pot-phi.dat for that state
    (--phi-start), which agrees row by row with the reference's own
    write_phi_data_to_file (pot.c:3001-3042) over the same particles; after
    one step potgpu -f writes its state, which the reference's
    read_sim_state_from_file (pot.c:3904-4019) reads back: the particles
    it holds are the file's, bit for bit."""
    a = tmp_path / "ref_state"
    ref = _reference_state(a, steps=30)
    ref.build_tree()
    ref_phi = tmp_path / "ref_phi.dat"
    ref.write_phi(str(ref_phi), 30)
    out = tmp_path / "out"
    out.mkdir()
    b = tmp_path / "gpu_state"
    p = run(SMALL_FLAGS + ["--oap", "0.5", "--form", "plain", "-g", str(a), "-i", "31", "--phi-start",
                           "--output-dir", str(out), "-f", str(b)])
    assert p.returncode == 0, p.stderr
    rows_g = (out / "pot-phi.dat").read_text().splitlines()
    rows_r = ref_phi.read_text().splitlines()
    assert len(rows_r) == 50 * 4 * 11 and rows_g[:len(rows_r)] and len(rows_g) >= len(rows_r)
    for lg, lr in zip(rows_g, rows_r):
        fg, fr = lg.split(), lr.split()
        assert fg[:4] == fr[:4]
        assert abs(float(fg[4]) - float(fr[4])) <= 2e-5 * abs(float(fr[4])) + 1e-12
    head, parts = _parse_state_c(b, 8193)
    assert head["t_steps"] == 31
    ref.read_state(str(b))
    g = ref.grain()
    assert g["t_steps"] == 31 and g["q"] == head["q"] and g["tot_absor_e"] == head["tot_absor_e"]
    assert ref.particles().tobytes() == parts.tobytes()
