"""A compiled host program (tests/c_host/pictor_main.c, built here with gcc
against libpictor_b200.so and include/pictor_b200.h) that makes the calls of
the reference's main loop (src/MAIN.F90:42-284) in its order through the C
ABI: the drop-in as a Fortran host would use it, from a compiled language.
Its result, with the exact-order current, equals the CPU restatement's
steps bit for bit."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "c_host", "pictor_main.c")


def _build(tmp):
    from pictor_b200 import _capi

    lib = _capi.library_path()
    if not os.path.exists(lib):
        pytest.skip("libpictor_b200.so not built")
    gcc = shutil.which("gcc")
    if not gcc:
        pytest.skip("no gcc")
    exe = os.path.join(tmp, "pictor_main")
    cmd = [gcc, "-O2", "-std=c11", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), SRC,
           "-L", os.path.dirname(lib), "-lpictor_b200", f"-Wl,-rpath,{os.path.dirname(lib)}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return exe


def test_c_host_builds_and_links(tmp_path):
    """The host program compiles against the header without warnings and
    links against the library (no GPU needed)."""
    exe = _build(str(tmp_path))
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 64 and "usage" in r.stderr


@pytest.mark.gpu
def test_c_host_main_loop_equals_oracle(tmp_path):
    """25 steps of a 48 x 40 Weibel run (output every 7 steps, reorder
    every 10) by the compiled host; the final particles and fields equal 25
    oracle steps bit for bit."""
    exe = _build(str(tmp_path))
    nx, ny, steps, period = 48, 40, 25, 10
    qi = 0.00158203125
    g = O.make_grid(2, nx, ny, c=0.45, qi=qi)
    p = O.load_weibel(2, nx, ny, epc=8, drift=0.5, temp=0.005, seed=21)
    v = p.view()
    fin, fout = os.path.join(str(tmp_path), "in.bin"), os.path.join(str(tmp_path), "out.bin")
    with open(fin, "wb") as f:
        np.array([p.used], dtype=np.int64).tofile(f)
        for k in ("q", "x", "y", "z", "u", "v", "w"):
            v[k].astype(np.float64).tofile(f)
        v["flv"].astype(np.int32).tofile(f)
    r = subprocess.run([exe, "2", str(nx), str(ny), "1", "0.45", repr(qi), str(steps), str(period), "7", "1", fin,
                        fout], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    o = O.Oracle(g, p.copy())
    for t in range(1, steps + 1):
        o.step(t, period)
    with open(fout, "rb") as f:
        n = int(np.fromfile(f, dtype=np.int64, count=1)[0])
        got = {k: np.fromfile(f, dtype=np.float64, count=n) for k in ("q", "x", "y", "z", "u", "v", "w")}
        got["flv"] = np.fromfile(f, dtype=np.int32, count=n)
        nf = (nx + 5) * (ny + 5)
        fields = {k: np.fromfile(f, dtype=np.float64, count=nf) for k in ("Ex", "Ey", "Ez", "Bx", "By", "Bz")}
    assert n == o.p.used
    ov = o.p.view()
    for k in ("q", "x", "y", "z", "u", "v", "w", "flv"):
        assert np.array_equal(got[k], ov[k]), k
    for k, a in fields.items():
        assert np.array_equal(a, getattr(o.f, k).ravel(order="F")), k
