"""CULQCD-style C++ code (the reference's entry points, include/culqcd_b200.hpp)
compiled against libsun_b200.so gives the same lattice as the same call
sequence through the Python API, and writes a reference-format file the
oracle reads back."""
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_culqcd_program_matches_python_api(ctx, tmp_path):
    exe = str(tmp_path / "culqcd_demo")
    lib = os.path.join(ROOT, "sun_b200")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "culqcd_demo.cpp"), "-L" + lib, "-lsun_b200",
                    "-Wl,-rpath," + lib, "-o", exe], check=True)
    f_cpp = str(tmp_path / "cpp.bin")
    out = subprocess.run([exe, f_cpp], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    vals = {l.split()[0]: [float(v) for v in l.split()[1:]] for l in out.stdout.splitlines()
            if l.split() and l.split()[0] in ("plaquette", "polyakov", "wilson11", "wilson11_smeared")}

    from sun_b200 import (SOA12, HeatBath, OnePolyakovLoop, OverRelaxation, PlaquetteCUB, Reunitarize,
                          SaveBin_Gauge, gauge)
    g = gauge(ctx, N=3, dims=(4, 4, 4, 8), beta=6.0, atype=SOA12, evenodd=True, prec="f32", seed=1234)
    g.Init(hot=True)
    for _ in range(3):
        HeatBath(g).Run(1)
        for _ in range(4):
            OverRelaxation(g).Run(1)
    Reunitarize(g).Run()
    f_py = str(tmp_path / "py.bin")
    SaveBin_Gauge(g, f_py, True, True)
    assert open(f_cpp, "rb").read() == open(f_py, "rb").read()

    p = PlaquetteCUB(g).Run()
    assert abs(vals["plaquette"][0] - p.real) < 1e-6 and abs(vals["plaquette"][1] - p.imag) < 1e-6
    rc, U, grid, beta = O.load_bin(3, [4, 4, 4, 8], f_cpp, save_fp64=True, header_fp64=False)
    assert rc == 0 and grid == [4, 4, 4, 8]
    assert np.abs(O.plaquette(U, [4, 4, 4, 8]) - np.array(vals["plaquette"])).max() < 1e-6
    l = OnePolyakovLoop(g).Run()
    assert abs(vals["polyakov"][0] - l.real) < 1e-6
    w = O.wilson_loops(U, [4, 4, 4, 8], 2, 3)
    assert abs(vals["wilson11"][0] - w[1, 1, 0]) < 1e-6

    # the same smearing through the Python API on a normal-order SOA copy
    from sun_b200 import SOA, ApplyAPEinSpace, ApplyMultiHit, WilsonLoop
    bb = gauge(ctx, N=3, dims=(4, 4, 4, 8), beta=6.0, atype=SOA, evenodd=False, prec="f32", seed=1234)
    bb.Copy(g)
    ApplyAPEinSpace(bb, 0.2, 3, 10, 1e-10)
    dd = gauge(ctx, N=3, dims=(4, 4, 4, 8), beta=6.0, atype=SOA, evenodd=False, prec="f32", seed=1234)
    dd.Copy(bb)
    ApplyMultiHit(dd, bb, 1234, 5)
    ws = WilsonLoop(bb, 2, 3)
    # the C++ side returns the loop as _complex<float>: rounding of the result only
    assert abs(vals["wilson11_smeared"][0] - ws[1, 1].real) < 1e-6
    assert abs(vals["wilson11_smeared"][0] - vals["wilson11"][0]) > 1e-3
