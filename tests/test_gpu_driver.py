"""The command-line driver (bin/f3r-run) end to end on the GPU: Matrix Market
in, the reference drivers' CSV line out (work/src/f3r-gpu.cpp:44-104,
267-285; static.cpp; depth.cpp), checked against the same solve through the
Python API."""
import os
import subprocess

import numpy as np
import pytest

import f3r_b200 as F

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "f3r_b200", "bin", "f3r-run")


@pytest.fixture(scope="module")
def suite_dirs(tmp_path_factory):
    """the reference suites' layout: matrices in ../matrix/ seen from the run directory"""
    top = tmp_path_factory.mktemp("suite")
    os.makedirs(top / "matrix")
    os.makedirs(top / "work")
    F.stencil27(16, 16, 16, 1, 0.5).write_mm(str(top / "matrix" / "hpgmp_4_4_4.mtx"))
    return top


def run(args, cwd):
    r = subprocess.run([EXE] + args, capture_output=True, text=True, cwd=cwd, timeout=300)
    assert r.returncode == 0, r.stderr
    return r.stdout.strip().splitlines()


def python_solve(path, **kw):
    A, b, _ = F.read_system(path)
    A.scale()
    S = F.Solver(F.Context(0), A, rel_tol=1e-8, **kw)
    return S.solve(b, np.zeros(len(b)))


def test_f3r_line(suite_dirs):
    lines = run(["--header", "hpgmp_4_4_4.mtx", "1.0", "2", "8", "4", "2", "8", "3"], cwd=suite_dirs / "work")
    assert lines[0] == F.CSV_HEADER
    f = lines[1].split(",")
    assert f[:9] == ["hpgmp_4_4_4", "F3R", "__half", "8", "4", "2", "8", "SDAINV", "1.0"]
    t, it, impl, expl = float(f[9]), int(f[10]), float(f[11]), float(f[12])
    r = python_solve(str(suite_dirs / "matrix" / "hpgmp_4_4_4.mtx"), m2=8, m3=4, m4=2, c=8)
    assert it == r.res_iter * 8 * 4 * 2
    assert impl < 1e-8 and expl < 1e-7
    assert 0 < t < 60


def test_static_and_depth_lines(suite_dirs):
    cwd = suite_dirs / "work"
    f = run(["--method", "F3R-Static", "--blocks", "16", "hpgmp_4_4_4.mtx", "1.0", "1", "8", "4", "2", "8", "3",
             "1.2"], cwd)[0].split(",")
    assert f[:9] == ["hpgmp_4_4_4", "F3R-Static", "_Float16", "8", "4", "2", "1.2", "BJILU0", "1.0"]
    r = python_solve(str(suite_dirs / "matrix" / "hpgmp_4_4_4.mtx"), m2=8, m3=4, m4=2, static_weight=1.2,
                     precond=F.PRECOND_ILU0_BJ, ilu_blocks=16, max_restarts=3)
    assert int(f[10]) == r.res_iter * 64 and float(f[12]) < 1e-7
    # the CPU driver's CSR storage: the same sums, so the same line but for the time
    fc = run(["--method", "F3R-Static", "--blocks", "16", "--format", "CSR", "hpgmp_4_4_4.mtx", "1.0", "1", "8", "4",
              "2", "8", "3", "1.2"], cwd)[0].split(",")
    assert fc[:9] == f[:9] and fc[10:] == f[10:]
    for method in ("F3", "F2", "F4", "F3H", "F2H"):
        f = run(["--method", method, "--blocks", "16", "hpgmp_4_4_4.mtx", "1.0", "1", "8", "4", "2", "8", "3"],
                cwd)[0].split(",")
        assert f[1] == method and float(f[12]) < 1e-7
        assert int(f[10]) % 64 == 0  # outer iterations * 64, as depth.cpp's test(..., 64)
