"""The reference driver's own solve call site against this library.

oracle/_ref/kmm_drop_in compiles the body of the driver's test() lambda
(work/src/f3r-gpu.cpp:76-104, extracted from the reference tree at build time,
not copied) around kmm::Solver<host>(f3r::kmm::F3R<host>(data, params))
(include/f3r_b200_kmm.hpp).  The lambda's `solver.solve(b, x, cond)` runs
unchanged; its printed line (time, outer iterations, implicit and explicit
relative residual, as the driver prints them) is checked against the
reference's own solve of the same system (tests/golden/solves.npz)."""
import os
import subprocess

import numpy as np
import pytest

from test_oracle_pins import golden_system

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "kmm_drop_in")


def write_system(path, r, i, v, b):
    with open(path, "wb") as f:
        np.array([len(r) - 1, len(i)], np.int32).tofile(f)
        np.asarray(r, np.int32).tofile(f)
        np.asarray(i, np.int32).tofile(f)
        np.asarray(v, np.float64).tofile(f)
        np.asarray(b, np.float64).tofile(f)


@pytest.mark.parametrize("name,sigma,precond,blocks", [("sdainv_hpgmp16", 256, 0, 16), ("sdainv_half16", 1, 0, 16),
                                                       ("bjilu_hpcg16", 1, 1, 16)])
def test_driver_call_site_unchanged(tmp_path, name, sigma, precond, blocks):
    if not os.path.exists(EXE):
        pytest.skip("oracle/_ref/kmm_drop_in is built where the reference tree is present")
    r, i, v, b, xs, sol = golden_system(name)
    sysf = str(tmp_path / "system.bin")
    write_system(sysf, r, i, v, b)
    out = subprocess.run([EXE, sysf, str(sigma), "8", str(precond), str(blocks)], capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    lines = out.stdout.strip().splitlines()
    t, iters, impl, expl = lines[0].split(",")
    ref_iters = int(sol[name + "_iters"])
    assert abs(int(iters) - ref_iters) <= 1, (iters, ref_iters)
    assert float(impl) < 1e-10 and float(expl) < 1e-10, (impl, expl)
    assert float(t) > 0
    # float right-hand side and solution through the same Solver<host>
    tag, rel = lines[1].split(",")
    assert tag == "float_solve" and float(rel) < 1e-5, lines[1]
