"""The C++ adapter (include/f3r_b200.hpp) drives a solve from a
reference-style C++ driver, linked against libf3r_b200.so."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cpp_driver(tmp_path):
    exe = str(tmp_path / "adapter_demo")
    libdir = os.path.join(ROOT, "f3r_b200")
    r = subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "cpp", "adapter_demo.cpp"), "-L", libdir, "-lf3r_b200",
                        f"-Wl,-rpath,{libdir}", "-o", exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([exe, "20"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    fields = out.stdout.split()
    assert fields[0] == "solved" and fields[1] == "1"
    iters, calls = int(fields[3]), int(fields[5])
    assert calls == iters + 1  # cond(0, |r0|) then once per outer step
