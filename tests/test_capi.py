"""CPU-side checks of the C ABI: every entry point declared in include/*.h is
exported by libf3r_b200.so, errors come back as status codes with messages
(never an exit), the parameter defaults are the reference drivers', and the
C++ adapter header compiles.  No GPU is needed (and none is touched)."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import f3r_b200 as F
from f3r_b200 import _capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")


def declared_functions():
    names = set()
    for h in os.listdir(INC):
        if not h.endswith(".h"):
            continue
        src = open(os.path.join(INC, h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b(f3r_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return names


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) >= 37
    lib = C.CDLL(_capi.LIB_PATH)
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding table covers the whole ABI
    assert names == set(_capi.SIGNATURES), names ^ set(_capi.SIGNATURES)


def test_params_default_match_drivers():
    p = F.Params()
    # work/src/f3r-gpu.cpp:264-265 (FGMRES(100), Restarted 20), suite-gpu.py:49 (8,4,2,64),
    # f3r-gpu.cpp:74 (tol 0.1), f3r-gpu.cpp:18 (eps 1e-8), f3r.cpp:57 (112 blocks)
    assert (p.m_outer, p.max_restarts, p.m2, p.m3, p.m4, p.c) == (100, 20, 8, 4, 2, 64)
    assert (p.sdainv_tol, p.acc, p.rel_tol, p.ilu_blocks, p.sell_c, p.sell_sigma) == (0.1, 1.0, 1e-8, 112, 32, 1)
    assert p.half_scale_log2 == 0 and p.use_graphs == 1 and p.sell_index16 == 0
    assert p.static_weight == 0.0 and (p.trsv_iters, p.trsv_omega) == (2, 1.0) and p.inner_sstep == 0
    assert p.sell_align == 0 and p.format == 0 and p.sell_autotune == 0
    # the ctypes mirror has the C struct's size
    assert C.sizeof(p) == 144


def test_struct_layouts_match_header(tmp_path):
    """every ctypes mirror has the C header's field offsets and size: a small
    C program built with the host compiler against include/f3r_b200.h prints
    offsetof / sizeof for each field the binding declares"""
    structs = {"f3r_csr": _capi.CSR, "f3r_params": _capi.Params, "f3r_result": _capi.Result,
               "f3r_sell_info": _capi.SellInfo, "f3r_tune_entry": _capi.TuneEntry}
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "f3r_b200.h"', "int main(void) {"]
    expect = []
    for cname, py in structs.items():
        lines.append(f'  printf("%zu\\n", sizeof({cname}));')
        expect.append(C.sizeof(py))
        for fname, _ in py._fields_:
            lines.append(f'  printf("%zu\\n", offsetof({cname}, {fname}));')
            expect.append(getattr(py, fname).offset)
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    assert got == expect
    # the newest field keeps its documented default
    assert F.Params().diag_load == 0


def test_errors_are_status_codes():
    # non-monotone rptr
    with pytest.raises(F.F3RError) as e:
        F.HostMatrix.from_csr(np.array([0, 3, 2], np.int32), np.array([0, 1, 0], np.int32), np.ones(3), 2)
    assert e.value.status == 1 and "rptr" in str(e.value)
    # column out of range
    with pytest.raises(F.F3RError):
        F.HostMatrix.from_csr(np.array([0, 1], np.int32), np.array([5], np.int32), np.ones(1))
    # unsorted row
    with pytest.raises(F.F3RError):
        F.HostMatrix.from_csr(np.array([0, 2], np.int32), np.array([1, 0], np.int32), np.ones(2), 2)
    with pytest.raises(F.F3RError):
        F.stencil27(0, 4, 4)
    # SDAINV / ILU need stored diagonals
    A = F.HostMatrix.from_csr(np.array([0, 1, 2], np.int32), np.array([1, 0], np.int32), np.ones(2))
    with pytest.raises(F.F3RError):
        A.sdainv()
    with pytest.raises(F.F3RError):
        A.ilu0_bj(1)
    assert _capi.lib().f3r_status_string(7) == b"device wait timed out"


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="checks the no-GPU path")
def test_no_device_is_reported_not_fallen_back():
    with pytest.raises(F.F3RError) as e:
        F.Context(0)
    assert e.value.status == 9


def test_host_helpers():
    A = F.stencil27(4, 5, 6, 2, 0.5)
    r, i, v = A.arrays()
    x = F.random_uniform(3, -1, 1, A.shape[0])
    assert np.all((x >= -1) & (x < 1)) and np.array_equal(x, F.random_uniform(3, -1, 1, A.shape[0]))
    dense = np.zeros(A.shape)
    for row in range(A.shape[0]):
        dense[row, i[r[row]:r[row + 1]]] = v[r[row]:r[row + 1]]
    assert np.allclose(A.spmv(x), dense @ x, rtol=0, atol=1e-12)
    D = F.diffusion7(6, 6, 6, 2.5, 2.0, 1)
    rd, idd, vd = D.arrays()
    # symmetric, positive diagonal, weakly diagonally dominant
    Dd = np.zeros(D.shape)
    for row in range(D.shape[0]):
        Dd[row, idd[rd[row]:rd[row + 1]]] = vd[rd[row]:rd[row + 1]]
    assert np.allclose(Dd, Dd.T) and np.all(np.diag(Dd) > 0)
    assert np.all(np.diag(Dd) >= np.abs(Dd).sum(1) - np.diag(Dd) - 1e-12)


def test_cpp_adapter_compiles():
    src = os.path.join(ROOT, "tests", "cpp", "adapter_demo.cpp")
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I", INC, src], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
