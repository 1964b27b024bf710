"""f3r_dot_noalloc: the dot product for callers that cannot allocate device
memory (its reduction scratch is a fixed array inside the library), checked
through the C ABI against f3r_dot on two calls in a row.

This file is collected last on purpose (tests/test_zz_*): if it fails, a run
that stops at the first failure has already run every other test."""
import ctypes as C

import numpy as np
import pytest
import torch

import f3r_b200 as F
from f3r_b200 import _capi

pytestmark = pytest.mark.gpu

# same tolerances as the f3r_dot test in test_gpu_spmv.py, relative to |x|.|y|
TOL = {torch.float64: 1e-12, torch.float32: 1e-5, torch.float16: 1e-5}
DT = {torch.float64: F.F64, torch.float32: F.F32, torch.float16: F.F16}


def test_dot_noalloc_matches_f3r_dot():
    lib = F.lib()
    ctx = F.Context(0)
    stream = torch.cuda.current_stream().cuda_stream
    gen = torch.Generator(device="cuda").manual_seed(7)
    for call in range(2):  # two calls in a row share the static scratch
        for dt in (torch.float64, torch.float32, torch.float16):
            n = 3_000_001 + call
            x = torch.randn(n, device="cuda", dtype=torch.float64, generator=gen).to(dt)
            y = torch.randn(n, device="cuda", dtype=torch.float64, generator=gen).to(dt)
            torch.cuda.synchronize()  # ctx.dot runs on the context's own stream
            want = ctx.dot(x, y)
            out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
            _capi.check(lib.f3r_dot_noalloc(DT[dt], n, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                                            C.c_void_p(out.data_ptr()), C.c_void_p(stream)))
            torch.cuda.synchronize()
            got = float(out.item())
            scale = float(torch.dot(x.double().abs(), y.double().abs()).item())
            assert abs(got - want) <= TOL[dt] * scale + 1e-300, (call, dt, got, want)
    ctx.close()


def test_dot_noalloc_rejects_oversize_and_bad_args():
    lib = F.lib()
    x = torch.zeros(8, dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    too_big = 8192 * 4096 + 1   # rejected before any memory is touched
    st = lib.f3r_dot_noalloc(F.F64, too_big, C.c_void_p(x.data_ptr()), C.c_void_p(x.data_ptr()),
                             C.c_void_p(out.data_ptr()), None)
    assert st == 1 and b"static scratch maximum" in lib.f3r_last_error_string()
    assert lib.f3r_dot_noalloc(F.F64, 4, None, None, C.c_void_p(out.data_ptr()), None) == 1
    # empty input: the result is 0
    _capi.check(lib.f3r_dot_noalloc(F.F64, 0, None, None, C.c_void_p(out.data_ptr()), None))
    torch.cuda.synchronize()
    assert out.item() == 0.0
