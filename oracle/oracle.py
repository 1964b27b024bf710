"""TEST INFRASTRUCTURE -- ctypes bindings to the CPU oracle.

Two libraries are bound here, both built by ``oracle/Makefile``:

* ``liboracle.so``: the plain-C restatement of the reference F3R algorithm
  (``oracle/f3r_oracle.c``).
* ``_ref/libf3r_ref*.so``: the reference's own C++ templates compiled in place
  with a C shim (``oracle/ref_lib.cpp``, ``oracle/ref_gen.cpp``).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
and reference legs import this module.  The product package ``f3r_b200``
never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

DT_F64, DT_F32, DT_F16 = 0, 1, 2
ARITH_PRODUCT, ARITH_REF = 0, 1
PRECOND_SDAINV, PRECOND_ILU0_BJ, PRECOND_ILU0_JACOBI, PRECOND_ILU0_BAJ = 0, 1, 2, 3
FORM_LOWER, FORM_LOWER_D, FORM_D_UPPER = 0, 1, 2

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_u16p = np.ctypeslib.ndpointer(np.uint16, flags="C_CONTIGUOUS")


# The read-only reference checkout the _ref targets compile from (the Makefile's REF).
REF_TREE = os.environ.get("F3R_REF", "/root/reference")


def build() -> None:
    """Compile liboracle.so (and oracle/_ref when the reference tree exists)."""
    targets = ["liboracle.so"]
    if os.path.isdir(os.path.join(REF_TREE, "library")):
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", HERE, f"REF={REF_TREE}"] + targets, check=True)


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        _lib = C.CDLL(path)
        L = _lib
        L.or_stencil27.restype = C.c_int64
        L.or_stencil27.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, _i32p, _i32p, _f64p]
        L.or_scaling.argtypes = [C.c_int32, _i32p, _i32p, _f64p]
        L.or_sell_nnz.restype = C.c_int64
        L.or_sell_nnz.argtypes = [C.c_int32, _i32p, C.c_int32]
        L.or_csr_to_sell.argtypes = [C.c_int32, _i32p, _i32p, _f64p, C.c_int32, _i32p, _i32p, _f64p]
        L.or_sell_operate_f64.argtypes = [C.c_int32, C.c_int32, _i32p, _i32p, _f64p, _f64p, _f64p]
        L.or_sell_sigma_perm.argtypes = [C.c_int32, _i32p, C.c_int32, _i32p]
        L.or_spmv.argtypes = [C.c_int32, _i32p, _i32p, _f64p, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                              C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int]
        L.or_mat_from.restype = C.c_void_p
        L.or_mat_from.argtypes = [C.c_int32, C.c_int32, C.c_int32, _i32p, _i32p, _f64p]
        L.or_mat_free.argtypes = [C.c_void_p]
        L.or_mat_n.argtypes = [C.c_void_p]
        L.or_mat_nnz.argtypes = [C.c_void_p]
        L.or_mat_copy_out.argtypes = [C.c_void_p, _i32p, _i32p, _f64p]
        L.or_sdainv.argtypes = [C.c_void_p, C.c_double, C.c_double, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]
        L.or_ilu0_bj.restype = C.c_int
        L.or_ilu0_bj.argtypes = [C.c_void_p, C.c_int32, C.c_double, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]
        L.or_trsv_lower.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int]
        L.or_jacobi_trsv.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int32, C.c_double, C.c_int, _u16p, _u16p]
        L.or_trsv_upper.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int]
        L.or_dot_f32.restype = C.c_float
        L.or_dot_f32.argtypes = [C.c_int32, _f32p, _f32p]
        L.or_dot_f64.restype = C.c_double
        L.or_dot_f64.argtypes = [C.c_int32, _f64p, _f64p]
        L.or_f3r_solve.restype = C.c_int
        L.or_f3r_solve.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, _f64p, _f64p, C.c_void_p, _f64p,
                                   C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                   C.POINTER(C.c_double), C.POINTER(C.c_int64)]
        L.or_richardson_apply.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                          _f32p, _f32p, _f32p, _f32p]
        L.or_inner_level_apply.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                           _f32p, _f32p]
        L.or_f64_to_f16.argtypes = [C.c_int64, _f64p, _u16p]
    return _lib


class F3RParams(C.Structure):
    _fields_ = [("m1", C.c_int32), ("restarts", C.c_int32), ("m2", C.c_int32), ("m3", C.c_int32),
                ("m4", C.c_int32), ("c", C.c_int32), ("precond", C.c_int32), ("arith", C.c_int32),
                ("half_scale_log2", C.c_int32), ("tol", C.c_double), ("static_weight", C.c_double),
                ("trsv_iters", C.c_int32), ("pad_", C.c_int32), ("trsv_omega", C.c_double),
                ("sstep", C.c_int32), ("half_m", C.c_int32)]


def params(m1=100, restarts=20, m2=8, m3=4, m4=2, c=64, precond=PRECOND_SDAINV, arith=ARITH_PRODUCT,
           half_scale_log2=0, tol=1e-10, static_weight=0.0, trsv_iters=2, trsv_omega=1.0, sstep=0,
           half_m=0) -> F3RParams:
    return F3RParams(m1, restarts, m2, m3, m4, c, precond, arith, half_scale_log2, tol, static_weight, trsv_iters,
                     0, trsv_omega, sstep, half_m)


class Mat:
    """An oracle-owned CSR matrix (fp64 values)."""

    def __init__(self, ptr):
        self.ptr = C.c_void_p(ptr) if not isinstance(ptr, C.c_void_p) else ptr

    @classmethod
    def from_csr(cls, rptr, idx, val, ncols=None):
        n = len(rptr) - 1
        return cls(lib().or_mat_from(n, ncols if ncols else n, len(idx), np.ascontiguousarray(rptr, np.int32),
                                     np.ascontiguousarray(idx, np.int32), np.ascontiguousarray(val, np.float64)))

    def csr(self):
        L = lib()
        n, nnz = L.or_mat_n(self.ptr), L.or_mat_nnz(self.ptr)
        r = np.zeros(n + 1, np.int32)
        i = np.zeros(max(nnz, 1), np.int32)
        v = np.zeros(max(nnz, 1), np.float64)
        L.or_mat_copy_out(self.ptr, r, i, v)
        return r, i[:nnz], v[:nnz]

    def __del__(self):
        if getattr(self, "ptr", None) is not None and _lib is not None:
            _lib.or_mat_free(self.ptr)
            self.ptr = None


def stencil27(nx, ny, nz, variant=0, beta=0.5):
    n = nx * ny * nz
    rptr = np.zeros(n + 1, np.int32)
    idx = np.zeros(27 * n, np.int32)
    val = np.zeros(27 * n, np.float64)
    nnz = lib().or_stencil27(nx, ny, nz, variant, beta, rptr, idx, val)
    return rptr, idx[:nnz].copy(), val[:nnz].copy()


def scaling(rptr, idx, val):
    val = np.array(val, np.float64)
    lib().or_scaling(len(rptr) - 1, rptr, idx, val)
    return val


def csr_to_sell(rptr, idx, val, w=32):
    n = len(rptr) - 1
    nnz = lib().or_sell_nnz(n, rptr, w)
    ns = (n + w - 1) // w
    sptr = np.zeros(ns + 1, np.int32)
    sidx = np.zeros(max(nnz, 1), np.int32)
    sval = np.zeros(max(nnz, 1), np.float64)
    lib().or_csr_to_sell(n, rptr, idx, np.ascontiguousarray(val, np.float64), w, sptr, sidx, sval)
    return sptr, sidx[:nnz], sval[:nnz]


def sell_sigma_perm(rptr, sigma):
    perm = np.zeros(len(rptr) - 1, np.int32)
    lib().or_sell_sigma_perm(len(rptr) - 1, rptr, sigma, perm)
    return perm


_NP = {DT_F64: np.float64, DT_F32: np.float32, DT_F16: np.float16}


def spmv(rptr, idx, val, x, val_t, y_t, acc_t, b=None, ref_mul_add=False):
    """y = A x (or b - A x); x and b are numpy arrays whose dtype selects the type."""
    n = len(rptr) - 1
    x = np.ascontiguousarray(x)
    x_t = {np.dtype(np.float64): DT_F64, np.dtype(np.float32): DT_F32, np.dtype(np.float16): DT_F16}[x.dtype]
    y = np.zeros(n, _NP[y_t])
    bp, b_t = None, 0
    if b is not None:
        b = np.ascontiguousarray(b)
        b_t = {np.dtype(np.float64): DT_F64, np.dtype(np.float32): DT_F32, np.dtype(np.float16): DT_F16}[b.dtype]
        bp = b.ctypes.data
    lib().or_spmv(n, rptr, idx, np.ascontiguousarray(val, np.float64), val_t, x.ctypes.data, x_t,
                  y.ctypes.data, y_t, acc_t, int(ref_mul_add), bp, b_t)
    return y


def sdainv(A: Mat, tol=0.1, acc=1.0):
    z, w = C.c_void_p(), C.c_void_p()
    lib().or_sdainv(A.ptr, tol, acc, C.byref(z), C.byref(w))
    return Mat(z), Mat(w)


def ilu0_bj(A: Mat, blocks=112, acc=1.0):
    l, u = C.c_void_p(), C.c_void_p()
    if lib().or_ilu0_bj(A.ptr, blocks, acc, C.byref(l), C.byref(u)) != 0:
        raise ValueError(f"block count {blocks} is invalid for this matrix size")
    return Mat(l), Mat(u)


def trsv(M: Mat, upper: bool, x: np.ndarray, prod_fma=False):
    x = np.ascontiguousarray(x, np.float16)
    out = np.zeros_like(x)
    f = lib().or_trsv_upper if upper else lib().or_trsv_lower
    f(M.ptr, DT_F16, x.ctypes.data, DT_F16, out.ctypes.data, int(prod_fma))
    return out


def jacobi_trsv(M: Mat, form: int, x: np.ndarray, iters: int, omega: float = 1.0, baj: bool = False,
                arith: int = ARITH_PRODUCT) -> np.ndarray:
    """Jacobi (trsv/jacobi.hpp) or BAJ (trsv/baj.hpp, one-thread row order)
    triangular solve of fp16 vectors; form FORM_LOWER / FORM_LOWER_D /
    FORM_D_UPPER."""
    xin = np.ascontiguousarray(x, np.float16).view(np.uint16)
    out = np.zeros(len(xin), np.uint16)
    lib().or_jacobi_trsv(M.ptr, form, int(baj), iters, omega, arith, xin, out)
    return out.view(np.float16)


def f3r_solve(A: Mat, P1: Mat, P2: Mat, b, p: F3RParams, x0=None, hist_cap=4096):
    n = len(b)
    x = np.zeros(n) if x0 is None else np.array(x0, np.float64)
    hist = np.zeros(hist_cap)
    nh, it, r_calls = C.c_int32(), C.c_int32(), C.c_int64()
    res = C.c_double()
    solved = lib().or_f3r_solve(A.ptr, P1.ptr, P2.ptr, np.ascontiguousarray(b, np.float64), x, C.byref(p),
                                hist, hist_cap, C.byref(nh), C.byref(it), C.byref(res), C.byref(r_calls))
    return dict(x=x, solved=bool(solved), iters=it.value, impl_res=res.value,
                hist=hist[:min(nh.value, hist_cap)].copy(), r_calls=r_calls.value)


def richardson_apply(A: Mat, P1: Mat, P2: Mat, p: F3RParams, cnt0: int, sums, omes, x):
    sums = np.array(sums, np.float32)
    omes = np.array(omes, np.float32)
    out = np.zeros(len(x), np.float32)
    lib().or_richardson_apply(A.ptr, P1.ptr, P2.ptr, C.byref(p), cnt0, sums, omes,
                              np.ascontiguousarray(x, np.float32), out)
    return out, sums, omes


def inner_level_apply(A: Mat, P1: Mat, P2: Mat, p: F3RParams, level: int, x):
    out = np.zeros(len(x), np.float32)
    lib().or_inner_level_apply(A.ptr, P1.ptr, P2.ptr, C.byref(p), level, np.ascontiguousarray(x, np.float32), out)
    return out


def f64_to_f16_bits(a):
    a = np.ascontiguousarray(a, np.float64)
    out = np.zeros(len(a), np.uint16)
    lib().or_f64_to_f16(len(a), a, out)
    return out


# --------------------------------------------------------------------------
# the reference compiled in place (oracle/_ref)
# --------------------------------------------------------------------------
def _cpu_has(flag: str) -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return flag in line.split()
    except OSError:
        pass
    return False


class Ref:
    """Bindings to oracle/_ref/libf3r_ref*.so.

    variant "golden": deterministic flags (no FMA contraction), used for the
    golden vectors.  variant "fast": the reference build's speed flags for this
    CPU (AVX-512 FP16 when present), used for the timed CPU baseline.
    """

    def __init__(self, variant="golden"):
        if variant == "golden":
            name = "libf3r_ref.so"
        else:
            name = "libf3r_ref_spr.so" if _cpu_has("avx512_fp16") else "libf3r_ref_fast.so"
        self.name = name
        path = os.path.join(REF_DIR, name)
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref` where the reference tree exists")
        L = self.L = C.CDLL(path)
        L.ref_gen27.restype = C.c_int64
        L.ref_gen27.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f64p]
        L.ref_gen27_halfspace.restype = C.c_int64
        L.ref_gen27_halfspace.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, _i32p, _i32p, _f64p]
        L.ref_scaling.argtypes = [C.c_int32, C.c_int32, _i32p, _i32p, _f64p]
        L.ref_sell32_build.restype = C.c_void_p
        L.ref_sell32_build.argtypes = [C.c_int32, C.c_int32, _i32p, _i32p, _f64p]
        L.ref_sell32_size.restype = C.c_int64
        L.ref_sell32_size.argtypes = [C.c_void_p]
        L.ref_sell32_nslice.restype = C.c_int32
        L.ref_sell32_nslice.argtypes = [C.c_void_p]
        L.ref_sell32_copy.argtypes = [C.c_void_p, _i32p, _i32p, _f64p]
        L.ref_sell32_free.argtypes = [C.c_void_p]
        L.ref_sell32_operate.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        L.ref_sell32_residual.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_sdainv.restype = C.c_void_p
        L.ref_sdainv.argtypes = [C.c_int32, C.c_int32, _i32p, _i32p, _f64p, C.c_double, C.c_double]
        L.ref_ilu0_bj.restype = C.c_void_p
        L.ref_ilu0_bj.argtypes = [C.c_int32, C.c_int32, _i32p, _i32p, _f64p, C.c_int, C.c_double]
        L.ref_pair_nnz.restype = C.c_int32
        L.ref_pair_nnz.argtypes = [C.c_void_p, C.c_int]
        L.ref_pair_copy.argtypes = [C.c_void_p, C.c_int, _i32p, _i32p, _f64p]
        L.ref_bj_solve_f16.argtypes = [C.c_void_p, C.c_int, C.c_int, _u16p, _u16p]
        L.ref_pair_free.argtypes = [C.c_void_p]
        L.ref_jacobi_trsv_f16.argtypes = [C.c_int32, C.c_int32, _i32p, _i32p, _f64p, C.c_int, C.c_int, C.c_int,
                                          C.c_double, _u16p, _u16p]
        L.ref_gen27_save.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_char_p]
        L.ref_mm_read_system.restype = C.c_void_p
        L.ref_mm_read_system.argtypes = [C.c_char_p]
        L.ref_mm_dims.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
        L.ref_mm_copy.argtypes = [C.c_void_p, _i32p, _i32p, _f64p, _f64p]
        L.ref_mm_free.argtypes = [C.c_void_p]
        L.ref_f3r_solve.restype = C.c_int
        L.ref_f3r_solve.argtypes = [C.c_int, C.c_int32, C.c_int32, _i32p, _i32p, _f64p, _f64p, _f64p,
                                    C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                    C.c_double, C.c_int, _f64p, _f64p, C.c_int, C.c_int, C.c_double]

    def gen27(self, nx, ny, nz, variant=0, beta=0.5):
        n = nx * ny * nz
        rptr = np.zeros(n + 1, np.int32)
        idx = np.zeros(27 * n, np.int32)
        val = np.zeros(27 * n, np.float64)
        if variant == 2:
            nnz = self.L.ref_gen27_halfspace(nx, ny, nz, beta, rptr, idx, val)
        else:
            nnz = self.L.ref_gen27(variant, nx, ny, nz, rptr, idx, val)
        return rptr, idx[:nnz].copy(), val[:nnz].copy()

    def scaling(self, rptr, idx, val):
        val = np.array(val, np.float64)
        self.L.ref_scaling(len(rptr) - 1, len(idx), rptr, idx, val)
        return val

    def sell32(self, rptr, idx, val):
        h = self.L.ref_sell32_build(len(rptr) - 1, len(idx), rptr, idx, np.ascontiguousarray(val, np.float64))
        try:
            nnz, ns = self.L.ref_sell32_size(h), self.L.ref_sell32_nslice(h)
            sptr = np.zeros(ns + 1, np.int32)
            sidx = np.zeros(max(nnz, 1), np.int32)
            sval = np.zeros(max(nnz, 1), np.float64)
            self.L.ref_sell32_copy(h, sptr, sidx, sval)
        finally:
            self.L.ref_sell32_free(h)
        return sptr, sidx[:nnz], sval[:nnz]

    def sell32_operate(self, rptr, idx, val, kind, x):
        """kind 0: f64*f64->f64, 1: f32*f32->f32, 2: f16*f32->f32, 3: f16*f16->f16"""
        out_dt = {0: np.float64, 1: np.float32, 2: np.float32, 3: np.float16}[kind]
        in_dt = {0: np.float64, 1: np.float32, 2: np.float32, 3: np.float16}[kind]
        x = np.ascontiguousarray(x, in_dt)
        y = np.zeros(len(rptr) - 1, out_dt)
        h = self.L.ref_sell32_build(len(rptr) - 1, len(idx), rptr, idx, np.ascontiguousarray(val, np.float64))
        try:
            self.L.ref_sell32_operate(h, kind, x.ctypes.data, y.ctypes.data)
        finally:
            self.L.ref_sell32_free(h)
        return y

    def sell32_residual(self, rptr, idx, val, kind, b, x):
        dt = np.float64 if kind == 0 else np.float16
        b = np.ascontiguousarray(b, dt)
        x = np.ascontiguousarray(x, dt)
        r = np.zeros(len(rptr) - 1, dt)
        h = self.L.ref_sell32_build(len(rptr) - 1, len(idx), rptr, idx, np.ascontiguousarray(val, np.float64))
        try:
            self.L.ref_sell32_residual(h, kind, b.ctypes.data, x.ctypes.data, r.ctypes.data)
        finally:
            self.L.ref_sell32_free(h)
        return r

    def _pair(self, h):
        out = []
        n = None
        for which in (0, 1):
            nnz = self.L.ref_pair_nnz(h, which)
            out.append(nnz)
        return out

    def _copy_pair(self, h, n):
        mats = []
        for which in (0, 1):
            nnz = self.L.ref_pair_nnz(h, which)
            r = np.zeros(n + 1, np.int32)
            i = np.zeros(max(nnz, 1), np.int32)
            v = np.zeros(max(nnz, 1), np.float64)
            self.L.ref_pair_copy(h, which, r, i, v)
            mats.append((r, i[:nnz], v[:nnz]))
        return mats

    def jacobi_trsv(self, rptr, idx, val, form, x16, iters, omega=1.0, baj=False, csr=False):
        """trsv::{l,ld,du}::Jacobi / BAJ <SELL<32, _Float16>> (or <CSR<_Float16>>) solve of fp16 x"""
        n = len(rptr) - 1
        xin = np.ascontiguousarray(x16, np.float16).view(np.uint16)
        out = np.zeros(n, np.uint16)
        self.L.ref_jacobi_trsv_f16(n, len(idx), np.ascontiguousarray(rptr, np.int32), np.ascontiguousarray(idx, np.int32),
                                   np.ascontiguousarray(val, np.float64), form, int(baj) + 2 * int(csr), iters, omega, xin,
                                   out)
        return out.view(np.float16)

    def gen27_save(self, variant, nx, ny, nz, path):
        """the reference generator's own .mtx writer (variant 0 hpcg, 1 hpgmp)"""
        self.L.ref_gen27_save(variant, nx, ny, nz, os.fsencode(path))

    def mm_read_system(self, path):
        """(rptr, idx, val, b): io::mm::read_system + io::CSR with the drivers' init"""
        h = self.L.ref_mm_read_system(os.fsencode(path))
        try:
            n, nnz = C.c_int32(), C.c_int32()
            self.L.ref_mm_dims(h, C.byref(n), C.byref(nnz))
            r = np.zeros(n.value + 1, np.int32)
            i = np.zeros(max(nnz.value, 1), np.int32)
            v = np.zeros(max(nnz.value, 1), np.float64)
            b = np.zeros(max(n.value, 1), np.float64)
            self.L.ref_mm_copy(h, r, i, v, b)
            return r, i[:nnz.value], v[:nnz.value], b[:n.value]
        finally:
            self.L.ref_mm_free(h)

    def sdainv(self, rptr, idx, val, tol=0.1, acc=1.0):
        """returns (Z, Wt) as CSR tuples"""
        n = len(rptr) - 1
        h = self.L.ref_sdainv(n, len(idx), rptr, idx, np.ascontiguousarray(val, np.float64), tol, acc)
        try:
            return tuple(self._copy_pair(h, n))
        finally:
            self.L.ref_pair_free(h)

    def ilu0_bj(self, rptr, idx, val, blocks=112, acc=1.0, solve_in=None):
        """returns (L, U) as CSR tuples, and the fp16 BJ solves of solve_in if given"""
        n = len(rptr) - 1
        h = self.L.ref_ilu0_bj(n, len(idx), rptr, idx, np.ascontiguousarray(val, np.float64), blocks, acc)
        try:
            mats = tuple(self._copy_pair(h, n))
            if solve_in is None:
                return mats
            xin = np.ascontiguousarray(solve_in, np.float16).view(np.uint16)
            lo = np.zeros(n, np.uint16)
            up = np.zeros(n, np.uint16)
            self.L.ref_bj_solve_f16(h, blocks, 0, xin, lo)
            self.L.ref_bj_solve_f16(h, blocks, 1, xin, up)
            return mats, lo.view(np.float16), up.view(np.float16)
        finally:
            self.L.ref_pair_free(h)

    def f3r_solve(self, config, rptr, idx, val, b, m2=8, m3=4, m4=2, c=64, restarts=20, tol=1e-10,
                  acc=1.0, sdainv_tol=0.1, blocks=112, hist_cap=4096, stop_after=0, weight=1.0):
        n = len(rptr) - 1
        x = np.zeros(n)
        out = np.zeros(5)
        hist = np.zeros(hist_cap)
        nh = self.L.ref_f3r_solve(config, n, len(idx), rptr, idx, np.ascontiguousarray(val, np.float64),
                                  np.ascontiguousarray(b, np.float64), x, m2, m3, m4, c, restarts, tol, acc,
                                  sdainv_tol, blocks, out, hist, hist_cap, stop_after, weight)
        return dict(x=x, time_s=out[0], iters=int(out[1]), impl_res=out[2], expl_res=out[3],
                    solved=bool(out[4]), hist=hist[:min(nh, hist_cap)].copy())

    def f3r_solve_depth_half(self, variant, rptr, idx, val, b, restarts=20, tol=1e-10, acc=1.0, blocks=112,
                             hist_cap=4096):
        """the depth ablations with an fp16-vector innermost FGMRES level over
        block-Jacobi ILU(0) (work/src/depth.cpp): variant 0 F4, 1 F3H, 2 F2H"""
        if getattr(self, "D", None) is None:
            path = os.path.join(REF_DIR, "libf3r_ref_depth.so")
            if not os.path.exists(path):
                raise FileNotFoundError(f"{path} missing: run `make -C oracle ref` where the reference tree exists")
            self.D = C.CDLL(path)
            self.D.ref_f3r_solve_depth_half.restype = C.c_int
            self.D.ref_f3r_solve_depth_half.argtypes = [C.c_int, C.c_int32, C.c_int32, _i32p, _i32p, _f64p, _f64p,
                                                        _f64p, C.c_int, C.c_double, C.c_double, C.c_int, _f64p, _f64p,
                                                        C.c_int]
        n = len(rptr) - 1
        x = np.zeros(n)
        out = np.zeros(5)
        hist = np.zeros(hist_cap)
        nh = self.D.ref_f3r_solve_depth_half(variant, n, len(idx), np.ascontiguousarray(rptr, np.int32),
                                             np.ascontiguousarray(idx, np.int32), np.ascontiguousarray(val, np.float64),
                                             np.ascontiguousarray(b, np.float64), x, restarts, tol, acc, blocks, out,
                                             hist, hist_cap)
        return dict(x=x, time_s=out[0], iters=int(out[1]), impl_res=out[2], expl_res=out[3],
                    solved=bool(out[4]), hist=hist[:min(nh, hist_cap)].copy())

    def f3r_solve_sstep(self, mask, rptr, idx, val, b, m2=8, m3=4, m4=2, c=64, restarts=20, tol=1e-10, acc=1.0,
                        sdainv_tol=0.1, hist_cap=4096):
        """the SDAINV + SELL-32 F3R solve with sFGMRES (gmres2.hpp:137-221) at
        level 2 (mask bit 0) and / or level 3 (mask bit 1)"""
        if getattr(self, "S", None) is None:
            path = os.path.join(REF_DIR, "libf3r_ref_sstep.so")
            if not os.path.exists(path):
                raise FileNotFoundError(f"{path} missing: run `make -C oracle ref` where the reference tree exists")
            self.S = C.CDLL(path)
            self.S.ref_f3r_solve_sstep.restype = C.c_int
            self.S.ref_f3r_solve_sstep.argtypes = [C.c_int, C.c_int32, C.c_int32, _i32p, _i32p, _f64p, _f64p, _f64p,
                                                   C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                                   C.c_double, C.c_double, _f64p, _f64p, C.c_int]
        n = len(rptr) - 1
        x = np.zeros(n)
        out = np.zeros(5)
        hist = np.zeros(hist_cap)
        nh = self.S.ref_f3r_solve_sstep(mask, n, len(idx), np.ascontiguousarray(rptr, np.int32),
                                        np.ascontiguousarray(idx, np.int32), np.ascontiguousarray(val, np.float64),
                                        np.ascontiguousarray(b, np.float64), x, m2, m3, m4, c, restarts, tol, acc,
                                        sdainv_tol, out, hist, hist_cap)
        return dict(x=x, time_s=out[0], iters=int(out[1]), impl_res=out[2], expl_res=out[3],
                    solved=bool(out[4]), hist=hist[:min(nh, hist_cap)].copy())
