"""f3r_b200 -- a B200-native (sm_100a) nested mixed-precision F3R solver.

Python view of the C ABI (include/f3r_b200.h), used by the tests and the
benchmark.  The compute path is the CUDA library libf3r_b200.so; there is no
CPU fallback: every object here calls into that library and raises if it is
missing or if no B200 is visible.

Names follow the reference's solver interface (umineko-sparse/models.hpp):
``Solver.solve(b, x, cond) -> solve_res_t``, ``Sell.operate(in, out)``,
``Sell.compute_residual(rhs, in, res)``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Callable, Optional

import numpy as np

from . import _capi
from ._capi import (F16, F32, F64, FORMAT_CSR, FORMAT_SELL, PRECOND_ILU0_BAJ, PRECOND_ILU0_BJ, PRECOND_ILU0_JACOBI,
                    PRECOND_ILU0_LEVEL, PRECOND_SDAINV, TRSV_BAJ, TRSV_D_UPPER, TRSV_JACOBI, TRSV_LOWER, TRSV_LOWER_D, F3RError, check, lib)

__all__ = ["HostMatrix", "Context", "Sell", "Solver", "Params", "solve_res_t", "F3RError", "F64", "F32", "F16",
           "FORMAT_SELL", "FORMAT_CSR", "PRECOND_ILU0_LEVEL",
           "PRECOND_SDAINV", "PRECOND_ILU0_BJ", "PRECOND_ILU0_JACOBI", "PRECOND_ILU0_BAJ", "Trsv", "TRSV_LOWER",
           "TRSV_LOWER_D", "TRSV_D_UPPER", "TRSV_JACOBI", "TRSV_BAJ", "stencil27", "diffusion7", "random_uniform", "host_spmv",
           "read_matrix", "read_system", "read_vector", "write_vector", "CSV_HEADER", "csv_row", "solve_batch"]

_NP2DT = {np.dtype(np.float64): F64, np.dtype(np.float32): F32, np.dtype(np.float16): F16}

# Live device objects, closed at interpreter exit in dependency order (solvers,
# matrices and triangular solves before the contexts they run on), before the
# CUDA runtime itself shuts down.
import atexit
import weakref

_LIVE = {k: weakref.WeakSet() for k in ("solver", "sell", "trsv", "learned", "context")}


@atexit.register
def _close_all():
    for kind in ("solver", "sell", "trsv", "learned", "context"):
        for obj in list(_LIVE[kind]):
            try:
                obj.close()
            except Exception:
                pass


class HostMatrix:
    """A library-owned host CSR matrix (f3r_host_matrix)."""

    def __init__(self, handle):
        self._h = C.c_void_p(handle) if not isinstance(handle, C.c_void_p) else handle

    @classmethod
    def from_csr(cls, rptr, idx, val, ncols=None) -> "HostMatrix":
        rptr = np.ascontiguousarray(rptr, np.int32)
        idx = np.ascontiguousarray(idx, np.int32)
        val = np.ascontiguousarray(val, np.float64)
        n = len(rptr) - 1
        v = _capi.CSR(n, ncols if ncols is not None else n, len(idx), rptr.ctypes.data_as(C.POINTER(C.c_int32)),
                      idx.ctypes.data_as(C.POINTER(C.c_int32)), val.ctypes.data_as(C.POINTER(C.c_double)))
        h = C.c_void_p()
        check(lib().f3r_host_matrix_from_csr(C.byref(v), C.byref(h)))
        return cls(h)

    def view(self) -> _capi.CSR:
        v = _capi.CSR()
        check(lib().f3r_host_matrix_view(self._h, C.byref(v)))
        return v

    @property
    def shape(self):
        v = self.view()
        return (v.nrows, v.ncols)

    @property
    def nnz(self) -> int:
        return self.view().nnz

    def arrays(self):
        """(rptr, idx, val) as numpy copies."""
        v = self.view()
        rptr = np.ctypeslib.as_array(v.rptr, (v.nrows + 1,)).copy()
        if v.nnz == 0:
            return rptr, np.zeros(0, np.int32), np.zeros(0)
        idx = np.ctypeslib.as_array(v.idx, (v.nnz,)).copy()
        val = np.ctypeslib.as_array(v.val, (v.nnz,)).copy()
        return rptr, idx, val

    def scale(self) -> "HostMatrix":
        """D^{-1/2} A D^{-1/2} in place (kmm::algorithm::scaling)."""
        check(lib().f3r_host_scaling(self._h))
        return self

    def spmv(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float64)
        y = np.zeros(self.shape[0])
        v = self.view()
        check(lib().f3r_host_spmv(C.byref(v), x.ctypes.data, y.ctypes.data))
        return y

    def sdainv(self, tol=0.1, acc=1.0):
        """(Z, W^T) with M r = Z (W^T r) (kmm::algorithm::sdainv)."""
        z, w = C.c_void_p(), C.c_void_p()
        v = self.view()
        check(lib().f3r_host_sdainv(C.byref(v), tol, acc, C.byref(z), C.byref(w)))
        return HostMatrix(z), HostMatrix(w)

    def ilu0_bj(self, blocks=112, acc=1.0):
        """(L, U) block-Jacobi ILU(0) factors."""
        l, u = C.c_void_p(), C.c_void_p()
        v = self.view()
        check(lib().f3r_host_ilu0_bj(C.byref(v), blocks, acc, C.byref(l), C.byref(u)))
        return HostMatrix(l), HostMatrix(u)

    def write_mm(self, path) -> None:
        """Matrix Market "coordinate real general" file, %.17g values."""
        v = self.view()
        check(lib().f3r_mm_write(_path(path), C.byref(v)))

    def __del__(self):
        if getattr(self, "_h", None) is not None and _capi is not None and _capi._lib is not None:
            _capi._lib.f3r_host_matrix_destroy(self._h)
            self._h = None


def stencil27(nx, ny, nz, variant=0, beta=0.5) -> HostMatrix:
    h = C.c_void_p()
    check(lib().f3r_problem_stencil27(nx, ny, nz, variant, beta, C.byref(h)))
    return HostMatrix(h)


def diffusion7(nx, ny, nz, sigma=2.5, corr_len=8.0, seed=0) -> HostMatrix:
    h = C.c_void_p()
    check(lib().f3r_problem_diffusion7(nx, ny, nz, sigma, corr_len, seed, C.byref(h)))
    return HostMatrix(h)


def random_uniform(seed: int, lo: float, hi: float, n: int) -> np.ndarray:
    out = np.zeros(n)
    check(lib().f3r_random_uniform(seed, lo, hi, n, out.ctypes.data))
    return out


def host_spmv(A: HostMatrix, x) -> np.ndarray:
    return A.spmv(x)


# ---- Matrix Market files and the drivers' CSV line (matrix/io.hpp, f3r-gpu.cpp)

def _path(p) -> bytes:
    import os
    return os.fsencode(p)


def read_matrix(path) -> HostMatrix:
    """A "matrix coordinate" file as CSR (io::mm::read_matrix + io::CSR)."""
    h = C.c_void_p()
    check(lib().f3r_mm_read(_path(path), C.byref(h)))
    return HostMatrix(h)


def read_vector(path, n: int) -> np.ndarray:
    """An n x 1 "matrix array real general" file."""
    out = np.zeros(n)
    check(lib().f3r_mm_read_vector(_path(path), n, out.ctypes.data))
    return out


def read_system(path):
    """(A, b, b_from_file) as io::mm::read_system with the drivers' init:
    b from "<stem>_b.mtx" if it exists, else U(0, 1) from mt19937_64(0)."""
    A = read_matrix(path)
    b = np.zeros(A.shape[0])
    ff = C.c_int32(0)
    check(lib().f3r_mm_read_rhs(_path(path), len(b), b.ctypes.data, C.byref(ff)))
    return A, b, bool(ff.value)


def write_vector(path, x) -> None:
    x = np.ascontiguousarray(x, np.float64)
    check(lib().f3r_mm_write_vector(_path(path), len(x), x.ctypes.data))


CSV_HEADER = "Problem,Method,Prec,M2,M3,M4,W,Precond,ACC,Time,Iter,ImplRes,ExplRes"


def csv_row(problem, method, prec, m2, m3, m4, w, precond, acc, time_s, iters, impl_res, expl_res) -> str:
    """One result line in the drivers' format (f3r-gpu.cpp:94-103, 267-272):
    Time, ImplRes and ExplRes as C's %e, Iter as an integer, the other
    fields as given (ACC as typed on the command line)."""
    return "%s,%s,%s,%d,%d,%d,%s,%s,%s,%e,%d,%e,%e" % (problem, method, prec, m2, m3, m4, w, precond, acc, time_s,
                                                        iters, impl_res, expl_res)


class Context:
    """One device and one CUDA stream (f3r_context)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib().f3r_context_create(device, C.byref(h)))
        self._h = h
        _LIVE["context"].add(self)
        self.device = device

    def set_stream(self, stream_ptr: Optional[int]) -> None:
        check(lib().f3r_context_set_stream(self._h, C.c_void_p(stream_ptr) if stream_ptr else None))

    def synchronize(self) -> None:
        check(lib().f3r_context_synchronize(self._h))

    def wait_probe(self, set_flag: bool, limit_ms: int) -> None:
        """The library's bounded device wait on a flag that is set or that
        nothing sets (f3r_context_wait_probe); raises F3RError (TIMEOUT) when
        the limit passes."""
        check(lib().f3r_context_wait_probe(self._h, 1 if set_flag else 0, limit_ms))

    def dot(self, x, y) -> float:
        """<x, y> of two device tensors (torch) of the same dtype."""
        dt = _torch_dt(x)
        out = C.c_double()
        check(lib().f3r_dot(self._h, dt, x.numel(), C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), C.byref(out)))
        return out.value

    def close(self):
        if getattr(self, "_h", None) is not None and _capi is not None and _capi._lib is not None:
            _capi._lib.f3r_context_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def _torch_dt(t):
    import torch
    return {torch.float64: F64, torch.float32: F32, torch.float16: F16}[t.dtype]


class Sell:
    """Device SELL-32-sigma matrix (f3r_sell) -- CoefficientMatrix::operate /
    compute_residual on device tensors."""

    def __init__(self, ctx: Context, A: HostMatrix, sigma: int = 1, dtypes=(F64, F32, F16), index16: bool = False,
                 aligned: bool = False, csr: bool = False, height: int = 32):
        """csr: keep the matrix in CSR (F3R_SELL_CSR) instead of SELL-32;
        height 64: 64-row offset-aligned slices (sigma 1)"""
        mask = ((_capi.SELL_INDEX16 if index16 else 0) | (_capi.SELL_ALIGNED if aligned else 0) |
                (_capi.SELL_CSR if csr else 0))
        for d in dtypes:
            mask |= 1 << d
        h = C.c_void_p()
        v = A.view()
        check(lib().f3r_sell_create(ctx._h, C.byref(v), height, sigma, mask, C.byref(h)))
        self._h = h
        _LIVE["sell"].add(self)
        self.ctx = ctx

    def info(self) -> _capi.SellInfo:
        i = _capi.SellInfo()
        check(lib().f3r_sell_info_get(self._h, C.byref(i)))
        return i

    def operate(self, x, y, val_t=None) -> None:
        """y = A x; val_t defaults to the vector type of x (fp16 for fp16 x)."""
        xt, yt = _torch_dt(x), _torch_dt(y)
        vt = xt if val_t is None else val_t
        check(lib().f3r_sell_operate(self._h, vt, xt, C.c_void_p(x.data_ptr()), yt, C.c_void_p(y.data_ptr())))

    def compute_residual(self, b, x, r, val_t=None) -> None:
        """r = b - A x."""
        bt, xt, rt = _torch_dt(b), _torch_dt(x), _torch_dt(r)
        vt = xt if val_t is None else val_t
        check(lib().f3r_sell_compute_residual(self._h, vt, bt, C.c_void_p(b.data_ptr()), xt,
                                              C.c_void_p(x.data_ptr()), rt, C.c_void_p(r.data_ptr())))

    def tune(self, val_t=F16, reps=20):
        """Times out = A x at every launch shape the library carries (fastest first)."""
        buf = (_capi.TuneEntry * 64)()
        cnt = C.c_int32()
        check(lib().f3r_sell_tune(self._h, val_t, reps, buf, 64, C.byref(cnt)))
        return [dict(warps=e.warps, stages=e.stages, kc=e.kc, index_bits=e.index_bits, default=bool(e.is_default),
                     us=e.microseconds, gbs=e.gbs_algorithmic) for e in buf[:cnt.value]]

    def close(self):
        if getattr(self, "_h", None) is not None and _capi is not None and _capi._lib is not None:
            _capi._lib.f3r_sell_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


class Trsv:
    """Jacobi-iteration triangular solve on the device (f3r_trsv):
    trsv::{l,ld,du}::Jacobi / BAJ <SELL<32, __half>> (trsv/jacobi.hpp,
    trsv/baj.hpp).  ``solve(in, out)`` takes fp16 device tensors."""

    def __init__(self, ctx: Context, M: HostMatrix, form: int, kind: int = TRSV_JACOBI, iters: int = 2,
                 omega: float = 1.0):
        h = C.c_void_p()
        v = M.view()
        check(lib().f3r_trsv_create(ctx._h, C.byref(v), form, kind, iters, omega, C.byref(h)))
        self._h = h
        _LIVE["trsv"].add(self)
        self.ctx = ctx

    def solve(self, x, y) -> None:
        check(lib().f3r_trsv_solve(self._h, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr())))

    def close(self):
        if getattr(self, "_h", None) is not None and _capi is not None and _capi._lib is not None:
            _capi._lib.f3r_trsv_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


@dataclass
class solve_res_t:
    """Mirror of kmm::solve_res_t (umineko-sparse/models.hpp:191-200) plus the
    explicit residual and device time."""
    is_solved: bool
    res_iter: int
    res_nrm2: float
    impl_rel_res: float
    expl_rel_res: float
    restarts: int
    inner_applications: int
    solve_seconds: float
    kernel_launches: int


def Params(**kw) -> _capi.Params:
    p = _capi.Params()
    lib().f3r_params_default(C.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


class Solver:
    """The nested F3R solver (f3r_solver): Restarted(FGMRES<double>(A,
    FGMRES<float>(A32, FGMRES<float>(A16, R)))) with R the adaptive fp16
    Richardson over SDAINV or block-Jacobi ILU(0)."""

    def __init__(self, ctx: Context, A: HostMatrix, params: Optional[_capi.Params] = None, factors=None, **kw):
        """factors: optional (Z, W^T) HostMatrix pair used as the SDAINV
        factors instead of computing them (f3r_solver_create_factors)."""
        p = params if params is not None else Params(**kw)
        h = C.c_void_p()
        v = A.view()
        if factors is None:
            check(lib().f3r_solver_create(ctx._h, C.byref(v), C.byref(p), C.byref(h)))
        else:
            zv, wv = factors[0].view(), factors[1].view()
            check(lib().f3r_solver_create_factors(ctx._h, C.byref(v), C.byref(p), C.byref(zv), C.byref(wv),
                                                  C.byref(h)))
        self._h = h
        _LIVE["solver"].add(self)
        self.ctx = ctx
        self.params = p
        self.n = v.nrows

    def info(self):
        i = _capi.SellInfo()
        d = C.c_int32()
        check(lib().f3r_solver_info(self._h, C.byref(i), C.byref(d)))
        return i, bool(d.value)

    @property
    def unit_diagonal(self) -> bool:
        """True when the diagonal SDAINV factors are 1 in fp16 and the
        Richardson kernels take the constant instead of loading them"""
        i = _capi.SellInfo()
        d = C.c_int32()
        check(lib().f3r_solver_info(self._h, C.byref(i), C.byref(d)))
        return d.value == 2

    def operate(self, x, y, val_t=None) -> None:
        """y = A x with the solver's own device matrix (storage order P A P^T)."""
        xt, yt = _torch_dt(x), _torch_dt(y)
        vt = xt if val_t is None else val_t
        check(lib().f3r_solver_operate(self._h, vt, xt, C.c_void_p(x.data_ptr()), yt, C.c_void_p(y.data_ptr())))

    def solve(self, b, x, cond: Optional[Callable[[int, float], bool]] = None) -> solve_res_t:
        """Solve A x = b.  b, x: numpy float64 arrays (x is updated in place and
        holds the initial guess) or torch CUDA float64 tensors."""
        res = _capi.Result()
        cb = COND_NONE if cond is None else _capi.COND_FN(lambda i, e, u: 1 if cond(i, e) else 0)
        check(lib().f3r_solver_solve(self._h, C.c_void_p(_ptr(b)), C.c_void_p(_ptr(x)), cb, None, C.byref(res)))
        return _res(res)

    def solve_multi(self, B, X, cond: Optional[Callable[[int, float], bool]] = None):
        """Solve A X = B for several right-hand sides: B and X of shape
        (nrhs, n), row k one system (numpy float64 C-contiguous, or torch CUDA
        float64); X is updated in place.  Returns one solve_res_t per row."""
        nrhs, ld = _rows(B, self.n)
        _rows(X, self.n)
        res = (_capi.Result * max(nrhs, 1))()
        cb = COND_NONE if cond is None else _capi.COND_FN(lambda i, e, u: 1 if cond(i, e) else 0)
        check(lib().f3r_solver_solve_multi(self._h, nrhs, C.c_void_p(_ptr(B)), ld, C.c_void_p(_ptr(X)), ld, cb,
                                           None, res))
        return [_res(r) for r in res[:nrhs]]

    def close(self):
        if getattr(self, "_h", None) is not None and _capi is not None and _capi._lib is not None:
            _capi._lib.f3r_solver_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


class Batch:
    """Up to 16 systems of one sparsity pattern solved together
    (f3r_batch_*): one lockstep solve whose columns are the systems, each
    with its own values and SDAINV factors (computed, or given as
    factors=[(Z, W^T), ...])."""

    def __init__(self, ctx: Context, systems, params: Optional[_capi.Params] = None, factors=None, **kw):
        p = params if params is not None else Params(**kw)
        self._views = [A.view() for A in systems]
        count = len(systems)
        arr = (C.POINTER(_capi.CSR) * count)(*[C.pointer(v) for v in self._views])
        zarr = warr = None
        if factors is not None:
            self._fviews = [(Z.view(), W.view()) for Z, W in factors]
            zarr = (C.POINTER(_capi.CSR) * count)(*[C.pointer(z) for z, _ in self._fviews])
            warr = (C.POINTER(_capi.CSR) * count)(*[C.pointer(w) for _, w in self._fviews])
        h = C.c_void_p()
        check(lib().f3r_batch_create(ctx._h, count, arr, C.byref(p), zarr, warr, C.byref(h)))
        self._h = h
        _LIVE["solver"].add(self)
        self.ctx = ctx
        self.count = count
        self.n = self._views[0].nrows

    def info(self):
        """(systems, block width K, diagonal SDAINV)"""
        c, k, d = C.c_int32(), C.c_int32(), C.c_int32()
        check(lib().f3r_batch_info(self._h, C.byref(c), C.byref(k), C.byref(d)))
        return c.value, k.value, bool(d.value)

    @property
    def unit_diagonal(self) -> bool:
        """True when every system's diagonal SDAINV factors are 1 in fp16
        (the Richardson kernels take the constant)"""
        c, k, d = C.c_int32(), C.c_int32(), C.c_int32()
        check(lib().f3r_batch_info(self._h, C.byref(c), C.byref(k), C.byref(d)))
        return d.value == 2

    def solve(self, bs, xs, cond: Optional[Callable[[int, float], bool]] = None):
        """Solve system i for bs[i] into xs[i] (numpy float64 or torch CUDA
        float64 vectors; xs[i] holds the initial guess).  Returns one
        solve_res_t per system."""
        if len(bs) != self.count or len(xs) != self.count:
            raise ValueError("one right-hand side and one solution vector per system")
        for v in list(bs) + list(xs):
            if tuple(v.shape) != (self.n,):
                raise ValueError("vectors must have the systems' row count")
        bp = (C.c_void_p * self.count)(*[_ptr(b) for b in bs])
        xp = (C.c_void_p * self.count)(*[_ptr(x) for x in xs])
        res = (_capi.Result * self.count)()
        cb = COND_NONE if cond is None else _capi.COND_FN(lambda i, e, u: 1 if cond(i, e) else 0)
        check(lib().f3r_batch_solve(self._h, bp, xp, cb, None, res))
        return [_res(r) for r in res]

    def close(self):
        if getattr(self, "_h", None) is not None and _capi is not None and _capi._lib is not None:
            _capi._lib.f3r_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


COND_NONE = _capi.COND_FN()


def _ptr(a) -> int:
    if isinstance(a, np.ndarray):
        if a.dtype != np.float64 or not a.flags.c_contiguous:
            raise TypeError("numpy vectors must be contiguous float64")
        return a.ctypes.data
    if a.dtype != __import__("torch").float64 or not a.is_contiguous():
        raise TypeError("torch vectors must be contiguous float64")
    return a.data_ptr()


def _rows(M, n: int):
    """(nrhs, leading dimension) of a (nrhs, n) block of right-hand sides"""
    shape = tuple(M.shape)
    if len(shape) != 2 or shape[1] != n:
        raise ValueError(f"expected shape (nrhs, {n}), got {shape}")
    return shape[0], n


def _res(res) -> solve_res_t:
    return solve_res_t(bool(res.is_solved), res.res_iter, res.res_nrm2, res.impl_rel_res, res.expl_rel_res,
                       res.restarts, res.inner_applications, res.solve_seconds, res.kernel_launches)


def solve_batch(systems, cond: Optional[Callable[[int, float], bool]] = None):
    """Independent systems at once (f3r_solve_batch): systems is a list of
    (solver, B, X) with B, X of shape (nrhs, n) as in Solver.solve_multi.
    Solvers on different contexts run concurrently.  Returns, per system, the
    list of its solve_res_t."""
    count = len(systems)
    S = (C.c_void_p * max(count, 1))()
    nr = (C.c_int32 * max(count, 1))()
    bp = (C.c_void_p * max(count, 1))()
    xp = (C.c_void_p * max(count, 1))()
    ld = (C.c_int64 * max(count, 1))()
    for i, (solver, B, X) in enumerate(systems):
        k, n = _rows(B, solver.n)
        _rows(X, solver.n)
        S[i], nr[i], bp[i], xp[i], ld[i] = solver._h.value, k, _ptr(B), _ptr(X), n
    total = sum(nr[i] for i in range(count))
    res = (_capi.Result * max(total, 1))()
    cb = COND_NONE if cond is None else _capi.COND_FN(lambda i, e, u: 1 if cond(i, e) else 0)
    check(lib().f3r_solve_batch(count, S, nr, bp, ld, xp, ld, cb, None, res))
    out, at = [], 0
    for i in range(count):
        out.append([_res(r) for r in res[at:at + nr[i]]])
        at += nr[i]
    return out
