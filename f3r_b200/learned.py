"""The learned correction of SDAINV's values (the f3r_learned_* entry points):
training data from the solver's own residual / error pairs, training by the
library's CUDA forward / backward kernels, and corrected factors for new
systems (BF16 tensor-core inference).  The reference has no counterpart; the
plain SDAINV that is corrected is preconditioner/ainv.hpp:27-65.

A workflow::

    ts = training_set(ctx, seeds=range(256), nt=24)      # 7-point fields
    L = Learned(ctx)
    L.set_data(**ts.data())
    losses = L.train(500, lr=2e-3)
    A = diffusion7(128, 128, 128, 1.5, 6.0, seed).scale()
    Z, Wt = A.sdainv()
    S = Solver(ctx, A, factors=L.correct(A, 128, 128, Z, Wt))
"""
import ctypes as C
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _LIVE, HostMatrix, Solver, _capi, check, diffusion7, lib, random_uniform

N_PARAMS = 5192
HIDDEN = 64
# parameter blocks of the flat vector: name -> (offset, shape)
LAYOUT = {"W1": (0, (64, 7)), "b1": (448, (64,)), "W2": (512, (64, 64)), "b2": (4608, (64,)),
          "W3": (4672, (8, 64)), "b3": (5184, (8,))}


class Learned:
    """The network (f3r_learned): 7 -> 64 -> 64 -> 8, ReLU, fp32 master
    weights on the device."""

    def __init__(self, ctx, seed: int = 0, hidden: int = HIDDEN):
        h = C.c_void_p()
        check(lib().f3r_learned_create(ctx._h, hidden, seed, C.byref(h)))
        self._h = h
        self.ctx = ctx
        _LIVE["learned"].add(self)

    @property
    def params(self) -> np.ndarray:
        p = np.zeros(N_PARAMS, np.float32)
        check(lib().f3r_learned_params(self._h, p.ctypes.data, 0, None))
        return p

    @params.setter
    def params(self, p) -> None:
        p = np.ascontiguousarray(p, np.float32)
        if p.shape != (N_PARAMS,):
            raise ValueError(f"expected {N_PARAMS} parameters")
        check(lib().f3r_learned_params(self._h, p.ctypes.data, 1, None))

    def set_data(self, A: HostMatrix, nx: int, ny: int, Z: HostMatrix, Wt: HostMatrix, r, e) -> None:
        """Training system and pairs: r, e of shape (npairs, n), A e_p = r_p."""
        r = np.ascontiguousarray(r, np.float64)
        e = np.ascontiguousarray(e, np.float64)
        n = A.shape[0]
        if r.ndim != 2 or r.shape != e.shape or r.shape[1] != n:
            raise ValueError("r and e must both be (npairs, n)")
        av, zv, wv = A.view(), Z.view(), Wt.view()
        check(lib().f3r_learned_set_data(self._h, C.byref(av), nx, ny, C.byref(zv), C.byref(wv), r.shape[0],
                                         r.ctypes.data, e.ctypes.data))

    def evaluate(self, grad: bool = False):
        """The loss at the current parameters (and its gradient)."""
        loss = C.c_double()
        g = np.zeros(N_PARAMS, np.float32) if grad else None
        check(lib().f3r_learned_evaluate(self._h, C.byref(loss), None if g is None else g.ctypes.data))
        return (loss.value, g) if grad else loss.value

    def train(self, steps: int, lr: float = 1e-3) -> np.ndarray:
        """steps full-batch Adam steps; returns the loss before each step."""
        losses = np.zeros(max(steps, 0))
        check(lib().f3r_learned_train(self._h, steps, lr, losses.ctypes.data))
        return losses

    ENGINES = {"tcgen05": 1, "mma.sync": 2}

    def _mode(self, bf16: bool, engine: str) -> int:
        if not bf16:
            return 0
        if engine not in self.ENGINES:
            raise ValueError(f"engine must be one of {sorted(self.ENGINES)}")
        return self.ENGINES[engine]

    def correct(self, A: HostMatrix, nx: int, ny: int, Z: HostMatrix, Wt: HostMatrix, bf16: bool = True,
                want_delta: bool = False, engine: str = "tcgen05"):
        """(Z', W'^T): the factors with corrected values (same pattern).
        bf16: BF16 tensor-core inference on `engine` ("tcgen05": TMEM
        accumulators, 128-row tiles; "mma.sync": warp-level 16-row tiles),
        else the fp32 training forward pass."""
        mode = self._mode(bf16, engine)
        av, zv, wv = A.view(), Z.view(), Wt.view()
        zr, zi, _ = Z.arrays()
        wr, wi, _ = Wt.arrays()
        zval, wval = np.zeros(zv.nnz), np.zeros(wv.nnz)
        delta = np.zeros((av.nrows, 8), np.float32) if want_delta else None
        check(lib().f3r_learned_correct(self._h, C.byref(av), nx, ny, C.byref(zv), C.byref(wv), mode,
                                        zval.ctypes.data, wval.ctypes.data,
                                        None if delta is None else delta.ctypes.data))
        out = (HostMatrix.from_csr(zr, zi, zval), HostMatrix.from_csr(wr, wi, wval))
        return out + (delta,) if want_delta else out

    def time_inference(self, A: HostMatrix, nx: int, ny: int, Z: HostMatrix, Wt: HostMatrix, bf16: bool = True,
                       engine: str = "tcgen05", reps: int = 20) -> float:
        """device microseconds of one launch of the network on A's features"""
        av, zv, wv = A.view(), Z.view(), Wt.view()
        us = C.c_double()
        check(lib().f3r_learned_time_inference(self._h, C.byref(av), nx, ny, C.byref(zv), C.byref(wv),
                                               self._mode(bf16, engine), reps, C.byref(us)))
        return us.value

    def close(self):
        if getattr(self, "_h", None) is not None and _capi is not None and _capi._lib is not None:
            _capi._lib.f3r_learned_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def block_diag(mats: Sequence[HostMatrix]) -> HostMatrix:
    """The block-diagonal stack of square matrices (one system per block)."""
    rp, ix, vs = [np.zeros(1, np.int64)], [], []
    off_r, off_nz = 0, 0
    for M in mats:
        r, i, v = M.arrays()
        rp.append(r[1:].astype(np.int64) + off_nz)
        ix.append(i.astype(np.int64) + off_r)
        vs.append(v)
        off_r += len(r) - 1
        off_nz += len(i)
    if off_nz >= 2 ** 31 or off_r >= 2 ** 31:
        raise ValueError("stack exceeds 32-bit indices")
    return HostMatrix.from_csr(np.concatenate(rp).astype(np.int32), np.concatenate(ix).astype(np.int32),
                               np.concatenate(vs))


def solver_pairs(ctx, A: HostMatrix, factors, xs: np.ndarray, outer_steps=(0, 1), **solver_kw):
    """Residual / error pairs the solver generates: for each k in outer_steps,
    the F3R iterate x_k after k outer steps from x0 = 0 (b = A xs), giving
    e = xs - x_k and r = b - A x_k (fp64 on the host)."""
    b = A.spmv(xs)
    S = None
    rs, es = [], []
    for k in outer_steps:
        x = np.zeros(len(b))
        if k > 0:
            if S is None:
                S = Solver(ctx, A, factors=factors, **solver_kw)
            S.solve(b, x, cond=lambda i, e, k=k: i >= k)
        rs.append(b - A.spmv(x))
        es.append(xs - x)
    if S is not None:
        S.close()
    return np.stack(rs), np.stack(es)


@dataclass
class TrainingSet:
    A: HostMatrix
    Z: HostMatrix
    Wt: HostMatrix
    nx: int
    ny: int
    r: np.ndarray
    e: np.ndarray
    fields: int

    def data(self):
        return dict(A=self.A, nx=self.nx, ny=self.ny, Z=self.Z, Wt=self.Wt, r=self.r, e=self.e)


def training_set(ctx, seeds: Sequence[int], nt: int = 24, sigma: float = 1.5, corr_len: float = 6.0,
                 n_initial: int = 4, inner_m4=(2, 8, 16), xseed: int = 12345, **solver_kw) -> TrainingSet:
    """Seeded 7-point log-normal diffusion fields on nt^3 grids (each scaled
    to unit diagonal as the drivers do), stacked block-diagonally into one
    system (a 7-point matrix in natural order on nt x nt x (nt * fields)),
    its SDAINV factors, and residual / error pairs the solver generates:
      - n_initial initial pairs (x0 = 0: e = x*, r = b) for x* ~ U(-1, 1);
      - for each m4 in inner_m4, the iterate after one outer step of a
        shallow F3R (m2 = 1, m3 = 0, Richardson m4 steps) over plain SDAINV,
        whose error is smoothed by the innermost level.
    Later iterates of the full solver (errors in the lowest modes, which no
    fixed-pattern approximate inverse resolves) are left out: trained on
    them, the correction amplifies the high-frequency modes and the solve
    stalls."""
    mats = [diffusion7(nt, nt, nt, sigma, corr_len, int(s)).scale() for s in seeds]
    A = block_diag(mats)
    del mats
    Z, Wt = A.sdainv()
    n = A.shape[0]
    rs, es = [], []
    for j in range(n_initial):
        xs = random_uniform(xseed + j, -1.0, 1.0, n)
        rs.append(A.spmv(xs))
        es.append(xs)
    for j, m4 in enumerate(inner_m4):
        xs = random_uniform(xseed + 1000 + j, -1.0, 1.0, n)
        kw = dict(solver_kw, m2=1, m3=0, m4=m4)
        r, e = solver_pairs(ctx, A, (Z, Wt), xs, (1,), **kw)
        rs.append(r[0])
        es.append(e[0])
    return TrainingSet(A, Z, Wt, nt, nt, np.stack(rs), np.stack(es), len(seeds))


def solve_with_fallback(ctx, A: HostMatrix, b, x, learned_factors, plain_factors, **solver_kw):
    """Solves with the learned factors; should that solve stop unsolved or
    break down (the FP64 outer residual judges it), solves again with plain
    SDAINV: from the learned iterate when it stopped unsolved, from the
    initial guess after a breakdown.  b, x: numpy float64 vectors (x holds
    the initial guess, updated in place).  Returns (result, used_fallback)."""
    from . import F3RError
    x0 = np.array(x, copy=True)
    S = Solver(ctx, A, factors=learned_factors, **solver_kw)
    try:
        res = S.solve(b, x)
        if res.is_solved:
            return res, False
    except F3RError as err:
        if err.status != 5:  # anything but an Arnoldi breakdown is an error of the call itself
            raise
        x[:] = x0
    finally:
        S.close()
    S = Solver(ctx, A, factors=plain_factors, **solver_kw)
    try:
        return S.solve(b, x), True
    finally:
        S.close()
