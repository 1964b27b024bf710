"""SELL-32(-sigma) SpMV / residual / dot on the GPU against the oracle.

The oracle's fma-chain SpMV in stored column order is the CUDA kernel's exact
arithmetic, so fp64 and fp32 results must agree bit for bit, and fp16 results
(fp32 accumulation, one rounding at the store) as well.  The reference's own
fp16-accumulating SpMV is compared within the bound nnz_row * 2^-11 * |A||x|.
"""
import numpy as np
import pytest
import torch

import f3r_b200 as F
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return F.Context(0)


def ragged_matrix(n=1000, m=None, seed=0, empty_every=7):
    """random sparse matrix with empty rows and rows of very different lengths"""
    m = n if m is None else m
    rng = np.random.default_rng(seed)
    rptr = [0]
    idx, val = [], []
    for i in range(n):
        k = 0 if i % empty_every == 3 else int(rng.integers(1, 70 if i % 97 == 0 else 12))
        cols = np.sort(rng.choice(m, size=min(k, m), replace=False))
        idx.extend(cols.tolist())
        val.extend(rng.standard_normal(len(cols)).tolist())
        rptr.append(len(idx))
    return np.array(rptr, np.int32), np.array(idx, np.int32), np.array(val)


CASES = [("stencil", None), ("ragged", None)]


def matrices():
    A = F.stencil27(12, 13, 11, 2, 0.5).scale()
    yield "stencil27", A
    yield "ragged", F.HostMatrix.from_csr(*ragged_matrix(1000))
    yield "ragged_odd", F.HostMatrix.from_csr(*ragged_matrix(77, seed=3))
    yield "diffusion7", F.diffusion7(10, 9, 8, 2.5, 3.0, 1).scale()


FORM_BITS = {"int32": 32, "index16": 16, "aligned": 0, "csr": 32}


def make_sell(ctx, A, sigma, form):
    return F.Sell(ctx, A, sigma=sigma, index16=form == "index16", aligned=form == "aligned", csr=form == "csr")


@pytest.mark.parametrize("sigma,form", [(1, "int32"), (256, "int32"), (1, "index16"), (256, "index16"),
                                        (1, "aligned"), (256, "aligned"), (32, "aligned"), (1, "csr")])
def test_operate_bitexact(ctx, sigma, form):
    """every index form gives the oracle's sums bit for bit.  The aligned
    cases cover the fully aligned form (stencils in natural order, clamped
    edge slices), the mixed form (ragged matrices, sorted rows) and its
    explicit slices"""
    for name, A in matrices():
        rptr, idx, val = A.arrays()
        n = A.shape[0]
        S = make_sell(ctx, A, sigma, form)
        assert S.info().index_bits == FORM_BITS[form]
        rng = np.random.default_rng(1)
        x64 = rng.standard_normal(n)
        x32 = x64.astype(np.float32)
        x16 = (x64 * 0.25).astype(np.float16)
        cases = [
            (F.F64, x64, torch.float64, O.DT_F64, O.DT_F64, O.DT_F64),
            (F.F32, x32, torch.float32, O.DT_F32, O.DT_F32, O.DT_F32),
            (F.F16, x32, torch.float32, O.DT_F16, O.DT_F32, O.DT_F32),
            (F.F16, x16, torch.float16, O.DT_F16, O.DT_F16, O.DT_F32),
        ]
        for vt, x, ydt, ov, oy, oacc in cases:
            xt = torch.from_numpy(x).cuda()
            yt = torch.zeros(n, dtype=ydt, device="cuda")
            S.operate(xt, yt, val_t=vt)
            torch.cuda.synchronize()
            ref = O.spmv(rptr, idx, val, x, ov, oy, oacc)
            assert np.array_equal(yt.cpu().numpy().view(np.uint8), ref.view(np.uint8)), (name, vt, x.dtype)
        # fp16 vector output
        xt = torch.from_numpy(x16).cuda()
        yt = torch.zeros(n, dtype=torch.float16, device="cuda")
        S.operate(xt, yt)
        torch.cuda.synchronize()
        ref = O.spmv(rptr, idx, val, x16, O.DT_F16, O.DT_F16, O.DT_F32)
        assert np.array_equal(yt.cpu().numpy().view(np.uint16), ref.view(np.uint16)), name
        info = S.info()
        assert info.nrows == n and info.nnz == len(idx) and info.nnz_padded >= len(idx)
        S.close()


@pytest.mark.parametrize("sigma,form", [(1, "int32"), (32, "int32"), (32, "index16"), (1, "aligned"),
                                        (32, "aligned"), (1, "csr")])
def test_residual_bitexact(ctx, sigma, form):
    for name, A in matrices():
        rptr, idx, val = A.arrays()
        n = A.shape[0]
        S = make_sell(ctx, A, sigma, form)
        rng = np.random.default_rng(2)
        for dt, odt in ((np.float64, O.DT_F64), (np.float32, O.DT_F32), (np.float16, O.DT_F16)):
            x = (rng.standard_normal(n) * 0.1).astype(dt)
            b = rng.standard_normal(n).astype(dt)
            tdt = {np.float64: torch.float64, np.float32: torch.float32, np.float16: torch.float16}[dt]
            r = torch.zeros(n, dtype=tdt, device="cuda")
            S.compute_residual(torch.from_numpy(b).cuda(), torch.from_numpy(x).cuda(), r)
            torch.cuda.synchronize()
            acc = O.DT_F64 if dt == np.float64 else O.DT_F32
            ref = O.spmv(rptr, idx, val, x, odt, odt, acc, b=b)
            assert np.array_equal(r.cpu().numpy().view(np.uint8), ref.view(np.uint8)), (name, dt)
        S.close()


def test_wide_columns_fall_back_to_32bit(ctx):
    """rows whose columns spread over more than 65536 keep 32-bit indices"""
    n = 70000
    rptr, idx, val = ragged_matrix(n, seed=11, empty_every=5)
    A = F.HostMatrix.from_csr(rptr, idx, val)
    S = F.Sell(ctx, A, index16=True)
    assert S.info().index_bits == 32
    x = np.random.default_rng(4).standard_normal(n)
    y = torch.zeros(n, dtype=torch.float64, device="cuda")
    S.operate(torch.from_numpy(x).cuda(), y)
    torch.cuda.synchronize()
    ref = O.spmv(rptr, idx, val, x, O.DT_F64, O.DT_F64, O.DT_F64)
    assert np.array_equal(y.cpu().numpy(), ref)


@pytest.mark.parametrize("dims", [(32, 20, 9), (16, 16, 16), (33, 7, 5)])
def test_aligned_stencil_matches_packed(ctx, dims):
    """a 27-point stencil in natural order takes the fully aligned form (no
    index stored, widths padded from 27 to 28): every value type's product
    equals the packed int32 form's bit for bit, including the clamped slices
    at the matrix's first and last rows"""
    A = F.stencil27(*dims, 2, 0.5).scale()
    n = A.shape[0]
    S32, SA = F.Sell(ctx, A), F.Sell(ctx, A, aligned=True)
    assert SA.info().index_bits == 0
    assert S32.info().nnz_padded < SA.info().nnz_padded <= S32.info().nnz_padded * 1.2  # widths to a multiple of 4
    rng = np.random.default_rng(9)
    for vt, dt in ((F.F16, torch.float32), (F.F32, torch.float32), (F.F64, torch.float64), (F.F16, torch.float16)):
        x = torch.from_numpy(rng.standard_normal(n)).to(dt).cuda()
        y1 = torch.zeros(n, dtype=dt, device="cuda")
        y2 = torch.zeros_like(y1)
        S32.operate(x, y1, val_t=vt)
        SA.operate(x, y2, val_t=vt)
        torch.cuda.synchronize()
        assert np.array_equal(y1.cpu().numpy().view(np.uint8), y2.cpu().numpy().view(np.uint8)), (vt, dt)


@pytest.mark.parametrize("dims", [(32, 20, 9), (16, 16, 16), (33, 7, 5), (64, 3, 3)])
def test_slice_height_64_matches_32(ctx, dims):
    """64-row offset-aligned slices (each lane two rows, one set of slot
    bases): every value type's product, residual included, equals the 32-row
    layouts' bit for bit, clamped first and last slices and a ragged last
    slice included"""
    A = F.stencil27(*dims, 2, 0.5).scale()
    n = A.shape[0]
    S32, S64 = F.Sell(ctx, A, aligned=True), F.Sell(ctx, A, height=64)
    assert S64.info().slice_height == 64 and S64.info().index_bits == 0
    assert S64.info().nslices == (n + 63) // 64
    rng = np.random.default_rng(19)
    for vt, dt in ((F.F16, torch.float32), (F.F32, torch.float32), (F.F64, torch.float64), (F.F16, torch.float16)):
        x = torch.from_numpy(rng.standard_normal(n)).to(dt).cuda()
        y1 = torch.zeros(n, dtype=dt, device="cuda")
        y2 = torch.zeros_like(y1)
        S32.operate(x, y1, val_t=vt)
        S64.operate(x, y2, val_t=vt)
        torch.cuda.synchronize()
        assert np.array_equal(y1.cpu().numpy().view(np.uint8), y2.cpu().numpy().view(np.uint8)), (vt, dt)
    b = torch.from_numpy(rng.standard_normal(n)).cuda()
    x = torch.from_numpy(rng.standard_normal(n)).cuda()
    r1, r2 = torch.zeros_like(b), torch.zeros_like(b)
    S32.compute_residual(b, x, r1)
    S64.compute_residual(b, x, r2)
    assert torch.equal(r1, r2)
    # rows with scattered columns share no offsets: far more slots than entries
    with pytest.raises(F.F3RError):
        F.Sell(ctx, F.HostMatrix.from_csr(*ragged_matrix(640, seed=5)), height=64)


def test_fp16_within_reference_bound(ctx):
    """against the reference's fp16-accumulated SELL<32,__half>::operate"""
    ref = O.Ref("golden")
    A = F.stencil27(16, 16, 16, 2, 0.5).scale()
    rptr, idx, val = A.arrays()
    n = A.shape[0]
    x16 = np.random.default_rng(5).standard_normal(n).astype(np.float16)
    S = F.Sell(ctx, A)
    y = torch.zeros(n, dtype=torch.float16, device="cuda")
    S.operate(torch.from_numpy(x16).cuda(), y)
    got = y.cpu().numpy().astype(np.float64)
    want = ref.sell32_operate(rptr, idx, val, 3, x16).astype(np.float64)
    absAx = O.spmv(rptr, idx, np.abs(val), np.abs(x16.astype(np.float64)), O.DT_F64, O.DT_F64, O.DT_F64)
    rowlen = np.diff(rptr)
    bound = rowlen * 2.0 ** -11 * absAx + 2.0 ** -24
    assert np.all(np.abs(got - want) <= 2 * bound)


def test_dot(ctx):
    rng = np.random.default_rng(3)
    for n in (0, 1, 1000, 1 << 20):
        a = rng.standard_normal(n)
        b = rng.standard_normal(n)
        got = ctx.dot(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda())
        assert abs(got - float(a @ b)) <= 1e-12 * (np.abs(a) @ np.abs(b) + 1)
        a32, b32 = a.astype(np.float32), b.astype(np.float32)
        got = ctx.dot(torch.from_numpy(a32).cuda(), torch.from_numpy(b32).cuda())
        assert abs(got - float(a32.astype(np.float64) @ b32)) <= 1e-5 * (np.abs(a) @ np.abs(b) + 1)


def test_csr_rows_across_tiles(ctx):
    """CSR rows longer than a staging tile (512 entries) and groups whose
    range starts mid-tile: the sums stay the oracle's"""
    n = 300
    rng = np.random.default_rng(6)
    lens = rng.integers(0, 40, n)
    lens[[5, 33, 34, 200]] = [700, 1300, 513, 2048]
    rptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    idx = np.concatenate([np.sort(rng.choice(4096, size=k, replace=False)) for k in lens]).astype(np.int32)
    val = rng.standard_normal(len(idx))
    A = F.HostMatrix.from_csr(rptr, idx, val, ncols=4096)
    S = F.Sell(ctx, A, csr=True)
    assert S.info().slice_height == 0 and S.info().max_width == 2048
    x = rng.standard_normal(4096)
    for vt, xd, ov in ((F.F64, x, O.DT_F64), (F.F32, x.astype(np.float32), O.DT_F32)):
        y = torch.zeros(n, dtype=torch.float64 if vt == F.F64 else torch.float32, device="cuda")
        S.operate(torch.from_numpy(xd).cuda(), y, val_t=vt)
        torch.cuda.synchronize()
        assert np.array_equal(y.cpu().numpy(), O.spmv(rptr, idx, val, xd, ov, ov, ov))


def test_empty_and_bad_inputs(ctx):
    A = F.HostMatrix.from_csr(np.zeros(5, np.int32), np.zeros(0, np.int32), np.zeros(0))
    S = F.Sell(ctx, A)
    y = torch.ones(4, dtype=torch.float64, device="cuda")
    S.operate(torch.ones(4, dtype=torch.float64, device="cuda"), y)
    torch.cuda.synchronize()
    assert torch.all(y == 0)
    with pytest.raises(F.F3RError):
        F.HostMatrix.from_csr(np.array([0, 2], np.int32), np.array([1, 0], np.int32), np.ones(2))
    with pytest.raises(F.F3RError):
        F.Sell(ctx, F.stencil27(4, 4, 4), sigma=0)
    # an empty CSR matrix, CSR with sorting or another layout flag, tuning a CSR matrix
    S = F.Sell(ctx, A, csr=True)
    y = torch.ones(4, dtype=torch.float64, device="cuda")
    S.operate(torch.ones(4, dtype=torch.float64, device="cuda"), y)
    torch.cuda.synchronize()
    assert torch.all(y == 0)
    with pytest.raises(F.F3RError, match="sigma 1"):
        F.Sell(ctx, F.stencil27(4, 4, 4), sigma=32, csr=True)
    with pytest.raises(F.F3RError, match="sigma 1"):
        F.Sell(ctx, F.stencil27(4, 4, 4), aligned=True, csr=True)
    with pytest.raises(F.F3RError, match="CSR"):
        F.Sell(ctx, F.stencil27(8, 8, 8), csr=True).tune(F.F16, reps=1)


@pytest.mark.parametrize("aligned", [False, True])
def test_tune_times_every_shape(ctx, aligned):
    A = F.stencil27(24, 24, 24, 2, 0.5).scale()
    S = F.Sell(ctx, A, aligned=aligned)
    for vt in (F.F16, F.F32, F.F64):
        rows = S.tune(vt, reps=3)
        # shapes whose rings exceed the shared memory are skipped; the aligned
        # forms are laid out for one chunk width
        assert len(rows) >= (2 if aligned else 3)
        assert sum(r["default"] for r in rows) == 1
        assert all(r["us"] > 0 for r in rows)
        assert rows == sorted(rows, key=lambda r: r["us"])
