"""Generates the golden fixtures in tests/golden/ from the reference itself.

Runs the reference's own code, compiled in place from the reference tree into
oracle/_ref/libf3r_ref.so (oracle/Makefile, deterministic flags: no FMA
contraction, one OpenMP thread), and records its outputs:

  generators.npz   matrix/hpcg.cpp and matrix/hpgmp.cpp stencils (+ the
                   half-space variant through io::CSR), small grids
  setup.npz        algorithm::scaling, csr_to_sell<32>, algorithm::sdainv,
                   block-Jacobi ILU(0) factors and their fp16 BJ solves
  spmv.npz         SELL<32>::operate / compute_residual at the F3R level types
  solves.npz       full F3R solves (SDAINV + SELL-32, and BJ-ILU(0) + CSR):
                   outer iteration counts, residual histories, final residuals
  trsv.npz         Jacobi-iteration and BAJ triangular solves (trsv/jacobi.hpp,
                   trsv/baj.hpp) in fp16 on the BJ-ILU(0) factors of setup.npz
                   and on a lower triangle with a real diagonal
  mm/*.mtx, mm.npz Matrix Market inputs (two written by the reference's own
                   stencil generators, the rest hand-made to cover comments,
                   symmetric expansion, explicit zeros, integer fields,
                   unsorted and rectangular input, a "_b" right-hand side)
                   and what io::mm::read_system + io::CSR make of them

Usage (needs the reference tree; the fixtures are committed):
    OMP_NUM_THREADS=1 python tests/golden/gen_golden.py [--big]
    python tests/golden/gen_golden.py --envelope [--big] [--only=name,name]
    python tests/golden/gen_golden.py --oracle [--big] [--only=name,name]
--big adds the 64^3 CPU configuration and the 192^3 GPU configuration solve
(about a minute of CPU each).  --envelope re-runs every golden solve at 1, 2,
3, 4 and 8 OpenMP threads (up to 64 for the fp16-vector depth ablations) and
stores the reference's residual histories as <name>_env, the thread counts as
<name>_env_threads: the spread the reference shows when only its summation
order changes.  --oracle stores the oracle's history of every golden solve in
the library's arithmetic as <name>_oracle.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
os.environ.setdefault("OMP_NUM_THREADS", "1")

from oracle import oracle as O  # noqa: E402


def rhs_for(ref, rptr, idx, val, seed):
    """b = A x*, x* ~ U(-1, 1) from a fixed numpy seed (fp64 SpMV of the reference)."""
    n = len(rptr) - 1
    xs = np.random.default_rng(seed).uniform(-1.0, 1.0, n)
    b = ref.sell32_operate(rptr, idx, val, 0, xs)
    return xs, b


MM_HAND = {
    # symmetric, comments and a blank line, an explicit off-diagonal zero
    # (dropped), an explicit zero on the diagonal (kept), entries out of
    # order, exponent and integer spellings; with a right-hand side file
    "sym_mixed.mtx": """%%MatrixMarket matrix coordinate real symmetric
% a comment line
%another one

6 6 12
1 1 4.0
3 1 -1.25e0
2 2 5
6 2 -0.5
3 3 6.5
4 3 0
4 4 3.0E+00
5 5 0.0
2 1 -1
6 6 7.25
5 4 1e-3
6 5 -2.5
""",
    "sym_mixed_b.mtx": """%%MatrixMarket matrix array real general
% b
6 1
1.0
-2.0
3.5e-1
0
4
-0.125
""",
    # integer field, general, rows out of order, a zero off-diagonal
    "gen_int.mtx": """%%MatrixMarket matrix coordinate integer general
5 5 11
5 5 9
1 1 3
2 1 -1
1 3 2
3 3 4
2 2 6
4 2 0
4 4 8
3 5 -2
5 1 1
4 3 -3
""",
    # rectangular (read_matrix does not require a square matrix)
    "rect.mtx": """%%MatrixMarket matrix coordinate real general
3 5 6
1 5 1.5
1 2 -2
2 4 3
3 1 4
3 3 5
2 1 6
""",
}


def mm_fixtures(ref):
    d = os.path.join(HERE, "mm")
    os.makedirs(d, exist_ok=True)
    for name, text in MM_HAND.items():
        with open(os.path.join(d, name), "w") as f:
            f.write(text)
    ref.gen27_save(0, 3, 4, 3, os.path.join(d, "hpcg_3_4_3.mtx"))
    ref.gen27_save(1, 4, 3, 3, os.path.join(d, "hpgmp_4_3_3.mtx"))
    out = {}
    for name in ("sym_mixed", "gen_int", "rect", "hpcg_3_4_3", "hpgmp_4_3_3"):
        r, i, v, b = ref.mm_read_system(os.path.join(d, name + ".mtx"))
        out[name + "_rptr"], out[name + "_idx"], out[name + "_val"], out[name + "_b"] = r, i, v, b
    np.savez_compressed(os.path.join(HERE, "mm.npz"), **out)


TRSV_CASES = [  # (kind, iters, omega): Jacobi on SELL, BAJ on SELL, and the CSR forms
    ("jac", 0, 1.0), ("jac", 1, 1.0), ("jac", 2, 0.7), ("jac", 5, 1.0), ("jac", 3, 1.2),
    ("baj", 1, 1.0), ("baj", 2, 1.0), ("baj", 6, 1.0),
    ("jaccsr", 3, 0.8), ("bajcsr", 1, 1.0), ("bajcsr", 3, 1.0)]


def tril_with_diagonal(rptr, idx, val):
    """lower triangle (diagonal last) of a CSR matrix"""
    rows = np.repeat(np.arange(len(rptr) - 1), np.diff(rptr))
    keep = idx <= rows
    r = np.concatenate([[0], np.cumsum(np.bincount(rows[keep], minlength=len(rptr) - 1))]).astype(np.int32)
    return r, idx[keep].astype(np.int32), val[keep].astype(np.float64)


def trsv_fixtures(ref, s):
    """s: the setup.npz dictionary (hpcg8 ILU factors, bj_in)"""
    t = {}
    r, i, v = ref.gen27(8, 8, 8, variant=0)  # unscaled: diagonal 26
    tl = tril_with_diagonal(r, i, v)
    t["tl_rptr"], t["tl_idx"], t["tl_val"] = tl
    key = "hpcg8_ilu16"
    mats = {"L": (s[key + "_L_rptr"], s[key + "_L_idx"], s[key + "_L_val"], 0), "Tl": tl + (1,),
            "U": (s[key + "_U_rptr"], s[key + "_U_idx"], s[key + "_U_val"], 2)}
    for name, (mr, mi, mv, form) in mats.items():
        for kind, iters, om in TRSV_CASES:
            if kind == "baj" and name == "U" and iters == 1:
                continue  # the SELL form's d_upper init pairs in[i] with row n-1-i's diagonal (baj.hpp:161-170)
            out = ref.jacobi_trsv(mr, mi, mv, form, s["bj_in"], iters, om, baj=kind.startswith("baj"),
                                  csr=kind.endswith("csr"))
            t[f"{name}_{kind}_{iters}_{om}"] = out
    np.savez_compressed(os.path.join(HERE, "trsv.npz"), **t)


# F3R-Static (static.cpp) and the fp32 depth ablations (depth.cpp), BJ-ILU(0)
VARIANTS = {"static_hpgmp16": dict(config=2, m2=8, m3=4, m4=2, weight=1.2),
            "depth3_hpgmp16": dict(config=3, m2=8, m3=8, m4=1, weight=1.0),
            "depth2_hpgmp16": dict(config=4, m2=64, m3=0, m4=1, weight=1.0)}
# 7-point log-normal diffusion systems: (nx, sigma, correlation length, field seed).  diffs25_48 is the
# precision-stress configuration (sigma 2.5, correlation length 8) at 48^3
DIFFUSION = {"sdainv_diff12": (12, 1.5, 3.0, 9), "sdainv_diffs25_48": (48, 2.5, 8.0, 3)}
# the depth ablations with an fp16-vector innermost FGMRES level (depth.cpp F4, F3H, F2H), BJ-ILU(0)
DEPTH_HALF = {"f4_hpgmp16": 0, "f3h_hpgmp16": 1, "f2h_hpgmp16": 2}
# OpenMP thread counts of the envelope: each changes only the summation order of the reference's reductions.
# The fp16-vector levels accumulate their dot products and norms in fp16, one partial sum per thread, so
# their accuracy grows with the thread count: their envelope reaches 64 threads.
ENV_THREADS = (1, 2, 3, 4, 8)
ENV_THREADS_WIDE = (1, 2, 3, 4, 8, 16, 32, 64)


def solve_cases(big):
    """(name, config, stencil spec or None for DIFFUSION, rhs seed) of every golden solve"""
    cases = [("sdainv_hpgmp16", 0, (16, 16, 16, 1), 0), ("sdainv_half16", 0, (16, 16, 16, 2), 1),
             ("sdainv_diff12", 0, None, 2), ("bjilu_hpcg16", 1, (16, 16, 16, 0), 3),
             ("sdainv_diffs25_48", 0, None, 16)]
    if big:
        cases += [("bjilu_hpcg64", 1, (64, 64, 64, 0), 4), ("sdainv_half192", 0, (192, 192, 192, 2), 5)]
    cases += [(k, v["config"], (16, 16, 16, 1), 6 + j) for j, (k, v) in enumerate(VARIANTS.items())]
    # sFGMRES inner levels (solver/gmres2.hpp:137-221): mask bit 0 level 2, bit 1 level 3
    cases += [(f"sstep{mask}_hpgmp16", 10 + mask, (16, 16, 16, 1), 12 + mask) for mask in (1, 2, 3)]
    cases += [(name, 20 + v, (16, 16, 16, 1), 17 + v) for name, v in DEPTH_HALF.items()]
    return cases


def case_system(ref, name, spec):
    """the scaled matrix of a golden solve"""
    import f3r_b200 as F  # host-side generator only (no GPU needed)
    if spec is None:
        nx, sg, cl, fs = DIFFUSION[name]
        rr, ii, vv = F.diffusion7(nx, nx, nx, sg, cl, fs).arrays()
    else:
        rr, ii, vv = ref.gen27(*spec[:3], variant=spec[3], beta=0.5)
    return rr, ii, ref.scaling(rr, ii, vv)


def case_blocks(spec):
    return 16 if spec is not None and spec[0] == 16 else 112


def run_case(ref, name, config, spec, seed):
    rr, ii, vv = case_system(ref, name, spec)
    xs, b = rhs_for(ref, rr, ii, vv, seed)
    extra = {k: v for k, v in VARIANTS.get(name, {}).items() if k != "config"}
    if config >= 20:
        return ref.f3r_solve_depth_half(config - 20, rr, ii, vv, b, tol=1e-10, blocks=case_blocks(spec))
    if config >= 10:
        return ref.f3r_solve_sstep(config - 10, rr, ii, vv, b, tol=1e-10, c=8)
    big = len(rr) - 1 >= 48 ** 3
    return ref.f3r_solve(config, rr, ii, vv, b, tol=1e-10, c=64 if big else 8, blocks=case_blocks(spec), **extra)


def envelope(big, only=None):
    """The reference's residual history of every golden solve at each thread
    count of ENV_THREADS, stored as <name>_env (rows: thread counts, NaN past a
    run's last step).  The reference is not reproducible across thread counts
    (OpenMP reductions), so its own spread bounds what any reimplementation can
    match step by step."""
    import ctypes
    gomp = ctypes.CDLL("libgomp.so.1")
    ref = O.Ref("golden")
    path = os.path.join(HERE, "solves.npz")
    sol = dict(np.load(path))
    for name, config, spec, seed in solve_cases(big):
        if only and name not in only:
            continue
        hs = []
        threads = ENV_THREADS_WIDE if name in DEPTH_HALF else ENV_THREADS
        for t in threads:
            gomp.omp_set_num_threads(t)
            hs.append(run_case(ref, name, config, spec, seed)["hist"])
        w = max(len(h) for h in hs)
        env = np.full((len(hs), w), np.nan)
        for k, h in enumerate(hs):
            env[k, :len(h)] = h
        sol[name + "_env"] = env
        sol[name + "_env_threads"] = np.array(threads)
        print(name, [len(h) for h in hs])
    gomp.omp_set_num_threads(1)
    np.savez_compressed(path, **sol)


def main(big: bool):
    O.build()
    ref = O.Ref("golden")
    mm_fixtures(ref)
    out = {}

    # ---- generators -------------------------------------------------------
    g = {}
    for variant in (0, 1, 2):
        for dims in ((5, 6, 7), (8, 8, 8)):
            r, i, v = ref.gen27(*dims, variant=variant, beta=0.5)
            key = f"v{variant}_{dims[0]}x{dims[1]}x{dims[2]}"
            g[key + "_rptr"], g[key + "_idx"], g[key + "_val"] = r, i, v
    np.savez_compressed(os.path.join(HERE, "generators.npz"), **g)

    # ---- set-up: scaling, SELL, SDAINV, ILU -------------------------------
    s = {}
    r, i, v = ref.gen27(8, 8, 8, variant=1)
    vs = ref.scaling(r, i, v)
    s["hpgmp8_rptr"], s["hpgmp8_idx"], s["hpgmp8_val"], s["hpgmp8_scaled"] = r, i, v, vs
    sp, si, sv = ref.sell32(r, i, vs)
    s["hpgmp8_sell_sptr"], s["hpgmp8_sell_idx"], s["hpgmp8_sell_val"] = sp, si, sv
    # a ragged matrix: 7-point diffusion with random coefficients, odd size
    import f3r_b200 as F  # host-side generator only (no GPU needed)
    D = F.diffusion7(6, 7, 9, 1.5, 2.0, 5)
    dr, di, dv = D.arrays()
    dvs = ref.scaling(dr, di, dv)
    s["diff_rptr"], s["diff_idx"], s["diff_val"], s["diff_scaled"] = dr, di, dv, dvs
    sp, si, sv = ref.sell32(dr, di, dvs)
    s["diff_sell_sptr"], s["diff_sell_idx"], s["diff_sell_val"] = sp, si, sv
    for name, (rr, ii, vv) in (("hpgmp8", (r, i, vs)), ("diff", (dr, di, dvs))):
        (zr, zi, zv), (wr, wi, wv) = ref.sdainv(rr, ii, vv, 0.1, 1.0)
        s[f"{name}_Z_rptr"], s[f"{name}_Z_idx"], s[f"{name}_Z_val"] = zr, zi, zv
        s[f"{name}_W_rptr"], s[f"{name}_W_idx"], s[f"{name}_W_val"] = wr, wi, wv
        (zr, zi, zv), (wr, wi, wv) = ref.sdainv(rr, ii, vv, 0.05, 1.2)
        s[f"{name}_Zb_rptr"], s[f"{name}_Zb_idx"], s[f"{name}_Zb_val"] = zr, zi, zv
        s[f"{name}_Wb_rptr"], s[f"{name}_Wb_idx"], s[f"{name}_Wb_val"] = wr, wi, wv
    hr, hi, hv = ref.gen27(8, 8, 8, variant=0)
    hvs = ref.scaling(hr, hi, hv)
    x16 = np.random.default_rng(3).standard_normal(len(hr) - 1).astype(np.float16)
    for blocks, acc in ((16, 1.0), (7, 1.3)):
        (L, U), lo, up = ref.ilu0_bj(hr, hi, hvs, blocks, acc, solve_in=x16)
        key = f"hpcg8_ilu{blocks}"
        s[key + "_L_rptr"], s[key + "_L_idx"], s[key + "_L_val"] = L
        s[key + "_U_rptr"], s[key + "_U_idx"], s[key + "_U_val"] = U
        s[key + "_lower"], s[key + "_upper"] = lo, up
    s["hpcg8_rptr"], s["hpcg8_idx"], s["hpcg8_scaled"], s["bj_in"] = hr, hi, hvs, x16
    np.savez_compressed(os.path.join(HERE, "setup.npz"), **s)
    trsv_fixtures(ref, s)

    # ---- SpMV kinds --------------------------------------------------------
    m = {}
    rng = np.random.default_rng(11)
    for name, (rr, ii, vv) in (("hpgmp8", (r, i, vs)), ("diff", (dr, di, dvs))):
        n = len(rr) - 1
        x64 = rng.standard_normal(n)
        m[f"{name}_x64"] = x64
        m[f"{name}_y0"] = ref.sell32_operate(rr, ii, vv, 0, x64)
        m[f"{name}_y1"] = ref.sell32_operate(rr, ii, vv, 1, x64.astype(np.float32))
        m[f"{name}_y2"] = ref.sell32_operate(rr, ii, vv, 2, x64.astype(np.float32))
        m[f"{name}_y3"] = ref.sell32_operate(rr, ii, vv, 3, (0.25 * x64).astype(np.float16))
        b64 = rng.standard_normal(n)
        m[f"{name}_b64"] = b64
        m[f"{name}_r0"] = ref.sell32_residual(rr, ii, vv, 0, b64, x64)
        m[f"{name}_r3"] = ref.sell32_residual(rr, ii, vv, 3, b64.astype(np.float16),
                                              (0.1 * x64).astype(np.float16))
    np.savez_compressed(os.path.join(HERE, "spmv.npz"), **m)

    # ---- solves --------------------------------------------------------------
    sol = {}
    for name, config, spec, seed in solve_cases(big):
        res = run_case(ref, name, config, spec, seed)
        rr = case_system(ref, name, spec)[0]
        blocks = case_blocks(spec)
        print(name, res["iters"], res["impl_res"], res["expl_res"], res["time_s"])
        sol[name + "_iters"] = np.array(res["iters"])
        sol[name + "_hist"] = res["hist"]
        sol[name + "_expl"] = np.array(res["expl_res"])
        sol[name + "_seed"] = np.array(seed)
        sol[name + "_blocks"] = np.array(blocks)
        if len(rr) - 1 <= 8192:
            sol[name + "_x"] = res["x"]
    existing = os.path.join(HERE, "solves.npz")
    if not big and os.path.exists(existing):
        old = dict(np.load(existing))
        for k, v in old.items():
            if k not in sol:
                sol[k] = v
    np.savez_compressed(existing, **sol)


def oracle_rows(big, only=None):
    """The oracle's history of every golden solve in the library's arithmetic
    (oracle/f3r_oracle.c, ARITH_PRODUCT: fp16 products accumulated in fp32),
    stored as <name>_oracle.  It restates the reference's algorithm exactly
    and differs from it only in that arithmetic, so the band of
    tests/history_band.py spans it beside the reference's own runs."""
    sys.path.insert(0, os.path.dirname(HERE))
    from history_band import CASES
    path = os.path.join(HERE, "solves.npz")
    sol = dict(np.load(path))
    ref = O.Ref("golden")
    for name, config, spec, seed in solve_cases(big):
        if only and name not in only:
            continue
        rr, ii, vv = case_system(ref, name, spec)
        xs, b = rhs_for(ref, rr, ii, vv, seed)
        cfg = CASES[name]
        A = O.Mat.from_csr(rr, ii, vv)
        if cfg.get("precond", 0) == 1:
            P1, P2 = O.ilu0_bj(A, cfg["ilu_blocks"])
        else:
            Z, W = O.sdainv(A)
            P1, P2 = W, Z
        kw = {k: cfg[k] for k in ("m2", "m3", "m4", "static_weight", "c", "half_m") if k in cfg}
        if "inner_sstep" in cfg:
            kw["sstep"] = cfg["inner_sstep"]
        o = O.f3r_solve(A, P1, P2, b, O.params(precond=cfg.get("precond", 0), tol=1e-10, **kw))
        sol[name + "_oracle"] = o["hist"]
        print(name, "oracle", o["iters"], flush=True)
    np.savez_compressed(path, **sol)


if __name__ == "__main__":
    sel = [a.split("=", 1)[1].split(",") for a in sys.argv if a.startswith("--only=")]
    if "--envelope" in sys.argv:
        envelope("--big" in sys.argv, sel[0] if sel else None)
    elif "--oracle" in sys.argv:
        oracle_rows("--big" in sys.argv, sel[0] if sel else None)
    else:
        main("--big" in sys.argv)
