"""Launch-shape and layout sweep of the SELL SpMV (the library's autotuner).

    python -m f3r_b200.tune [--nx 192] [--reps 20] [--forms aligned,int32,...] [--types f16,f32,f64]

Builds the nonsymmetric 27-point matrix of the benchmark (scaled), stores it
as SELL-32 with sigma in {1, 256} and 32- or 16-bit column indices, and with
sigma = 1 also offset-aligned (no stored column index), and times out = A x
for fp16 values (fp32 vectors), fp32 and fp64 at every launch shape the
library carries for that layout (f3r_sell_tune).  Prints one markdown table
per case.
"""
from __future__ import annotations

import argparse

import f3r_b200 as F


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=192)
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--forms", default="aligned64,aligned,int32,index16,s256-int32,s256-index16",
                    help="layouts to sweep: aligned64, aligned, int32, index16 (sigma 1), s256-int32, s256-index16")
    ap.add_argument("--types", default="f16,f32,f64", help="value types to sweep")
    args = ap.parse_args()
    forms = set(args.forms.split(","))
    types = set(args.types.split(","))
    A = F.stencil27(args.nx, args.nx, args.nx, 2, 0.5).scale()
    ctx = F.Context(0)
    print(f"# SELL SpMV launch-shape sweep, {args.nx}^3 27-point (n={A.shape[0]}, nnz={A.nnz})\n")
    for sigma, form in ((1, "aligned64"), (1, "aligned"), (1, "int32"), (1, "index16"), (256, "int32"),
                        (256, "index16")):
        if (form if sigma == 1 else f"s256-{form}") not in forms:
            continue
        S = F.Sell(ctx, A, sigma=sigma, index16=form == "index16", aligned=form.startswith("aligned"),
                   height=64 if form == "aligned64" else 32)
        bits = S.info().index_bits
        label = "offset-aligned (no stored index)" if bits == 0 else f"{bits}-bit indices"
        if form == "aligned64":
            label = "64-row offset-aligned slices (two rows a lane, no stored index)"
        for vt, name, key in ((F.F16, "fp16 values x fp32 vectors", "f16"), (F.F32, "fp32", "f32"),
                              (F.F64, "fp64", "f64")):
            if key not in types:
                continue
            rows = S.tune(vt, args.reps)
            print(f"## sigma={sigma}, {label}, {name}\n")
            print("| warps | stages | cols/copy | us | GB/s (algorithmic) | default |")
            print("|---|---|---|---|---|---|")
            for r in rows:
                print(f"| {r['warps']} | {r['stages']} | {r['kc']} | {r['us']:.1f} | {r['gbs']:.0f} | "
                      f"{'yes' if r['default'] else ''} |")
            print()
        S.close()
    ctx.close()


if __name__ == "__main__":
    main()
