"""How far rounding-level changes move the reference's own solve.

Test infrastructure (the product never imports it). It runs the CPU
restatement of the reference's MIC(0)-PCG (oracle/shkz_oracle.c, bit-exact
against the compiled reference: local/include/pcgsolver/pcg_solver.h:246-295)
on one scene four times:

* as the reference assembles it (FP64 matrix and rhs);
* with the matrix entries rounded to FP32, as a solver with FP32 stencil
  coefficients holds them;
* with the rhs perturbed by one FP32 rounding (relative 2^-24, seeded signs);
* with both;

and a tight solve (1e-12) as the exact answer. For each it prints the
iteration count of the infinity-norm stop and the pressure's distance
(infinity norm over the reference's) to the reference run and to the tight
solve. A solver that computes in FP32 cannot be expected to land closer to the
reference than these runs of the reference's own algorithm do.

    python -m oracle.sensitivity --scene splash --n 384 \
        --out tests/golden/sensitivity_splash_384.json          # about 15 minutes
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np


def rel_inf(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def main(argv=None):
    from oracle import oracle
    from shiokaze_b200 import scenes
    ap = argparse.ArgumentParser()
    ap.add_argument("--scene", default="splash", choices=["splash", "sloshing_tank", "dambreak_sphere"])
    ap.add_argument("--n", type=int, default=384)
    ap.add_argument("--tol", type=float, default=1e-6)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=None, help="also write the result as JSON here")
    args = ap.parse_args(argv)
    sc = getattr(scenes, args.scene)(n=args.n, seed=args.seed, tol=args.tol)
    t0 = time.time()
    area, rho = oracle.fractions(sc)
    S = oracle.assemble(sc, area, rho)
    print(f"{args.scene} {args.n}^3: {S.n} unknowns, assembled in {time.time() - t0:.0f} s", flush=True)
    rng = np.random.default_rng(1234)
    sign = rng.choice([-1.0, 1.0], size=S.n)
    data32 = S.data.astype(np.float32).astype(np.float64)
    rhs_p = S.rhs * (1.0 + sign * 2.0 ** -24)
    runs = {
        "reference": (S.data, S.rhs),
        "fp32_matrix": (data32, S.rhs),
        "rhs_rounding": (S.data, rhs_p),
        "fp32_matrix_and_rhs_rounding": (data32, rhs_p),
    }
    out = {}
    sols = {}
    for name, (data, rhs) in runs.items():
        t = time.time()
        sys_v = oracle.System(index=S.index, n=S.n, indptr=S.indptr, indices=S.indices, data=data, rhs=rhs)
        x, it, rr = oracle.pcg(sys_v, args.tol, mic0=True)
        sols[name] = x
        out[name] = {"iterations": it, "reresid": rr}
        print(f"  {name}: {it} iterations, reresid {rr:.3e} ({time.time() - t:.0f} s)", flush=True)
    t = time.time()
    xt, itt, rrt = oracle.pcg(S, 1e-12, mic0=True)
    print(f"  tight solve: {itt} iterations, reresid {rrt:.3e} ({time.time() - t:.0f} s)", flush=True)
    for name in runs:
        out[name]["pressure_vs_reference"] = rel_inf(sols[name], sols["reference"])
        out[name]["pressure_vs_tight"] = rel_inf(sols[name], xt)
    doc = {"scene": args.scene, "n": args.n, "tol": args.tol, "unknowns": S.n, "runs": out,
           "command": f"python -m oracle.sensitivity --scene {args.scene} --n {args.n}",
           "what": ("The CPU restatement of the reference's MIC(0)-PCG (bit-exact against the compiled reference) "
                    f"on the {args.n}^3 {args.scene} at tol {args.tol:g}: as assembled, with the matrix rounded to "
                    "FP32, with the rhs perturbed by one FP32 rounding (relative 2^-24, seeded signs), and both; "
                    "pressure distances are infinity norms over the reference run's (or the 1e-12 tight solve's) "
                    "infinity norm.")}
    print(json.dumps(doc, indent=1))
    if args.out:
        with open(args.out, "w") as f:
            json.dump(doc, f, indent=1)


if __name__ == "__main__":
    main()
