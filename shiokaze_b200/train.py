"""Training of the learned preconditioner on systems the projection itself builds.

Each seeded training scene (pool height U[0.2,0.5], 1-50 spheres, 0-8 solid
boxes, Gaussian face velocities; ``scenes.training_scene``) is projected on the
GPU with the plain MIC(0) solver, which assembles the pressure system; the
network then takes ``steps`` Adam steps on that system (energy loss, residuals
b, A e and b + A e; see ``shkz_b200_learned_train``). All arithmetic runs in
the CUDA library.

    python -m shiokaze_b200.train --out net.bin --n 64 --scenes 40 --steps 30
"""
from __future__ import annotations

import argparse
import time

import numpy as np

from . import scenes
from .projection import MacPressureSolver3, grids_from_scene


def project_scene(solver: MacPressureSolver3, sc, **cfg) -> dict:
    if cfg:
        solver.configure(cfg)
    solver.initialize((sc.nx, sc.ny, sc.nz), sc.dx)
    vel, solid, svel, fluid = grids_from_scene(sc)
    return solver.project(sc.dt, vel, solid, svel, fluid)


def train(out_path: str, n: int = 64, n_scenes: int = 40, steps: int = 30, lr: float = 1e-3, seed: int = 0,
          init_path: str | None = None, log=print) -> dict:
    s = MacPressureSolver3({"Residual": 1e-6, "B200.Preconditioner": "mic0"})
    t0 = time.time()
    history = []
    for i in range(n_scenes):
        sc = scenes.training_scene(n=n, seed=seed * 100003 + i)
        project_scene(s, sc, **{"B200.Preconditioner": "mic0"})
        if i == 0:
            if init_path:
                s.learned_load(init_path)
            else:
                s.learned_init(seed)
        losses = s.learned_train(steps, lr=lr, seed=seed * 7 + i)
        history.append(float(np.mean(losses[-3:])))
        if log and (i % 5 == 0 or i == n_scenes - 1):
            log(f"scene {i + 1}/{n_scenes}: energy loss {losses[0]:.4g} -> {losses[-1]:.4g} ({time.time() - t0:.1f} s)")
    s.learned_save(out_path)
    return {"scenes": n_scenes, "n": n, "steps": steps, "lr": lr, "seconds": time.time() - t0,
            "final_losses": history[-5:]}


def evaluate(model_path: str, n: int = 64, n_scenes: int = 4, seed: int = 999, tol: float = 1e-6) -> list:
    """Iterations and solve time of identity CG, MIC(0)-PCG and learned FPCG on held-out scenes."""
    s = MacPressureSolver3({"Residual": tol})
    out = []
    for i in range(n_scenes):
        sc = scenes.training_scene(n=n, seed=seed + i)
        row = {"scene": seed + i}
        for name in ("none", "mic0", "learned"):
            if name == "learned":
                project_scene(s, sc, **{"B200.Preconditioner": "mic0"})
                s.learned_load(model_path)
            r = project_scene(s, sc, **{"B200.Preconditioner": name})
            row[name] = {"iterations": r["iterations"], "ms_solve": r["ms_solve"], "reresid": r["reresid"],
                         "fallbacks": r["fallbacks"], "status": r["status"]}
        out.append(row)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--scenes", type=int, default=40)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--init", default=None)
    ap.add_argument("--eval", type=int, default=4)
    args = ap.parse_args()
    info = train(args.out, args.n, args.scenes, args.steps, args.lr, args.seed, args.init)
    print("trained:", info, flush=True)
    if args.eval:
        for row in evaluate(args.out, n=args.n, n_scenes=args.eval):
            print("eval:", row, flush=True)


if __name__ == "__main__":
    main()
