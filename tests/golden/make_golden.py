"""Generate the golden fixtures in this directory from the compiled reference.

Runs the reference's own ``macpressuresolver3::project`` (built by
``oracle/ref/Makefile`` into ``oracle/_ref``) on small seeded scenes and
stores the inputs exactly as the reference grids read them, the assembled
system and the outputs. Needs the reference sources, so it only runs where
they are mounted; the fixtures it writes are committed.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from shiokaze_b200 import scenes  # noqa: E402
from oracle import ref_runner  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

CASES = {
    "dambreak_sphere_16": lambda: scenes.dambreak_sphere(n=16, seed=3, solid_velocity=True),
    "dambreak_sphere_24": lambda: scenes.dambreak_sphere(n=24, seed=7),
    "sloshing_tank_24": lambda: scenes.sloshing_tank(n=24, seed=1, tol=1e-6),
    "splash_24": lambda: scenes.splash(n=24, seed=4, spheres=12),
    "training_20": lambda: scenes.training_scene(n=20, seed=11),
    "analytic_sphere_16": lambda: scenes.analytic_sphere(16)[0],
}


def make(name: str, build) -> str:
    sc = build()
    res = {}
    for mode in ("mic0", "shipped"):
        r = ref_runner.run_reference(sc, mode=mode)
        res[mode] = r
    r = res["mic0"]
    S = r.system
    payload = dict(
        shape=np.array([sc.nx, sc.ny, sc.nz], np.int32),
        dx=np.float64(sc.dx), dt=np.float64(sc.dt), tol=np.float64(sc.tol),
        fluid=r.fluid.astype(np.float32), fluid_active=r.fluid_active,
        solid=r.solid.astype(np.float32), solid_active=r.solid_active,
        has_solid=np.int32(sc.solid_phi is not None),
        u_in=r.velocity_in[0].astype(np.float32), v_in=r.velocity_in[1].astype(np.float32),
        w_in=r.velocity_in[2].astype(np.float32),
        u_in_active=r.velocity_in_active[0], v_in_active=r.velocity_in_active[1],
        w_in_active=r.velocity_in_active[2],
        pressure=r.pressure.astype(np.float32), pressure_active=r.pressure_active,
        u=r.velocity[0].astype(np.float32), v=r.velocity[1].astype(np.float32), w=r.velocity[2].astype(np.float32),
        u_active=r.velocity_active[0], v_active=r.velocity_active[1], w_active=r.velocity_active[2],
        iterations_mic0=np.int32(r.iterations), reresid_mic0=np.float64(r.reresid),
        iterations_shipped=np.int32(res["shipped"].iterations), reresid_shipped=np.float64(res["shipped"].reresid),
        pressure_shipped=res["shipped"].pressure.astype(np.float32),
        indptr=S["indptr"], indices=S["indices"], data=S["data"], rhs=S["rhs"],
    )
    svel = sc.solid_velocity_effective()
    payload.update(us=svel[0], vs=svel[1], ws=svel[2])
    path = os.path.join(OUT, f"{name}.npz")
    np.savez_compressed(path, **payload)
    return path


def main():
    if not ref_runner.ref_available("float"):
        raise SystemExit("compiled reference not found: run `make -C oracle/ref` first")
    for name, build in CASES.items():
        p = make(name, build)
        print(p, os.path.getsize(p))


if __name__ == "__main__":
    main()
