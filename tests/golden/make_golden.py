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


# Optional terms of the projection (macpressuresolver3.cpp:75-80, 98-128,
# 219-259, 286-293): each case runs the reference's MIC(0) mode with one term on.
def _density(sc, seed):
    rng = np.random.default_rng(seed)
    shapes = [(sc.nz, sc.ny, sc.nx + 1), (sc.nz, sc.ny + 1, sc.nx), (sc.nz + 1, sc.ny, sc.nx)]
    return [rng.uniform(0.0, 1.0, s).astype(np.float32) for s in shapes]


TERM_CASES = {
    "term_surface_tension_20": lambda: (scenes.training_scene(n=20, seed=5), {"kappa": 0.05}),
    "term_solid_density_20": lambda: (scenes.dambreak_sphere(n=20, seed=2), {"density_seed": 17}),
    "term_volume_correction_20": lambda: (scenes.sloshing_tank(n=20, seed=2, tol=1e-6),
                                          {"volume": (1.05, 1.0), "gain": 1.0}),
    "term_warm_start_20": lambda: (scenes.training_scene(n=20, seed=9), {"warm_start": True, "tile": 16}),
}


def make_term(name: str, build) -> str:
    sc, opt = build()
    extra, density, tile, repeat = {}, None, 8, 1
    if "kappa" in opt:
        extra["HarnessSurfaceTension"] = repr(opt["kappa"])
    if "density_seed" in opt:
        density = _density(sc, opt["density_seed"])
    if "volume" in opt:
        extra["HarnessVolume"] = "%r:%r" % opt["volume"]
        extra["Gain"] = repr(opt["gain"])
    if opt.get("warm_start"):
        extra["WarmStart"] = "Yes"
        tile, repeat = opt["tile"], 2
    r = ref_runner.run_reference(sc, mode="mic0", tile_size=tile, repeat=repeat, extra=extra, density=density)
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
        rhs=r.system["rhs"], kappa=np.float64(opt.get("kappa", 0.0)),
        volume=np.array(opt.get("volume", (0.0, 0.0)), np.float64), gain=np.float64(opt.get("gain", 1.0)),
        warm_start=np.int32(bool(opt.get("warm_start"))), tile=np.int32(tile), repeat=np.int32(repeat),
    )
    if density is not None:
        payload.update(density_u=density[0], density_v=density[1], density_w=density[2])
    svel = sc.solid_velocity_effective()
    payload.update(us=svel[0], vs=svel[1], ws=svel[2])
    path = os.path.join(OUT, f"{name}.npz")
    np.savez_compressed(path, **payload)
    return path


# Velocity extension after the projection (macliquid3::extend_both,
# src/liquid/macliquid3.cpp:330-340): the reference's projected velocity, and
# the same after macarray_extrapolator3::extrapolate(width) and (when on)
# macutility3::constrain_velocity.
EXTEND_CASES = {
    "ext_sloshing_tank_24": lambda: (scenes.sloshing_tank(n=24, seed=1, tol=1e-6), 3, 1),
    "ext_dambreak_sphere_24": lambda: (scenes.dambreak_sphere(n=24, seed=7), 4, 1),
    "ext_splash_24": lambda: (scenes.splash(n=24, seed=4, spheres=12), 2, 0),
}


def make_extend(name: str, build) -> str:
    sc, width, constrain = build()
    r0 = ref_runner.run_reference(sc, mode="mic0", dump_system=False)
    r1 = ref_runner.run_reference(sc, mode="mic0", dump_system=False,
                                  extra={"HarnessExtend": width, "HarnessConstrain": constrain})
    payload = dict(
        shape=np.array([sc.nx, sc.ny, sc.nz], np.int32), dx=np.float64(sc.dx),
        width=np.int32(width), constrain=np.int32(constrain), has_solid=np.int32(sc.solid_phi is not None),
        solid=r0.solid.astype(np.float32), solid_active=r0.solid_active,
        u0=r0.velocity[0].astype(np.float32), v0=r0.velocity[1].astype(np.float32),
        w0=r0.velocity[2].astype(np.float32),
        u0_active=r0.velocity_active[0], v0_active=r0.velocity_active[1], w0_active=r0.velocity_active[2],
        u=r1.velocity[0].astype(np.float32), v=r1.velocity[1].astype(np.float32), w=r1.velocity[2].astype(np.float32),
        u_active=r1.velocity_active[0], v_active=r1.velocity_active[1], w_active=r1.velocity_active[2],
    )
    path = os.path.join(OUT, f"{name}.npz")
    np.savez_compressed(path, **payload)
    return path


# FLIP splat before the projection (macflipliquid3.cpp:135-151): seeded
# particles in the reference's record layout over a scene's grid velocity,
# and what macnbflip3::splat and the combined grid velocity make of them.
# name: scene, particles per liquid cell, bullet fraction, APIC, SplatBulletParticle
SPLAT_CASES = {
    "splat_dambreak_sphere_16": lambda: (scenes.dambreak_sphere(n=16, seed=3), 8, 0.02, True, False),
    "splat_sloshing_tank_16": lambda: (scenes.sloshing_tank(n=16, seed=2, tol=1e-6), 4, 0.05, False, True),
    "splat_splash_20": lambda: (scenes.splash(n=20, seed=4, spheres=8), 3, 0.10, True, True),
}


def make_splat(name: str, build) -> str:
    sc, per_cell, bullets, apic, splat_bullet = build()
    P = scenes.flip_particles(sc, per_cell=per_cell, seed=11, bullet_fraction=bullets)
    vel, vact = sc.velocity_effective(), [m.astype(np.uint8) for m in sc.velocity_active]
    r = ref_runner.run_reference_splat(sc.nx, sc.ny, sc.nz, sc.dx, P, vel, vact, apic=apic,
                                       splat_bullet=splat_bullet)
    payload = dict(shape=np.array([sc.nx, sc.ny, sc.nz], np.int32), dx=np.float64(sc.dx),
                   apic=np.int32(apic), splat_bullet=np.int32(splat_bullet),
                   particles=P.view(np.uint8).reshape(len(P), P.dtype.itemsize))
    for d, k in enumerate("uvw"):
        payload[k + "0"], payload[k + "0_active"] = vel[d], vact[d]
        payload[k], payload[k + "_active"] = r["velocity"][d], r["velocity_active"][d]
        payload[k + "_mass"], payload[k + "_momentum"] = r["mass"][d], r["momentum"][d]
        payload[k + "_splat_active"] = r["splat_active"][d]
    path = os.path.join(OUT, f"{name}.npz")
    np.savez_compressed(path, **payload)
    return path


def main():
    if not ref_runner.ref_available("float"):
        raise SystemExit("compiled reference not found: run `make -C oracle/ref` first")
    only = sys.argv[1:]
    for name, build in CASES.items():
        if only and name not in only:
            continue
        p = make(name, build)
        print(p, os.path.getsize(p))
    for name, build in TERM_CASES.items():
        if only and name not in only:
            continue
        p = make_term(name, build)
        print(p, os.path.getsize(p))
    for name, build in EXTEND_CASES.items():
        if only and name not in only:
            continue
        p = make_extend(name, build)
        print(p, os.path.getsize(p))
    for name, build in SPLAT_CASES.items():
        if only and name not in only:
            continue
        p = make_splat(name, build)
        print(p, os.path.getsize(p))


if __name__ == "__main__":
    main()
