"""Record the compiled reference's results on the full-size configurations
into ``full_size_reference.json``, for the full-size GPU tests, which cannot
run the reference themselves in the time a test has:

* iteration counts of MIC(0)-PCG to 1e-6 (sloshing tank 256^3, splash 384^3);
* the FLIP splat of the splat benchmark's workload (sloshing tank 256^3,
  2.4 M particles in the 3-cell narrow band): a SHA-256 of its outputs
  (``splat_digest``), so the device result can be compared bit for bit;
* the velocity extension (3 passes + constrain_velocity) of the 256^3 tank's
  input velocity, without a projection: a SHA-256 of the extended velocity
  and masks (``extend_digest``).

Runs the reference's own ``macpressuresolver3::project`` (built by
``oracle/ref/Makefile`` into ``oracle/_ref``); needs the reference sources,
so it only runs where they are mounted. Takes a few minutes.

    python tests/golden/make_full_size.py [name ...]    # only the named entries
"""
from __future__ import annotations

import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from shiokaze_b200 import scenes  # noqa: E402
from oracle import ref_runner  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "full_size_reference.json")

def splat_digest(velocity, velocity_active, mass, momentum, splat_active) -> str:
    """SHA-256 over the splat's outputs, axis by axis: mass, momentum (float32),
    splat_active (uint8), velocity (float32), velocity_active (uint8)."""
    import hashlib
    import numpy as np
    h = hashlib.sha256()
    for d in range(3):
        for a, dt in ((mass[d], np.float32), (momentum[d], np.float32), (splat_active[d], np.uint8),
                      (velocity[d], np.float32), (velocity_active[d], np.uint8)):
            h.update(np.ascontiguousarray(a, dt).tobytes())
    return h.hexdigest()


def extend_digest(velocity, velocity_active) -> str:
    """SHA-256 over the extended field, axis by axis: values (float32, only
    where active) and masks (uint8)."""
    import hashlib
    import numpy as np
    h = hashlib.sha256()
    for d in range(3):
        m = np.ascontiguousarray(velocity_active[d], np.uint8)
        v = np.where(m != 0, np.asarray(velocity[d], np.float32), np.float32(0))
        h.update(np.ascontiguousarray(v, np.float32).tobytes())
        h.update(m.tobytes())
    return h.hexdigest()


EXTEND_WIDTH = 3


def splat_case():
    sc = scenes.sloshing_tank(n=256, seed=0, tol=1e-6)
    return sc, scenes.flip_particles(sc, per_cell=8, seed=0, band=3.0)


CASES = {
    "sloshing_tank_256": lambda: scenes.sloshing_tank(n=256, seed=0, tol=1e-6),
    "splash_384": lambda: scenes.splash(n=384, seed=0, tol=1e-6),
}


def main():
    if not ref_runner.ref_available("float"):
        raise SystemExit("compiled reference not found: run `make -C oracle/ref` first")
    import numpy as np
    only = sys.argv[1:]
    out = json.load(open(OUT)) if os.path.exists(OUT) else {}
    if not only or "splat_sloshing_tank_256" in only:
        sc, P = splat_case()
        r = ref_runner.run_reference_splat(sc.nx, sc.ny, sc.nz, sc.dx, P, sc.velocity_effective(),
                                           [m.astype(np.uint8) for m in sc.velocity_active])
        out["splat_sloshing_tank_256"] = {
            "particles": int(len(P)), "splatted_faces": int(sum(int(a.sum()) for a in r["splat_active"])),
            "splat_digest": splat_digest(r["velocity"], r["velocity_active"], r["mass"], r["momentum"],
                                         r["splat_active"])}
        print("splat_sloshing_tank_256", out["splat_sloshing_tank_256"], flush=True)
    if not only or "extend_sloshing_tank_256" in only:
        sc = scenes.sloshing_tank(n=256, seed=0, tol=1e-6)
        r = ref_runner.run_reference(sc, mode="mic0", dump_system=False,
                                     extra={"HarnessProject": 0, "HarnessExtend": EXTEND_WIDTH, "HarnessConstrain": 1})
        out["extend_sloshing_tank_256"] = {
            "width": EXTEND_WIDTH, "constrain": 1,
            "active_faces": int(sum(int(np.asarray(a).sum()) for a in r.velocity_active)),
            "extend_digest": extend_digest([np.asarray(v, np.float32) for v in r.velocity], r.velocity_active)}
        print("extend_sloshing_tank_256", out["extend_sloshing_tank_256"], flush=True)
    for name, build in CASES.items():
        if only and name not in only:
            continue
        sc = build()
        r = ref_runner.run_reference(sc, mode="mic0", dump_system=False)
        it, rr = r.console_solves[-1]
        out[name] = {"iterations": int(it), "reresid": float(rr), "unknowns": int(r.pressure_active.sum()),
                     "tol": float(sc.tol), "projection_ms": float(r.projection_ms)}
        print(name, out[name], flush=True)
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
