"""Record the compiled reference's iteration counts on the full-size
configurations (sloshing tank 256^3, splash 384^3: MIC(0)-PCG to 1e-6) into
``full_size_reference.json``, for the full-size GPU tests, which cannot run
the reference themselves in the time a test has.

Runs the reference's own ``macpressuresolver3::project`` (built by
``oracle/ref/Makefile`` into ``oracle/_ref``); needs the reference sources,
so it only runs where they are mounted. Takes a few minutes.

    python tests/golden/make_full_size.py
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

CASES = {
    "sloshing_tank_256": lambda: scenes.sloshing_tank(n=256, seed=0, tol=1e-6),
    "splash_384": lambda: scenes.splash(n=384, seed=0, tol=1e-6),
}


def main():
    if not ref_runner.ref_available("float"):
        raise SystemExit("compiled reference not found: run `make -C oracle/ref` first")
    out = {}
    for name, build in CASES.items():
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
