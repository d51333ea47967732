"""The CPU restatement of the velocity extension after a projection
(oracle/extend.py: macarray_extrapolator3::extrapolate + constrain_velocity)
against the reference: bit-exact on the committed fixtures, and against the
compiled reference itself where it is built."""
import numpy as np
import pytest

from oracle import extend as ext
from oracle import ref_runner


def _inputs(g):
    vel = [g["u0"], g["v0"], g["w0"]]
    act = [g["u0_active"], g["v0_active"], g["w0_active"]]
    solid = g["solid"] if int(g["has_solid"]) else None
    sact = g["solid_active"] if int(g["has_solid"]) else None
    return vel, act, solid, sact


def assert_same_extension(v, a, want_v, want_a):
    for d in range(3):
        assert np.array_equal(np.asarray(a[d]).astype(bool), np.asarray(want_a[d]).astype(bool)), f"mask {d}"
        m = np.asarray(want_a[d]).astype(bool)
        got = np.asarray(v[d], np.float32)[m].view(np.uint32)
        want = np.asarray(want_v[d], np.float32)[m].view(np.uint32)
        assert np.array_equal(got, want), f"values {d}: {int(np.sum(got != want))} differ"


def test_oracle_extension_matches_reference_fixtures(golden_ext):
    name, g = golden_ext
    vel, act, solid, sact = _inputs(g)
    v, a = ext.extend(vel, act, solid, sact, float(g["dx"]), int(g["width"]), bool(g["constrain"]))
    assert_same_extension(v, a, [g["u"], g["v"], g["w"]], [g["u_active"], g["v_active"], g["w_active"]])
    # the extension grew every component and left the projected faces' masks on
    for d, key in enumerate("uvw"):
        assert g[key + "_active"].sum() > g[key + "0_active"].sum()
        assert np.all(g[key + "_active"][g[key + "0_active"] != 0])


@pytest.mark.skipif(not ref_runner.ref_available("float"), reason="compiled reference not built here")
@pytest.mark.parametrize("width,constrain", [(1, 1), (5, 1), (3, 0)])
def test_oracle_extension_matches_compiled_reference(width, constrain):
    from shiokaze_b200 import scenes
    sc = scenes.sloshing_tank(n=32, seed=3, tol=1e-6)
    r0 = ref_runner.run_reference(sc, dump_system=False)
    r1 = ref_runner.run_reference(sc, dump_system=False, extra={"HarnessExtend": width, "HarnessConstrain": constrain})
    v, a = ext.extend(r0.velocity, r0.velocity_active, r0.solid.astype(np.float32), r0.solid_active, sc.dx,
                      width, bool(constrain))
    assert_same_extension(v, a, r1.velocity, r1.velocity_active)


def test_oracle_extension_full_size_digest():
    """The 256^3 tank's input velocity extended 3 passes and constrained (no
    projection before it): the CPU restatement hashes to the digest of the
    compiled reference's result (tests/golden/make_full_size.py)."""
    import json
    import os
    from conftest import GOLDEN
    from golden.make_full_size import EXTEND_WIDTH, extend_digest
    from shiokaze_b200 import scenes
    ref = json.load(open(os.path.join(GOLDEN, "full_size_reference.json")))["extend_sloshing_tank_256"]
    sc = scenes.sloshing_tank(n=256, seed=0, tol=1e-6)
    v, a = ext.extend(sc.velocity_effective(), [m.astype(np.uint8) for m in sc.velocity_active],
                      sc.solid_effective(), sc.solid_active, sc.dx, EXTEND_WIDTH, True)
    assert sum(int(np.asarray(m).sum()) for m in a) == ref["active_faces"]
    assert extend_digest(v, a) == ref["extend_digest"]
