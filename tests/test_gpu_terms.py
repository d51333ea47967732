"""Optional projection terms on the GPU against the compiled reference.

Fixtures ``tests/golden/term_*.npz`` (make_golden.py) hold the reference's
macpressuresolver3 run with surface tension, solid density, PI volume
correction or warm start switched on. Bars as for the plain projection:
masks and (single-projection cases) the FP64 rhs bit-exact, pressure and
velocities within 1e-5 of the reference's infinity norm, MIC(0) iterations
within max(1, 2 %). The warm-start numbering (tiles of edge T in x-fastest
order, x fastest inside a tile) is checked directly against the oracle's
numbering for several tile edges.
"""
import numpy as np
import pytest

from conftest import GoldenScene, term_options
from oracle import oracle

pytestmark = pytest.mark.gpu

PARITY_TOL = 1e-5


def rel_inf(a, b):
    den = np.abs(b).max()
    return float(np.abs(a.astype(np.float64) - b.astype(np.float64)).max() / (den if den else 1.0))


def make_solver(sc, **cfg):
    from shiokaze_b200.projection import MacPressureSolver3
    s = MacPressureSolver3(cfg)
    s.initialize((sc.nx, sc.ny, sc.nz), sc.dx)
    return s


def project(s, sc, kappa=0.0):
    from shiokaze_b200.projection import grids_from_scene
    vel, solid, svel, fluid = grids_from_scene(sc)
    res = s.project(sc.dt, vel, solid, svel, fluid, surface_tension=kappa)
    return res, vel


def test_terms_match_reference(golden_term):
    name, g = golden_term
    sc = GoldenScene(g)
    opt = term_options(g)
    cfg = {"Residual": sc.tol, "TileSize": opt["tile"]}
    if opt.get("warm_start"):
        cfg["WarmStart"] = True
    if "volume" in opt:
        cfg["Gain"] = opt["volume"][3]
    s = make_solver(sc, **cfg)
    if "density" in opt:
        s.set_solid_density(opt["density"])
    for _ in range(opt["repeat"]):
        if "volume" in opt:
            s.set_target_volume(opt["volume"][0], opt["volume"][1])
        res, vel = project(s, sc, opt.get("kappa", 0.0))
        assert res["status"] == 0, res
    p = s.get_pressure()
    np.testing.assert_array_equal(p.active, g["pressure_active"])
    for d, k in enumerate("uvw"):
        np.testing.assert_array_equal(vel.active[d], g[k + "_active"])
    it_ref = int(g["iterations_mic0"])
    if opt.get("warm_start"):
        # the second solve starts from each side's own first solution
        assert res["iterations"] <= it_ref + max(3, it_ref // 2), (res["iterations"], it_ref)
    else:
        assert abs(res["iterations"] - it_ref) <= max(1, int(0.02 * it_ref)), (res["iterations"], it_ref)
        idx = oracle.assemble(sc, *oracle.fractions(sc, density=opt.get("density"))).index
        mask = idx >= 0
        rhs = s.inspect(5)
        np.testing.assert_array_equal(rhs[mask], g["rhs"][idx[mask]])
    assert rel_inf(p.values, g["pressure"]) <= PARITY_TOL
    for d, k in enumerate("uvw"):
        assert rel_inf(vel.values[d], g[k]) <= PARITY_TOL, (k, rel_inf(vel.values[d], g[k]))
    if "volume" in opt:
        assert res["volume_rhs_correct"] != 0.0


@pytest.mark.parametrize("tile", [8, 12, 16])
def test_warm_start_numbering(tile):
    """b - A x0 with x0 read through the reference's unknown numbering, and the
    stored vector written back by the same numbering."""
    from shiokaze_b200 import scenes
    sc = scenes.training_scene(n=28, seed=4)
    s = make_solver(sc, **{"Residual": 1e-6, "WarmStart": True, "TileSize": tile})
    area, rho = oracle.fractions(sc)
    S = oracle.assemble(sc, area, rho, tile=tile)
    rng = np.random.default_rng(tile)
    prev = rng.standard_normal(S.n + 5)  # longer than needed: the tail is dropped
    s.set_warm_start_vector(prev)
    res, _ = project(s, sc)
    assert res["status"] == 0
    mask = S.index >= 0
    want = S.rhs - oracle.spmv(S, prev[:S.n])
    got = s.inspect(5)[mask]
    order = S.index[mask]
    assert np.abs(got - want[order]).max() <= 1e-12 * max(1.0, np.abs(want).max())
    x64 = s.inspect(6)
    new = s.warm_start_vector()
    assert new.size == S.n
    np.testing.assert_array_equal(new[order], x64[mask])


def test_volume_state_round_trip():
    from shiokaze_b200 import scenes
    sc = scenes.sloshing_tank(n=24, seed=1, tol=1e-6)
    s = make_solver(sc, **{"Residual": 1e-6, "Gain": 1.0})
    s.set_target_volume(1.1, 1.0)
    r1, _ = project(s, sc)
    st = s.serialize()
    want, y = oracle.volume_correction(1, sc.dt, 1.1, 1.0, 0.0, 1.0)
    assert r1["volume_rhs_correct"] == want
    assert st["y_prev"] == y
    s2 = make_solver(sc, **{"Residual": 1e-6, "Gain": 1.0})
    s2.initialize_from(st)
    r2, _ = project(s2, sc)
    r1b, _ = project(s, sc)
    assert r2["volume_rhs_correct"] == r1b["volume_rhs_correct"]
