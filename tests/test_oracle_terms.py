"""The CPU oracle's optional projection terms against the compiled reference.

Fixtures ``tests/golden/term_*.npz`` come from the reference's own
macpressuresolver3 with one term switched on (make_golden.py): surface
tension (macpressuresolver3.cpp:98-128), solid density (:75-80, 286-293),
PI volume correction (:219-234) and warm start with the default tile edge 16
(:236-259). Masks are bit-exact; pressure and velocities within 1e-5 of the
reference's infinity norm; MIC(0) iterations within max(1, 2 %).
"""
import numpy as np

from conftest import GoldenScene, term_options
from oracle import oracle

PARITY_TOL = 1e-5


def rel_inf(a, b):
    den = np.abs(b).max()
    return float(np.abs(a.astype(np.float64) - b.astype(np.float64)).max() / (den if den else 1.0))


def oracle_run(sc, opt):
    kw = dict(tol=sc.tol, tile=opt["tile"], surface_tension_kappa=opt.get("kappa", 0.0),
              density=opt.get("density"), volume=opt.get("volume"))
    if opt.get("warm_start"):
        prev = None
        for _ in range(opt["repeat"]):
            res = oracle.project(sc, warm_start=True, warm_prev=prev, **kw)
            prev = res.warm_prev
        return res
    return oracle.project(sc, **kw)


def test_oracle_terms_match_reference(golden_term):
    name, g = golden_term
    sc = GoldenScene(g)
    opt = term_options(g)
    res = oracle_run(sc, opt)
    np.testing.assert_array_equal(res.pressure_active, g["pressure_active"])
    for d, k in enumerate("uvw"):
        np.testing.assert_array_equal(res.velocity_active[d], g[k + "_active"])
    # the rhs the reference solved last (after the correction / warm-start shift)
    if not opt.get("warm_start"):
        np.testing.assert_array_equal(res.system.rhs, g["rhs"])
    else:
        assert np.abs(res.system.rhs - g["rhs"]).max() <= 1e-3 * np.abs(g["rhs"]).max() + 1e-12
    it_ref = int(g["iterations_mic0"])
    assert abs(res.iterations - it_ref) <= max(1, int(0.02 * it_ref)), (res.iterations, it_ref)
    assert rel_inf(res.pressure, g["pressure"]) <= PARITY_TOL
    for d, k in enumerate("uvw"):
        assert rel_inf(res.velocity[d], g[k]) <= PARITY_TOL, k


def test_terms_change_the_result(golden_term):
    """Each fixture's term matters: without it the reference answer is missed."""
    name, g = golden_term
    sc = GoldenScene(g)
    opt = term_options(g)
    if opt.get("warm_start"):
        return  # warm start changes the path, not the solution
    plain = oracle.project(sc, tol=sc.tol, tile=opt["tile"])
    assert rel_inf(plain.pressure, g["pressure"]) > 10 * PARITY_TOL or any(
        rel_inf(plain.velocity[d], g[k]) > 10 * PARITY_TOL for d, k in enumerate("uvw"))
