"""The reference's own known-answer test for the projection, on the oracle.

src/examples/accuracytest3-example.cpp:68-139 projects u = grad |x - c|^2 with
dt = 1 inside a liquid sphere of radius r around c = (0.5, 0.5, 0.5) (a level
set banded at 2 dx, no solid, EpsFluid = 1e-18): div u = 6, so the exact
pressure is |x - c|^2 - r^2, zero on the free surface. It perturbs r over
2 * TrialCount + 1 values spaced sqrt(3) dx / TrialCount apart, takes the
largest infinity-norm error of the pressure on the unknown cells, and reports
the order between successive grid doublings, about 2 for the ghost-fluid free
surface. The reference ships no recorded numbers, so the test holds the order
(>= 1.5 at each doubling) and the error levels of this restatement, which is
bit-exact against the compiled reference (tests/test_oracle.py)."""
import math

import numpy as np

from oracle import oracle
from shiokaze_b200 import scenes

TRIALS = 2  # TrialCount: radii r0 + q sqrt(3) dx / TRIALS for q = -TRIALS..TRIALS
R0 = 0.4    # the example's default Radius


def worst_error(n, project):
    """Largest infinity-norm pressure error over the example's radii at n^3;
    project(scene) returns (pressure, unknown mask)."""
    dx = 1.0 / n
    worst = 0.0
    for q in range(-TRIALS, TRIALS + 1):
        sc, exact = scenes.analytic_sphere(n, R0 + math.sqrt(3.0) * dx / TRIALS * q)
        p, mask = project(sc)
        m = mask.astype(bool)
        assert m.any()
        worst = max(worst, float(np.abs(p[m].astype(np.float64) - exact[m]).max()))
    return worst


def oracle_project(sc):
    o = oracle.project(sc, tol=1e-12, eps_fluid=1e-18)
    return o.pressure, o.pressure_active


def test_oracle_second_order_on_the_reference_accuracy_test():
    e = {n: worst_error(n, oracle_project) for n in (16, 32, 64)}
    orders = [math.log2(e[16] / e[32]), math.log2(e[32] / e[64])]
    print(f"\nworst errors {e}, orders {orders}")
    assert all(o >= 1.5 for o in orders), (e, orders)
    # error levels of the restatement (6.8e-4, 2.0e-4, 5.1e-5): the pressure is
    # a few dx^2 from the exact one
    for n, v in e.items():
        assert v <= 0.5 / (n * n), (n, v)
