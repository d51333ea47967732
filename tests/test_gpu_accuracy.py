"""The reference's known-answer test for the projection (accuracytest3:
src/examples/accuracytest3-example.cpp:68-139) on the device: u = grad |x - c|^2,
dt = 1, a liquid sphere of radius r (band 2 dx, no solid, EpsFluid = 1e-18),
exact pressure |x - c|^2 - r^2. The device's largest error over the example's
radii falls at second order with each grid doubling up to 128^3 and equals the
oracle's (tests/test_oracle_accuracy.py) where both run."""
import math

import pytest

from test_oracle_accuracy import oracle_project, worst_error

pytestmark = pytest.mark.gpu


def device_project(sc):
    from shiokaze_b200.projection import MacPressureSolver3, grids_from_scene
    s = MacPressureSolver3({"Residual": 1e-9, "EpsFluid": 1e-18})
    s.initialize((sc.nx, sc.ny, sc.nz), sc.dx)
    vel, solid, svel, fluid = grids_from_scene(sc)
    res = s.project(sc.dt, vel, solid, svel, fluid)
    assert res["status"] == 0, res
    p = s.get_pressure()
    return p.values.copy(), p.active.copy()


def test_device_second_order_on_the_reference_accuracy_test():
    e = {n: worst_error(n, device_project) for n in (16, 32, 64, 128)}
    orders = [math.log2(e[a] / e[b]) for a, b in ((16, 32), (32, 64), (64, 128))]
    print(f"\nworst errors {e}, orders {orders}")
    assert all(o >= 1.5 for o in orders), (e, orders)
    for n in (16, 32, 64):
        eo = worst_error(n, oracle_project)
        assert abs(e[n] - eo) <= 0.01 * eo, (n, e[n], eo)
