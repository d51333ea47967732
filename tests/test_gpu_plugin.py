"""The Shiokaze module libshiokaze_macpressuresolver3_b200.so loaded by the
reference's own module loader (Projection=macpressuresolver3_b200) inside the
compiled reference harness, against Projection=macpressuresolver3 on the same
grids. This is the drop-in path a Shiokaze user takes."""
import os

import numpy as np
import pytest

from oracle import ref_runner
from shiokaze_b200 import scenes

pytestmark = pytest.mark.gpu

PKG = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "shiokaze_b200")
PLUGIN = os.path.join(PKG, "libshiokaze_macpressuresolver3_b200.so")


def rel_inf(a, b):
    den = np.abs(b).max()
    return float(np.abs(a - b).max() / (den if den else 1.0))


@pytest.mark.skipif(not (ref_runner.ref_available("float") and os.path.exists(PLUGIN)),
                    reason="needs the compiled reference harness and the plugin (built where the reference is mounted)")
@pytest.mark.parametrize("n,seed", [(32, 1), (48, 2)])
def test_plugin_matches_reference_module(n, seed):
    sc = scenes.dambreak_sphere(n=n, seed=seed, solid_velocity=(seed == 2))
    ref = ref_runner.run_reference(sc, mode="mic0", dump_system=False, linsolver="refmic0")
    got = ref_runner.run_reference(sc, mode="mic0", dump_system=False,
                                   extra={"Projection": "macpressuresolver3_b200"}, extra_libpath=[PKG])
    np.testing.assert_array_equal(got.pressure_active, ref.pressure_active)
    assert rel_inf(got.pressure, ref.pressure) <= 1e-5
    for d in range(3):
        np.testing.assert_array_equal(got.velocity_active[d], ref.velocity_active[d])
        assert rel_inf(got.velocity[d], ref.velocity[d]) <= 1e-5
