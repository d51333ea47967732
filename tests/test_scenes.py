"""Scene generator: determinism and the narrow-band conventions."""
import numpy as np

from shiokaze_b200 import scenes


def test_seeded_scenes_are_deterministic():
    a = scenes.dambreak_sphere(n=16, seed=3)
    b = scenes.dambreak_sphere(n=16, seed=3)
    np.testing.assert_array_equal(a.fluid_phi, b.fluid_phi)
    for u, v in zip(a.velocity, b.velocity):
        np.testing.assert_array_equal(u, v)
    c = scenes.dambreak_sphere(n=16, seed=4)
    assert not np.array_equal(a.velocity[0], c.velocity[0])


def test_band_and_effective_values():
    sc = scenes.sloshing_tank(n=32, seed=1)
    band = np.float32(sc.fluid_band)
    eff = sc.fluid_effective()
    act = sc.fluid_active.astype(bool)
    assert (np.abs(sc.fluid_phi[act].astype(np.float64)) < sc.fluid_band).all()
    assert set(np.unique(eff[~act])) <= {band, -band}
    assert np.array_equal(eff[act], sc.fluid_phi[act])


def test_scene_shapes():
    sc = scenes.splash(n=24, seed=1, spheres=5)
    assert sc.fluid_phi.shape == (24, 24, 24)
    assert sc.velocity[0].shape == (24, 24, 25)
    assert sc.velocity[1].shape == (24, 25, 24)
    assert sc.velocity[2].shape == (25, 24, 24)
