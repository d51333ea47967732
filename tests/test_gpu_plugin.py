"""The Shiokaze modules loaded by the reference's own module loader inside the
compiled reference harnesses: libshiokaze_macpressuresolver3_b200.so
(Projection=macpressuresolver3_b200) against Projection=macpressuresolver3 on
the same grids, libshiokaze_pcg_b200.so (LinSolver=pcg_b200), and
libshiokaze_macnbflip3_b200.so (FLIP=macnbflip3_b200) against the reference
macnbflip3's splat. This is the drop-in path a Shiokaze user takes."""
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


@pytest.mark.skipif(not (ref_runner.ref_available("float") and os.path.exists(PLUGIN)),
                    reason="needs the compiled reference harness and the plugin (built where the reference is mounted)")
@pytest.mark.parametrize("term", ["surface_tension", "solid_density", "volume_correction", "warm_start"])
def test_plugin_optional_terms(term):
    """Each optional term through the module loader, against the reference module
    with the same harness keys."""
    sc = scenes.training_scene(n=24, seed=13) if term != "solid_density" else scenes.dambreak_sphere(n=24, seed=5)
    extra, density, tile, repeat = {}, None, 8, 1
    if term == "surface_tension":
        extra["HarnessSurfaceTension"] = "0.05"
    elif term == "solid_density":
        rng = np.random.default_rng(3)
        density = [rng.uniform(0, 1, s).astype(np.float32) for s in
                   [(sc.nz, sc.ny, sc.nx + 1), (sc.nz, sc.ny + 1, sc.nx), (sc.nz + 1, sc.ny, sc.nx)]]
    elif term == "volume_correction":
        extra.update({"HarnessVolume": "0.9:1.0", "Gain": "1.0"})
    else:
        extra["WarmStart"] = "Yes"
        tile, repeat = 16, 2
    ref = ref_runner.run_reference(sc, mode="mic0", dump_system=False, tile_size=tile, repeat=repeat, extra=extra,
                                   density=density)
    got = ref_runner.run_reference(sc, mode="mic0", dump_system=False, tile_size=tile, repeat=repeat,
                                   extra=dict(extra, Projection="macpressuresolver3_b200"), extra_libpath=[PKG],
                                   density=density)
    np.testing.assert_array_equal(got.pressure_active, ref.pressure_active)
    assert rel_inf(got.pressure, ref.pressure) <= 1e-5
    for d in range(3):
        np.testing.assert_array_equal(got.velocity_active[d], ref.velocity_active[d])
        assert rel_inf(got.velocity[d], ref.velocity[d]) <= 1e-5


PCG_PLUGIN = os.path.join(PKG, "libshiokaze_pcg_b200.so")


@pytest.mark.skipif(not (ref_runner.ref_available("float") and os.path.exists(PCG_PLUGIN)),
                    reason="needs the compiled reference harness and the pcg_b200 module")
@pytest.mark.parametrize("n,seed,tol", [(24, 1, 1e-4), (32, 2, 1e-6)])
def test_pcg_b200_matches_reference_pcg(n, seed, tol):
    """The reference's own macpressuresolver3 with LinSolver=pcg_b200 (our module,
    loaded by the reference's loader) against LinSolver=pcg (the reference's)."""
    sc = scenes.dambreak_sphere(n=n, seed=seed, tol=tol)
    ref = ref_runner.run_reference(sc, linsolver="pcg", dump_system=False)
    got = ref_runner.run_reference(sc, linsolver="pcg_b200", dump_system=False, extra_libpath=[PKG])
    (it_ref, rr_ref), (it_got, rr_got) = ref.console_solves[-1], got.console_solves[-1]
    # unpreconditioned CG: summation order alone moves the stop by 3-5 %
    assert abs(it_got - it_ref) <= max(2, int(0.05 * it_ref)), (it_got, it_ref)
    assert rr_got <= tol
    tol_p = max(1e-5, 10 * tol)
    np.testing.assert_array_equal(got.pressure_active, ref.pressure_active)
    assert rel_inf(got.pressure, ref.pressure) <= tol_p
    for d in range(3):
        np.testing.assert_array_equal(got.velocity_active[d], ref.velocity_active[d])
        assert rel_inf(got.velocity[d], ref.velocity[d]) <= tol_p


@pytest.mark.skipif(not (ref_runner.ref_available("float") and os.path.exists(PCG_PLUGIN)),
                    reason="needs the compiled reference harness and the pcg_b200 module")
@pytest.mark.parametrize("n,seed,tol", [(24, 7, 1e-4), (32, 2, 1e-6)])
def test_streamfunc_projection_runs_on_pcg_b200(n, seed, tol):
    """The reference's other projection, macstreamfuncsolver3 (a vector-potential
    solve, src/projection/macstreamfuncsolver3.cpp), takes its linear solver
    from the same LinSolver plugin: with LinSolver=pcg_b200 its solves run on
    the GPU, and its projected velocity matches the one it gets from the
    reference's pcg."""
    sc = scenes.dambreak_sphere(n=n, seed=seed, tol=tol)
    extra = {"Projection": "macstreamfuncsolver3"}
    ref = ref_runner.run_reference(sc, linsolver="pcg", dump_system=False, extra=extra)
    got = ref_runner.run_reference(sc, linsolver="pcg_b200", dump_system=False, extra=extra, extra_libpath=[PKG])
    vin = sc.velocity_effective()
    tol_v = max(1e-5, 10 * tol)
    for d in range(3):
        np.testing.assert_array_equal(got.velocity_active[d], ref.velocity_active[d])
        # the projection did change the field, and both solvers agree on it
        m = ref.velocity_active[d] != 0
        assert np.abs(ref.velocity[d][m] - vin[d][m]).max() > 1e-2
        assert rel_inf(got.velocity[d], ref.velocity[d]) <= tol_v, (d, rel_inf(got.velocity[d], ref.velocity[d]))


@pytest.mark.skipif(not (ref_runner.ref_available("float") and os.path.exists(PCG_PLUGIN)),
                    reason="needs the compiled reference harness and the pcg_b200 module")
@pytest.mark.parametrize("projection", ["macpressuresolver3", "macstreamfuncsolver3"])
def test_pcg_b200_mic0_matches_reference_mic0(projection):
    """LinSolver=pcg_b200 with B200.Preconditioner=mic0 (the generic-matrix
    MIC(0) on the device) against the reference's own PCG loop with its
    header's MIC(0) applied (LinSolver=refmic0, RefMode=mic0), under both
    projections that solve through the LinSolver plugin."""
    sc = scenes.dambreak_sphere(n=24, seed=3, tol=1e-6)
    extra = {"Projection": projection}
    ref = ref_runner.run_reference(sc, linsolver="refmic0", mode="mic0", dump_system=False, extra=extra)
    got = ref_runner.run_reference(sc, linsolver="pcg_b200", dump_system=False,
                                   extra=dict(extra, **{"B200.Preconditioner": "mic0"}), extra_libpath=[PKG])
    # each projection's own console line per solve: "Took N iterations" (then ", Reresid" or ". Reresid")
    import re
    its_ref = [int(c) for c in re.findall(r"Took (\d+) iterations", ref.stdout)]
    its_got = [int(c) for c in re.findall(r"Took (\d+) iterations", got.stdout)]
    assert len(its_got) == len(its_ref) > 0, (its_got, its_ref)
    # The pressure system stops within 2 %. The stream-function system needs
    # about twice the iterations and stops 3 % from the reference (303 against
    # 313 at this scene); its bar is the 5 % that the dot products' summation
    # order alone needs for unpreconditioned CG on the pressure system
    # (test_pcg_b200_matches_reference_pcg).
    spread = 0.02 if projection == "macpressuresolver3" else 0.05
    for a, b in zip(its_got, its_ref):
        assert abs(a - b) <= max(1, int(spread * b)), (its_got, its_ref)
    for d in range(3):
        np.testing.assert_array_equal(got.velocity_active[d], ref.velocity_active[d])
        assert rel_inf(got.velocity[d], ref.velocity[d]) <= 1e-5, (d, rel_inf(got.velocity[d], ref.velocity[d]))


FLIP_PLUGIN = os.path.join(PKG, "libshiokaze_macnbflip3_b200.so")


@pytest.mark.skipif(not (os.path.exists(os.path.join(ref_runner.REF_DIR, "float", "shkz_ref_splat"))
                         and os.path.exists(FLIP_PLUGIN)),
                    reason="needs the compiled reference splat harness and the FLIP module")
def test_flip_module_splat_matches_reference(golden_splat):
    """FLIP=macnbflip3_b200 loaded by the reference's module loader, its
    particles handed over by the reference's own serialisation, splatting
    through macflip3_interface::splat: the splat grid and the combined
    velocity are bit-identical to the reference macnbflip3's."""
    from conftest import splat_particles
    from test_oracle_splat import assert_bitexact, reference_outputs
    name, g = golden_splat
    nx, ny, nz = (int(v) for v in g["shape"])
    r = ref_runner.run_reference_splat(nx, ny, nz, float(g["dx"]), splat_particles(g), [g["u0"], g["v0"], g["w0"]],
                                       [g["u0_active"], g["v0_active"], g["w0_active"]], apic=bool(g["apic"]),
                                       splat_bullet=bool(g["splat_bullet"]), module="macnbflip3_b200",
                                       extra_libpath=[PKG])
    got = [r[k] for k in ("velocity", "velocity_active", "mass", "momentum", "splat_active")]
    assert_bitexact(got, reference_outputs(g))
