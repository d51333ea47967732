"""The CPU restatement of the FLIP splat (shkzo_splat: macnbflip3::splat over
the pointgridhash3 edge hash, then macflipliquid3's combined grid velocity)
against fixtures written by the compiled reference: bit-exact."""
import numpy as np

from conftest import splat_particles
from oracle import oracle
from shiokaze_b200 import scenes

KEYS = ("velocity", "velocity_active", "mass", "momentum", "splat_active")


def reference_outputs(g):
    return {"velocity": [g["u"], g["v"], g["w"]],
            "velocity_active": [g["u_active"], g["v_active"], g["w_active"]],
            "mass": [g["u_mass"], g["v_mass"], g["w_mass"]],
            "momentum": [g["u_momentum"], g["v_momentum"], g["w_momentum"]],
            "splat_active": [g["u_splat_active"], g["v_splat_active"], g["w_splat_active"]]}


def assert_bitexact(got, want):
    for key, arrs in zip(KEYS, got):
        for d in range(3):
            a, b = np.asarray(arrs[d]), np.asarray(want[key][d])
            if a.dtype == np.float32:
                a, b = a.view(np.uint32), b.astype(np.float32).view(np.uint32)
            assert np.array_equal(a, b), f"{key}[{d}]: {int(np.sum(a != b))} differ"


def test_oracle_splat_matches_reference(golden_splat):
    name, g = golden_splat
    nx, ny, nz = (int(v) for v in g["shape"])
    P = splat_particles(g)
    got = oracle.splat(nx, ny, nz, float(g["dx"]), P, [g["u0"], g["v0"], g["w0"]],
                       [g["u0_active"], g["v0_active"], g["w0_active"]], apic=bool(g["apic"]),
                       splat_bullet=bool(g["splat_bullet"]))
    assert_bitexact(got, reference_outputs(g))
    # the fixtures cover faces the splat switched on, faces it left inactive
    # (zero mass) and bullets skipped or splatted
    assert sum(int(np.sum(g[k + "_splat_active"])) for k in "uvw") > 0
    assert int(np.sum(P["bullet"])) > 0


def test_single_particle_counts_twice():
    """A particle at a face centre has tent weight 1 there; the neighbour
    query visits its bucket twice (pointgridhash3.cpp:218-231), so the face
    receives twice its mass and momentum, and the combined velocity on a face
    the grid held inactive is the particle's own."""
    sc = scenes.dambreak_sphere(n=8, seed=0)
    nx, ny, nz, dx = sc.nx, sc.ny, sc.nz, sc.dx
    P = np.zeros(1, scenes.PARTICLE_DTYPE)
    P["p"] = np.array([3 * dx, 2.5 * dx, 4.5 * dx], np.float32)  # centre of u-face (3, 2, 4)
    P["velocity"] = np.array([0.75, -0.5, 0.25], np.float32)
    P["mass"] = np.float32(0.125)
    vel = [np.zeros_like(u) for u in sc.velocity]
    act = [np.zeros_like(m, dtype=np.uint8) for m in sc.velocity_active]
    v, a, mass, mom, sact = oracle.splat(nx, ny, nz, dx, P, vel, act, apic=False)
    assert mass[0][4, 2, 3] == np.float32(0.25)
    assert mom[0][4, 2, 3] == np.float32(2 * 0.125 * 0.75)
    assert v[0][4, 2, 3] == np.float32(0.75) and a[0][4, 2, 3] == 1


def test_empty_particle_set_leaves_velocity():
    sc = scenes.dambreak_sphere(n=8, seed=0)
    P = np.zeros(0, scenes.PARTICLE_DTYPE)
    vel = sc.velocity_effective()
    act = [m.astype(np.uint8) for m in sc.velocity_active]
    v, a, mass, mom, sact = oracle.splat(sc.nx, sc.ny, sc.nz, sc.dx, P, vel, act)
    for d in range(3):
        assert np.array_equal(v[d].view(np.uint32), vel[d].view(np.uint32))
        assert np.array_equal(a[d], act[d])
        assert not sact[d].any()


def test_particle_layout_is_the_reference_record():
    """84-byte records, fields at the offsets of macnbflip3::Particle."""
    dt = scenes.PARTICLE_DTYPE
    assert dt.itemsize == 84
    assert [dt.fields[k][1] for k in ("p", "c", "velocity", "mass", "r", "bullet", "bullet_time",
                                      "sizing_value", "live_count")] == [0, 12, 48, 60, 64, 68, 72, 76, 80]


def test_narrow_band_particles():
    """With a band, particles sit only where the analytic level set is within
    band cells of the surface."""
    sc = scenes.sloshing_tank(n=32, seed=0)
    full = scenes.flip_particles(sc, per_cell=2, seed=0, edge_cases=False)
    band = scenes.flip_particles(sc, per_cell=2, seed=0, edge_cases=False, band=3.0)
    assert 0 < len(band) < len(full)


def test_oracle_splat_full_size_digest():
    """The splat benchmark's workload (256^3 tank, 2.4 M particles in the
    3-cell band): the CPU restatement's outputs hash to the digest the
    compiled reference's outputs were recorded with (tests/golden/
    make_full_size.py)."""
    import json
    from conftest import GOLDEN
    from golden.make_full_size import splat_case, splat_digest
    import os
    ref = json.load(open(os.path.join(GOLDEN, "full_size_reference.json")))["splat_sloshing_tank_256"]
    sc, P = splat_case()
    assert len(P) == ref["particles"]
    v, a, mass, mom, sact = oracle.splat(sc.nx, sc.ny, sc.nz, sc.dx, P, sc.velocity_effective(),
                                         [m.astype(np.uint8) for m in sc.velocity_active])
    assert sum(int(s.sum()) for s in sact) == ref["splatted_faces"]
    assert splat_digest(v, a, mass, mom, sact) == ref["splat_digest"]


def test_harness_module_path_reproduces_compiled_in_splat():
    """The harness's FLIP=<module> path (particles handed to a module loaded
    by the reference's loader through the reference's own serialisation, then
    macflip3_interface::splat), run with the reference's own macnbflip3
    module, gives exactly the compiled-in splat: the path the GPU module is
    tested through adds nothing of its own."""
    import os
    import pytest
    from oracle import ref_runner
    if not os.path.exists(os.path.join(ref_runner.REF_DIR, "float", "libshiokaze_macnbflip3.so")):
        pytest.skip("reference macnbflip3 module not built (needs the reference sources)")
    sc = scenes.splash(n=20, seed=1, spheres=6)
    P = scenes.flip_particles(sc, per_cell=3, seed=4, bullet_fraction=0.1)
    args = (sc.nx, sc.ny, sc.nz, sc.dx, P, sc.velocity_effective(), [m.astype(np.uint8) for m in sc.velocity_active])
    a = ref_runner.run_reference_splat(*args)
    b = ref_runner.run_reference_splat(*args, module="macnbflip3")
    for key in KEYS:
        for d in range(3):
            assert np.array_equal(np.asarray(a[key][d]).view(np.uint8), np.asarray(b[key][d]).view(np.uint8)), key
