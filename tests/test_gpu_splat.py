"""FLIP splat before the projection on the device (shkz_b200_splat_host /
_device: macnbflip3::splat over the pointgridhash3 edge hash, then
macflipliquid3's combined grid velocity) against the reference: bit-exact,
through the C ABI."""
import ctypes

import numpy as np
import pytest

from conftest import splat_particles
from oracle import oracle
from test_oracle_splat import assert_bitexact, reference_outputs

pytestmark = pytest.mark.gpu


def test_splat_matches_reference_bitexact(golden_splat):
    """Host entry point on the fixture's particles and grid: the splat grid
    and the combined velocity are bit-identical to the reference's, twice in
    a row on one context (the second call reuses its buffers)."""
    from shiokaze_b200 import native
    name, g = golden_splat
    nx, ny, nz = (int(v) for v in g["shape"])
    P = splat_particles(g)
    ctx = native.Context(native.default_config())
    for _ in range(2):
        got = native.splat(ctx, nx, ny, nz, float(g["dx"]), P, [g["u0"], g["v0"], g["w0"]],
                           [g["u0_active"], g["v0_active"], g["w0_active"]], apic=bool(g["apic"]),
                           splat_bullet=bool(g["splat_bullet"]))
        assert_bitexact(got, reference_outputs(g))


def test_one_context_across_grid_shapes():
    """One context runs every splat fixture, of two grid shapes, in turn and
    twice around, bit-exact each time: the bucket counters stay zero between
    calls (each call clears only the tiles its particles reached), and the
    splat grid is zero wherever this call's particles do not reach, whatever
    the context's buffers held from the call before."""
    from conftest import golden_names, load_golden
    from shiokaze_b200 import native
    names = golden_names("splat_")
    assert len({tuple(load_golden(n)["shape"]) for n in names}) > 1
    ctx = native.Context(native.default_config())
    for name in names + names[::-1]:
        g = load_golden(name)
        nx, ny, nz = (int(v) for v in g["shape"])
        got = native.splat(ctx, nx, ny, nz, float(g["dx"]), splat_particles(g), [g["u0"], g["v0"], g["w0"]],
                           [g["u0_active"], g["v0_active"], g["w0_active"]], apic=bool(g["apic"]),
                           splat_bullet=bool(g["splat_bullet"]))
        assert_bitexact(got, reference_outputs(g))


@pytest.mark.parametrize("apic,n", [(True, 64), (False, 64), (True, 48)])
def test_splat_on_device_then_projection(apic, n):
    """n^3 dam break with 8 particles per liquid cell (about 0.6 M records of
    the reference's 84-byte layout at 64^3, edge cases included; dx = 1/48 is
    not a power of two, 1/64 is): splat_device on device arrays equals the
    reference-pinned CPU restatement bit for bit; the splatted velocity then
    goes straight to project_device, as the FLIP liquid solver's step does."""
    import torch
    from shiokaze_b200 import native, scenes
    L = native.load()
    sc = scenes.dambreak_sphere(n=n, seed=5)
    P = scenes.flip_particles(sc, per_cell=8, seed=2, bullet_fraction=0.03)
    vel0 = sc.velocity_effective()
    act0 = [m.astype(np.uint8) for m in sc.velocity_active]
    want = oracle.splat(sc.nx, sc.ny, sc.nz, sc.dx, P, vel0, act0, apic=apic)
    dev = torch.device("cuda:0")
    T = lambda arr: torch.from_numpy(np.ascontiguousarray(arr)).to(dev)
    rec = T(P.view(np.uint8))
    vel = [T(v) for v in vel0]
    act = [T(m) for m in act0]
    mass = [torch.zeros_like(v) for v in vel]
    mom = [torch.zeros_like(v) for v in vel]
    sact = [torch.zeros_like(m) for m in act]
    torch.cuda.synchronize()
    ctx = native.Context(native.default_config())
    a = native.splat_args(sc.nx, sc.ny, sc.nz, sc.dx, rec.data_ptr(), len(P), P.dtype, apic=apic)
    for d in range(3):
        a.velocity[d], a.velocity_active[d] = vel[d].data_ptr(), act[d].data_ptr()
        a.mass[d], a.momentum[d], a.splat_active[d] = mass[d].data_ptr(), mom[d].data_ptr(), sact[d].data_ptr()
    ctx.check(L.shkz_b200_splat_device(ctx.handle, ctypes.byref(a)), "splat_device")
    got = ([v.cpu().numpy() for v in vel], [m.cpu().numpy() for m in act], [m.cpu().numpy() for m in mass],
           [m.cpu().numpy() for m in mom], [m.cpu().numpy() for m in sact])
    assert_bitexact(got, dict(zip(("velocity", "velocity_active", "mass", "momentum", "splat_active"), want)))
    assert sum(int(s.sum()) for s in got[4]) > 1000
    # the splatted velocity is the projection's input
    fluid, fact = T(sc.fluid_effective()), T(sc.fluid_active.astype(np.uint8))
    solid, sact_ = T(sc.solid_effective()), T(sc.solid_active.astype(np.uint8))
    svel = [T(v) for v in sc.solid_velocity_effective()]
    p = native.ProjectArgs()
    p.nx, p.ny, p.nz, p.dx, p.dt = sc.nx, sc.ny, sc.nz, sc.dx, sc.dt
    p.fluid, p.fluid_active, p.solid, p.solid_active = fluid.data_ptr(), fact.data_ptr(), solid.data_ptr(), sact_.data_ptr()
    for d in range(3):
        p.velocity[d], p.velocity_active[d], p.solid_velocity[d] = vel[d].data_ptr(), act[d].data_ptr(), svel[d].data_ptr()
    res = native.Result()
    ctx.check(L.shkz_b200_project_device(ctx.handle, ctypes.byref(p), ctypes.byref(res)), "project_device")
    assert res.status == 0 and res.iterations > 0 and res.reresid <= sc.tol


def test_splat_without_particles_and_argument_errors():
    """No particles: the grid velocity is left as it is and nothing splats.
    Bad strides, offsets, misaligned device records or a partial set of
    outputs are refused before any device work."""
    from shiokaze_b200 import native, scenes
    sc = scenes.dambreak_sphere(n=12, seed=1)
    ctx = native.Context(native.default_config())
    vel0 = sc.velocity_effective()
    act0 = [m.astype(np.uint8) for m in sc.velocity_active]
    v, a, mass, mom, sact = native.splat(ctx, sc.nx, sc.ny, sc.nz, sc.dx, np.zeros(0, scenes.PARTICLE_DTYPE),
                                         vel0, act0)
    for d in range(3):
        assert np.array_equal(v[d].view(np.uint32), vel0[d].view(np.uint32))
        assert np.array_equal(a[d], act0[d]) and not sact[d].any()
    L = native.load()
    P = scenes.flip_particles(sc, per_cell=1, seed=0)
    buf = [np.zeros_like(x) for x in vel0]
    msk = [np.zeros_like(x) for x in act0]

    def args(**kw):
        s = native.splat_args(sc.nx, sc.ny, sc.nz, sc.dx, P.ctypes.data, len(P), P.dtype)
        for d in range(3):
            s.velocity[d], s.velocity_active[d] = buf[d].ctypes.data, msk[d].ctypes.data
        for k, val in kw.items():
            setattr(s, k, val)
        return s

    for bad in (dict(stride=83), dict(offset_mass=82), dict(offset_apic=60), dict(offset_position=-4),
                dict(offset_bullet=84), dict(dx=0.0), dict(nx=0), dict(count=-1)):
        assert L.shkz_b200_splat_host(ctx.handle, ctypes.byref(args(**bad))) == -1, bad
    partial = args()
    partial.mass[0] = buf[0].ctypes.data
    assert L.shkz_b200_splat_host(ctx.handle, ctypes.byref(partial)) == -1
    assert L.shkz_b200_splat_device(ctx.handle, ctypes.byref(args(particles=P.ctypes.data + 2))) == -1
    shifted = args()
    shifted.velocity[1] = buf[1].ctypes.data + 2
    assert L.shkz_b200_splat_device(ctx.handle, ctypes.byref(shifted)) == -1


def test_oversized_bucket_is_refused_and_grids_untouched():
    """More than 4096 particles in one edge bucket (never the case in a FLIP
    simulation, which keeps 8 to 12 per cell) returns SHKZ_B200_ERR_LIMIT and
    leaves the caller's grids as they were; the next normal call works."""
    import ctypes as C
    from shiokaze_b200 import native, scenes
    sc = scenes.dambreak_sphere(n=12, seed=1)
    ctx = native.Context(native.default_config())
    L = native.load()
    P = np.zeros(5000, scenes.PARTICLE_DTYPE)
    P["p"] = np.float32(5.3 * sc.dx)
    P["mass"] = np.float32(0.125)
    vel = [np.ascontiguousarray(v).copy() for v in sc.velocity_effective()]
    act = [m.astype(np.uint8) for m in sc.velocity_active]
    before = [v.copy() for v in vel], [m.copy() for m in act]
    a = native.splat_args(sc.nx, sc.ny, sc.nz, sc.dx, P.ctypes.data, len(P), P.dtype)
    for d in range(3):
        a.velocity[d], a.velocity_active[d] = vel[d].ctypes.data, act[d].ctypes.data
    assert L.shkz_b200_splat_host(ctx.handle, C.byref(a)) == -8
    for d in range(3):
        assert np.array_equal(vel[d].view(np.uint32), before[0][d].view(np.uint32))
        assert np.array_equal(act[d], before[1][d])
    small = P[:100]
    v, a_, mass, mom, sact = native.splat(ctx, sc.nx, sc.ny, sc.nz, sc.dx, small, vel, act)
    want = oracle.splat(sc.nx, sc.ny, sc.nz, sc.dx, small, vel, act)
    assert_bitexact((v, a_, mass, mom, sact), dict(zip(("velocity", "velocity_active", "mass", "momentum",
                                                        "splat_active"), want)))


def test_splat_grid_alone_without_velocity(golden_splat):
    """Velocity pointers NULL: the entry point returns the splat grid alone
    (what macflip3_interface::splat hands back), bit-identical to the
    reference's; with neither the velocity nor the splat grid the call is
    refused."""
    from shiokaze_b200 import native
    name, g = golden_splat
    nx, ny, nz = (int(v) for v in g["shape"])
    P = splat_particles(g)
    want = reference_outputs(g)
    ctx = native.Context(native.default_config())
    L = native.load()
    mass = [np.zeros_like(np.asarray(x, np.float32)) for x in want["mass"]]
    mom = [np.zeros_like(m) for m in mass]
    sact = [np.zeros(m.shape, np.uint8) for m in mass]
    a = native.splat_args(nx, ny, nz, float(g["dx"]), P.ctypes.data, len(P), P.dtype, apic=bool(g["apic"]),
                          splat_bullet=bool(g["splat_bullet"]))
    for d in range(3):
        a.mass[d], a.momentum[d], a.splat_active[d] = mass[d].ctypes.data, mom[d].ctypes.data, sact[d].ctypes.data
    ctx.check(L.shkz_b200_splat_host(ctx.handle, ctypes.byref(a)), "splat_host")
    for d in range(3):
        assert np.array_equal(sact[d], want["splat_active"][d])
        assert np.array_equal(mass[d].view(np.uint32), np.asarray(want["mass"][d], np.float32).view(np.uint32))
        assert np.array_equal(mom[d].view(np.uint32), np.asarray(want["momentum"][d], np.float32).view(np.uint32))
    b = native.splat_args(nx, ny, nz, float(g["dx"]), P.ctypes.data, len(P), P.dtype)
    assert L.shkz_b200_splat_host(ctx.handle, ctypes.byref(b)) == -1
