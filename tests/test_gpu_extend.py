"""Velocity extension after a projection on the device
(shkz_b200_extend_velocity_host / _device: macarray_extrapolator3::extrapolate
+ macutility3::constrain_velocity, as macliquid3::extend_both runs them)
against the reference: bit-exact, through the C ABI."""
import ctypes

import numpy as np
import pytest

from conftest import GoldenScene, load_golden
from oracle import extend as ext

pytestmark = pytest.mark.gpu


def _inputs(g):
    vel = [g["u0"], g["v0"], g["w0"]]
    act = [g["u0_active"], g["v0_active"], g["w0_active"]]
    solid = g["solid"] if int(g["has_solid"]) else None
    sact = g["solid_active"] if int(g["has_solid"]) else None
    return vel, act, solid, sact


def _assert_same(v, a, want_v, want_a):
    for d in range(3):
        assert np.array_equal(np.asarray(a[d]).astype(bool), np.asarray(want_a[d]).astype(bool)), f"mask {d}"
        m = np.asarray(want_a[d]).astype(bool)
        got = np.asarray(v[d], np.float32)[m].view(np.uint32)
        want = np.asarray(want_v[d], np.float32)[m].view(np.uint32)
        assert np.array_equal(got, want), f"values {d}: {int(np.sum(got != want))} differ"


def test_extension_matches_reference_bitexact(golden_ext):
    """Host entry point on the reference's projected velocity: identical
    masks and bit-identical values to the reference's extension, twice in a
    row on one context (the second call reuses its buffers)."""
    from shiokaze_b200 import native
    name, g = golden_ext
    ctx = native.Context(native.default_config())
    vel, act, solid, sact = _inputs(g)
    want_v, want_a = [g["u"], g["v"], g["w"]], [g["u_active"], g["v_active"], g["w_active"]]
    for _ in range(2):
        v, a = native.extend_velocity(ctx, vel, act, solid, sact, float(g["dx"]), int(g["width"]), bool(g["constrain"]))
        _assert_same(v, a, want_v, want_a)


def test_extension_on_device_after_device_projection():
    """project_device then extend_device on the same device arrays (the
    velocity never leaves the GPU in between); the result equals the
    reference-pinned CPU restatement applied to the projected velocity."""
    import torch
    from shiokaze_b200 import native
    L = native.load()
    g = load_golden("sloshing_tank_24")
    sc = GoldenScene(g)
    dev = torch.device("cuda:0")
    T = lambda arr: torch.from_numpy(np.ascontiguousarray(arr)).to(dev)
    fluid, fact = T(sc.fluid_effective()), T(sc.fluid_active.astype(np.uint8))
    solid, sact = T(sc.solid_effective()), T(sc.solid_active.astype(np.uint8))
    vel = [T(v) for v in sc.velocity_effective()]
    vact = [T(m.astype(np.uint8)) for m in sc.velocity_active]
    svel = [T(v) for v in sc.solid_velocity_effective()]
    ctx = native.Context(native.default_config())
    torch.cuda.synchronize()
    a = native.ProjectArgs()
    a.nx, a.ny, a.nz, a.dx, a.dt = sc.nx, sc.ny, sc.nz, sc.dx, sc.dt
    a.fluid, a.fluid_active = fluid.data_ptr(), fact.data_ptr()
    a.solid, a.solid_active = solid.data_ptr(), sact.data_ptr()
    for d in range(3):
        a.velocity[d], a.velocity_active[d], a.solid_velocity[d] = vel[d].data_ptr(), vact[d].data_ptr(), svel[d].data_ptr()
    res = native.Result()
    ctx.check(L.shkz_b200_project_device(ctx.handle, ctypes.byref(a), ctypes.byref(res)), "project_device")
    projected = [v.cpu().numpy().copy() for v in vel], [m.cpu().numpy().copy() for m in vact]
    e = native.ExtendArgs()
    e.nx, e.ny, e.nz, e.dx, e.width, e.constrain = sc.nx, sc.ny, sc.nz, sc.dx, 3, 1
    e.solid, e.solid_active = solid.data_ptr(), sact.data_ptr()
    for d in range(3):
        e.velocity[d], e.velocity_active[d] = vel[d].data_ptr(), vact[d].data_ptr()
    ctx.check(L.shkz_b200_extend_velocity_device(ctx.handle, ctypes.byref(e)), "extend_velocity_device")
    got_v, got_a = [v.cpu().numpy() for v in vel], [m.cpu().numpy() for m in vact]
    want_v, want_a = ext.extend(projected[0], projected[1], sc.solid_effective(), sc.solid_active, sc.dx, 3, True)
    _assert_same(got_v, got_a, want_v, want_a)
    assert all(got_a[d].sum() > projected[1][d].sum() for d in range(3))


def test_extension_without_constraint_or_passes_and_argument_errors():
    """width 0 without the constraint leaves the field as it is; bad sizes and
    widths are refused before any device work."""
    from shiokaze_b200 import native
    g = load_golden("ext_dambreak_sphere_24")
    ctx = native.Context(native.default_config())
    vel, act, solid, sact = _inputs(g)
    v, a = native.extend_velocity(ctx, vel, act, solid, sact, float(g["dx"]), 0, False)
    for d in range(3):
        assert np.array_equal(a[d], np.asarray(act[d], np.uint8))
        assert np.array_equal(v[d].view(np.uint32), np.asarray(vel[d], np.float32).view(np.uint32))
    L = native.load()
    e = native.ExtendArgs()
    buf = np.zeros(64, np.float32)
    m = np.zeros(64, np.uint8)
    for d in range(3):
        e.velocity[d], e.velocity_active[d] = buf.ctypes.data, m.ctypes.data
    e.nx, e.ny, e.nz, e.dx, e.width = 1, 4, 4, 1.0, 1
    assert L.shkz_b200_extend_velocity_host(ctx.handle, ctypes.byref(e)) == -1
    e.nx, e.width = 4, -1
    assert L.shkz_b200_extend_velocity_host(ctx.handle, ctypes.byref(e)) == -1
