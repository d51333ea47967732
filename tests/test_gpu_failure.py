"""Failure handling on the device, made without faulting the GPU.

The reference has no failure handling of its own on this path: a fatal module
error ends the process (src/core/module.cpp:141) and a solve that does not
converge returns silently after MaxIterations
(local/include/pcgsolver/pcg_solver.h:267-295). The B200 library reports each
failure as a status code instead, and the context stays usable:

* a bounded device wait that runs out returns SHKZ_B200_ERR_TIMEOUT. The test
  makes it run out on purpose: B200.FaultSkipPublish stops one tile of the
  forward MIC(0) sweep from publishing its faces (a flag that nothing sets),
  and B200.SpinLimit shortens the waits;
* the same for the generic CSR solve's MIC(0) triangular solves: there
  B200.FaultSkipPublish stops one row of the forward solve from storing its
  value, and the rows that wait on it give up;
* a device-memory cap that the tile pool does not fit under returns
  SHKZ_B200_ERR_NOMEM before cudaMalloc is asked;
* a learned preconditioner that breaks down (a network of zeros) falls back to
  MIC(0) and the solve still reaches the MIC(0) answer.
After each, the next call on the same context succeeds.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ERR_NOMEM, ERR_TIMEOUT = -3, -4


def _run(s, sc):
    from shiokaze_b200.projection import grids_from_scene
    vel, solid, svel, fluid = grids_from_scene(sc)
    res = s.project(sc.dt, vel, solid, svel, fluid)
    return res, s.get_pressure().values.copy(), [v.copy() for v in vel.values]


def _reference_solution(sc):
    from shiokaze_b200.projection import MacPressureSolver3
    s = MacPressureSolver3({"Residual": sc.tol})
    s.initialize((sc.nx, sc.ny, sc.nz), sc.dx)
    res, p, v = _run(s, sc)
    assert res["status"] == 0, res
    return res, p, v


def test_sweep_wait_timeout_returns_error_and_context_recovers():
    from shiokaze_b200 import scenes
    from shiokaze_b200.projection import MacPressureSolver3
    sc = scenes.dambreak_sphere(n=64, seed=1, tol=1e-6)
    res0, p0, v0 = _reference_solution(sc)
    # the first tile of the forward sweep's wavefront never publishes; its
    # consumers give up after 20000 polling rounds (milliseconds)
    s = MacPressureSolver3({"Residual": sc.tol, "B200.SpinLimit": 20000, "B200.FaultSkipPublish": 1})
    s.initialize((sc.nx, sc.ny, sc.nz), sc.dx)
    res, _, _ = _run(s, sc)
    assert res["status"] == ERR_TIMEOUT, res
    # the same context, fault off: a normal projection, identical to a fresh context's
    s.configure({"B200.SpinLimit": 0, "B200.FaultSkipPublish": 0})
    res1, p1, v1 = _run(s, sc)
    assert res1["status"] == 0, res1
    assert res1["iterations"] == res0["iterations"]
    assert np.array_equal(p1, p0)
    for d in range(3):
        assert np.array_equal(v1[d], v0[d])


def test_csr_solve_wait_timeout_returns_error_and_context_recovers():
    import ctypes
    from conftest import golden_names, load_golden
    from shiokaze_b200 import native
    g = load_golden(golden_names()[0])
    n = int(g["rhs"].size)
    indptr = np.ascontiguousarray(g["indptr"], np.int64)
    indices = np.ascontiguousarray(g["indices"], np.int64)
    data = np.ascontiguousarray(g["data"], np.float64)
    b = np.ascontiguousarray(g["rhs"], np.float64)
    L = native.load()

    def solve(ctx):
        x = np.zeros(n, np.float64)
        res = native.Result()
        rc = L.shkz_b200_solve_csr(ctx.handle, n, indptr.ctypes.data, indices.ctypes.data, data.ctypes.data,
                                   b.ctypes.data, x.ctypes.data, ctypes.byref(res))
        return rc, res, x

    cfg = native.default_config()
    cfg.residual = float(g["tol"])
    cfg.csr_preconditioner = native.PRECOND_MIC0
    rc0, res0, x0 = solve(native.Context(cfg))
    assert rc0 == 0 and res0.iterations > 0
    # the first row of the forward triangular solve never stores its value;
    # the rows that depend on it give up after 20000 polling rounds
    cfg.spin_limit, cfg.fault_skip_publish = 20000, 1
    ctx = native.Context(cfg)
    rc, _, _ = solve(ctx)
    assert rc == ERR_TIMEOUT, rc
    # the same context, fault off: the same solve as a fresh context's
    cfg.spin_limit, cfg.fault_skip_publish = 0, 0
    ctx.set_config(cfg)
    rc1, res1, x1 = solve(ctx)
    assert rc1 == 0 and res1.iterations == res0.iterations
    assert np.array_equal(x1, x0)


def test_device_memory_cap_returns_nomem_and_context_recovers():
    from shiokaze_b200 import native, scenes
    from shiokaze_b200.projection import MacPressureSolver3
    sc = scenes.dambreak_sphere(n=48, seed=2, tol=1e-6)
    res0, p0, _ = _reference_solution(sc)
    # 6 MiB holds the 48^3 grid and host-staging buffers (about 5 MB) but not
    # the tile pool (about 80 KB per tile for 100+ tiles)
    s = MacPressureSolver3({"Residual": sc.tol, "B200.DeviceMemoryLimitMB": 6})
    s.initialize((sc.nx, sc.ny, sc.nz), sc.dx)
    with pytest.raises(native.ShkzError) as e:
        _run(s, sc)
    assert e.value.code == ERR_NOMEM
    msg = str(e.value)
    assert "device memory cap of 6 MiB" in msg, msg
    pool_buffers = ("pool_tile", "nbr", "sched", "diag", "offx", "offy", "offz", "d32", "diag64", "offx64",
                    "offy64", "offz64", "rhs64", "colsum", "dmic64", "x64", "r64", "xref64", "p64", "q64", "z64")
    assert msg.split(" for ")[-1].split()[0] in pool_buffers, msg
    s.configure({"B200.DeviceMemoryLimitMB": 0})
    res1, p1, _ = _run(s, sc)
    assert res1["status"] == 0, res1
    assert np.array_equal(p1, p0)


def test_zero_network_falls_back_to_mic0_and_reaches_its_answer():
    from shiokaze_b200 import scenes
    from shiokaze_b200.projection import MacPressureSolver3
    sc = scenes.dambreak_sphere(n=32, seed=2, tol=1e-6)
    res0, p0, _ = _reference_solution(sc)
    s = MacPressureSolver3({"Residual": sc.tol})
    s.initialize((sc.nx, sc.ny, sc.nz), sc.dx)
    res, _, _ = _run(s, sc)
    assert res["status"] == 0
    s.learned_init(seed=3)
    s.learned_set_params(np.zeros_like(s.learned_params()))
    s.configure({"B200.Preconditioner": "learned"})
    res1, p1, _ = _run(s, sc)
    assert res1["status"] == 0, res1
    assert res1["fallbacks"] == 1, res1
    assert res1["reresid"] <= sc.tol
    assert np.abs(p1.astype(np.float64) - p0).max() / np.abs(p0).max() < 1e-4
