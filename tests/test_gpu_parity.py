"""Parity of the CUDA projection with the reference, through the C ABI.

Golden fixtures come from the compiled reference (tests/golden/make_golden.py);
larger cases are checked against the CPU restatement in oracle/. Bars:
* masks (unknowns, face active bits): bit-exact
* FP64 right-hand side: bit-exact; FP32 matrix weights: the FP64 value
  rounded once to FP32
* pressure and projected face velocities: within PARITY_TOL relative
  (infinity norm over the reference's infinity norm) at the same tolerance
* MIC(0) iteration count: within max(1, 2%) of the reference MIC(0) run
"""
import numpy as np
import pytest

from conftest import GoldenScene
from oracle import oracle

pytestmark = pytest.mark.gpu

PARITY_TOL = 1e-5


def solver(**cfg):
    from shiokaze_b200.projection import MacPressureSolver3
    return MacPressureSolver3(cfg)


def run(sc, **cfg):
    from shiokaze_b200.projection import grids_from_scene
    s = solver(**cfg)
    s.initialize((sc.nx, sc.ny, sc.nz), sc.dx)
    vel, solid, svel, fluid = grids_from_scene(sc)
    res = s.project(sc.dt, vel, solid, svel, fluid)
    return s, res, vel


def rel_inf(a, b):
    den = np.abs(b).max()
    return float(np.abs(a.astype(np.float64) - b.astype(np.float64)).max() / (den if den else 1.0))


def test_golden_projection_parity(golden):
    name, g = golden
    sc = GoldenScene(g)
    s, res, vel = run(sc, Residual=float(g["tol"]))
    assert res["status"] == 0, res
    p = s.get_pressure()
    np.testing.assert_array_equal(p.active, g["pressure_active"])
    for d, k in enumerate("uvw"):
        np.testing.assert_array_equal(vel.active[d], g[k + "_active"])
    it_ref = int(g["iterations_mic0"])
    assert abs(res["iterations"] - it_ref) <= max(1, int(0.02 * it_ref)), (res["iterations"], it_ref)
    assert rel_inf(p.values, g["pressure"]) <= PARITY_TOL
    for d, k in enumerate("uvw"):
        assert rel_inf(vel.values[d], g[k]) <= PARITY_TOL, (k, rel_inf(vel.values[d], g[k]))
    assert res["reresid"] <= float(g["tol"])


def test_golden_system_bitexact(golden):
    """rhs (FP64) bit-exact; FP32 weights are the reference's FP64 entries rounded once."""
    name, g = golden
    sc = GoldenScene(g)
    s, res, _ = run(sc, Residual=float(g["tol"]))
    area, rho = oracle.fractions(sc)
    S = oracle.assemble(sc, area, rho)
    idx = S.index
    mask = idx >= 0
    rhs = s.inspect(5)
    np.testing.assert_array_equal(rhs[mask], S.rhs[idx[mask]])
    assert (rhs[~mask] == 0).all()
    A = S.matrix().tocsr()
    diag = s.inspect(0)
    np.testing.assert_array_equal(diag[mask], A.diagonal()[idx[mask]].astype(np.float32))
    nz, ny, nx = idx.shape
    for d, what in ((0, 1), (1, 2), (2, 3)):
        w = s.inspect(what)
        sl = [slice(None)] * 3
        ax = 2 - d
        lo = np.zeros_like(w)
        # expected: -A(i, i-e) where both are unknowns
        src = [slice(None)] * 3
        src[ax] = slice(1, None)
        nb = [slice(None)] * 3
        nb[ax] = slice(0, -1)
        i1 = idx[tuple(src)]
        i0 = idx[tuple(nb)]
        both = (i1 >= 0) & (i0 >= 0)
        vals = np.zeros(i1.shape, np.float64)
        vals[both] = -np.asarray(A[i1[both], i0[both]]).ravel()
        lo[tuple(src)] = vals.astype(np.float32)
        np.testing.assert_array_equal(w, lo)


@pytest.mark.parametrize("block", [8, 16])
def test_mic0_sweeps_match_oracle(golden, block):
    """Both sweep layouts (8^3 tiles, 16^3 macro tiles) against the oracle's MIC(0) apply."""
    name, g = golden
    sc = GoldenScene(g)
    s, _, _ = run(sc, Residual=float(g["tol"]), **{"B200.MICBlock": block})
    area, rho = oracle.fractions(sc)
    S = oracle.assemble(sc, area, rho)
    rng = np.random.default_rng(0)
    r = np.zeros(S.index.shape, np.float32)
    mask = S.index >= 0
    r[mask] = rng.standard_normal(mask.sum()).astype(np.float32)
    z = s.apply_preconditioner(r)
    zref, _ = oracle.mic0_apply(S, r[mask].astype(np.float64)[np.argsort(S.index[mask])])
    zg = np.zeros(S.n)
    zg[S.index[mask]] = z[mask]
    assert rel_inf(zg, zref) <= 1e-5
    assert (z[~mask] == 0).all()


def test_mic0_sweep_layouts_bitexact():
    """The 16^3 macro-tile sweeps evaluate the same per-cell expressions in the
    same dependency order as the 8^3 sweeps: identical FP32 results."""
    from shiokaze_b200 import scenes
    sc = scenes.dambreak_sphere(n=80, seed=3)
    zs = []
    for block in (8, 16):
        s, res, _ = run(sc, Residual=1e-6, **{"B200.MICBlock": block})
        assert res["status"] == 0
        rng = np.random.default_rng(1)
        mask = s.get_pressure().active.astype(bool)
        r = np.zeros(mask.shape, np.float32)
        r[mask] = rng.standard_normal(mask.sum()).astype(np.float32)
        zs.append(s.apply_preconditioner(r))
    np.testing.assert_array_equal(zs[0], zs[1])


def test_spmv_matches_oracle(golden):
    name, g = golden
    sc = GoldenScene(g)
    s, _, _ = run(sc, Residual=float(g["tol"]))
    area, rho = oracle.fractions(sc)
    S = oracle.assemble(sc, area, rho)
    mask = S.index >= 0
    rng = np.random.default_rng(1)
    x = np.zeros(S.index.shape, np.float32)
    x[mask] = rng.standard_normal(mask.sum()).astype(np.float32)
    y = s.apply_matrix(x)
    xo = np.zeros(S.n)
    xo[S.index[mask]] = x[mask]
    yref = oracle.spmv(S, xo)
    yg = np.zeros(S.n)
    yg[S.index[mask]] = y[mask]
    assert rel_inf(yg, yref) <= 1e-5
    assert (y[~mask] == 0).all()


# Identity-preconditioned CG over hundreds of steps loses orthogonality in
# FP32 (the reference runs it in FP64): the iteration count grows by up to a
# third (tolerances >= 1e-8; to 1e-12 it grows further) and the iterate agrees
# with the reference's to the scale of the tolerance (within 10x), not to 1e-5.
# The MIC(0) mode above is the drop-in and meets the tight bars.
SHIPPED_ITER_SLACK = 0.35


def test_shipped_mode_iterations(golden):
    """Identity preconditioner = what the shipped reference runs."""
    name, g = golden
    sc = GoldenScene(g)
    tol = float(g["tol"])
    s, res, vel = run(sc, Residual=tol, **{"B200.Preconditioner": "none"})
    it_ref = int(g["iterations_shipped"])
    assert res["iterations"] >= it_ref - 2
    if tol >= 1e-8:
        assert res["iterations"] <= it_ref * (1 + SHIPPED_ITER_SLACK) + 2, (res["iterations"], it_ref)
    assert res["reresid"] <= tol
    assert rel_inf(s.get_pressure().values, g["pressure_shipped"]) <= max(10 * tol, PARITY_TOL)


def test_fp64_reference_solve(golden):
    name, g = golden
    sc = GoldenScene(g)
    s, res, _ = run(sc, Residual=float(g["tol"]), **{"B200.FP64Reference": 1})
    assert res["fp64_reresid"] <= 1e-12
    assert 0 <= res["err_fp64_inf"] < 1.0


def test_dambreak_64_vs_oracle():
    """CPU-runnable configuration: 64^3, MIC(0)-PCG to 1e-4."""
    from shiokaze_b200 import scenes
    sc = scenes.dambreak_sphere(n=64, seed=0)
    o = oracle.project(sc, mic0=True)
    s, res, vel = run(sc, Residual=sc.tol)
    np.testing.assert_array_equal(s.get_pressure().active, o.pressure_active)
    for d in range(3):
        np.testing.assert_array_equal(vel.active[d], o.velocity_active[d])
    assert abs(res["iterations"] - o.iterations) <= max(1, int(0.02 * o.iterations))
    assert rel_inf(s.get_pressure().values, o.pressure) <= PARITY_TOL
    for d in range(3):
        assert rel_inf(vel.values[d], o.velocity[d]) <= PARITY_TOL


def test_tight_tolerance_reaches_target():
    """1e-6 with FP32 iterates needs the FP64 refinement; the true residual
    (checked on the CPU with the oracle's FP64 matrix) meets the target."""
    from shiokaze_b200 import scenes
    sc = scenes.sloshing_tank(n=48, seed=2, tol=1e-6)
    s, res, vel = run(sc, Residual=1e-6)
    assert res["status"] == 0
    area, rho = oracle.fractions(sc)
    S = oracle.assemble(sc, area, rho)
    x64 = s.inspect(6)
    mask = S.index >= 0
    xo = np.zeros(S.n)
    xo[S.index[mask]] = x64[mask]
    r = S.rhs - oracle.spmv(S, xo)
    assert np.abs(r).max() <= 1e-6 * np.abs(S.rhs).max()


def test_no_liquid_returns_zero_iterations():
    from shiokaze_b200 import scenes
    sc = scenes.dambreak_sphere(n=16, seed=1)
    sc.fluid_phi[:] = 1.0
    sc.fluid_active[:] = 0
    s, res, vel = run(sc)
    assert res["unknowns"] == 0 and res["iterations"] == 0
    assert (s.get_pressure().active == 0).all()


def test_nan_input_reports_status_without_hanging():
    from shiokaze_b200 import scenes
    sc = scenes.dambreak_sphere(n=16, seed=1)
    sc.velocity[0][4, 4, 4] = np.nan
    sc.velocity_active[0][4, 4, 4] = 1
    s, res, vel = run(sc)
    assert res["status"] == -5


def test_solve_csr_matches_shipped_pcg(golden):
    """shkz_b200_solve_csr on the reference's own assembled CSR: the shipped
    algorithm's iteration count (+-2 %) and pressure (1e-5)."""
    import ctypes
    from shiokaze_b200 import native
    name, g = golden
    sc = GoldenScene(g)
    n = int(g["rhs"].size)
    if n == 0:
        return
    ctx = native.Context(native.default_config())
    cfg = native.default_config()
    cfg.residual = float(g["tol"])
    ctx.set_config(cfg)
    indptr = np.ascontiguousarray(g["indptr"], np.int64)
    indices = np.ascontiguousarray(g["indices"], np.int64)
    data = np.ascontiguousarray(g["data"], np.float64)
    b = np.ascontiguousarray(g["rhs"], np.float64)
    x = np.zeros(n, np.float64)
    res = native.Result()
    rc = native.load().shkz_b200_solve_csr(ctx.handle, n, indptr.ctypes.data, indices.ctypes.data, data.ctypes.data,
                                           b.ctypes.data, x.ctypes.data, ctypes.byref(res))
    assert rc == 0
    # Unpreconditioned CG stops on a noisy inf-norm: the same FP64 recurrence
    # with only the dot-product summation order changed (sequential, BLAS,
    # random permutations) stops 3-5 % apart on these systems (splash_24:
    # 265-277, training_20: 227-238), so the bar is 5 %.
    it_ref = int(g["iterations_shipped"])
    assert abs(res.iterations - it_ref) <= max(2, int(0.05 * it_ref)), (res.iterations, it_ref)
    assert res.reresid <= float(g["tol"])
    idx = oracle.assemble(sc, *oracle.fractions(sc)).index
    mask = idx >= 0
    p = np.zeros(idx.shape, np.float32)
    p[mask] = x[idx[mask]].astype(np.float32)
    # two FP64 CG runs with different summation orders stop at the same count
    # but hold different iterates; the bar of the shipped mode applies
    assert rel_inf(p, g["pressure_shipped"]) <= max(PARITY_TOL, 10 * float(g["tol"]))


def test_solve_csr_mic0_matches_reference_mic0(golden):
    """shkz_b200_solve_csr with csr_preconditioner = MIC0 on the reference's own
    assembled CSR: the generic-matrix MIC(0) (level-scheduled factor and
    sync-free triangular solves on the device) against the reference's
    MIC(0)-PCG on the same system:
    iteration count within max(1, 2 %) and pressure within PARITY_TOL."""
    import ctypes
    from shiokaze_b200 import native
    name, g = golden
    sc = GoldenScene(g)
    n = int(g["rhs"].size)
    if n == 0:
        return
    cfg = native.default_config()
    cfg.residual = float(g["tol"])
    cfg.csr_preconditioner = native.PRECOND_MIC0
    ctx = native.Context(cfg)
    indptr = np.ascontiguousarray(g["indptr"], np.int64)
    indices = np.ascontiguousarray(g["indices"], np.int64)
    data = np.ascontiguousarray(g["data"], np.float64)
    b = np.ascontiguousarray(g["rhs"], np.float64)
    x = np.zeros(n, np.float64)
    res = native.Result()
    rc = native.load().shkz_b200_solve_csr(ctx.handle, n, indptr.ctypes.data, indices.ctypes.data, data.ctypes.data,
                                           b.ctypes.data, x.ctypes.data, ctypes.byref(res))
    assert rc == 0
    it_ref = int(g["iterations_mic0"])
    assert abs(res.iterations - it_ref) <= max(1, int(0.02 * it_ref)), (res.iterations, it_ref)
    assert res.reresid <= float(g["tol"])
    idx = oracle.assemble(sc, *oracle.fractions(sc)).index
    mask = idx >= 0
    p = np.zeros(idx.shape, np.float32)
    p[mask] = x[idx[mask]].astype(np.float32)
    assert rel_inf(p, g["pressure"]) <= PARITY_TOL


def test_solve_csr_mic0_apply_matches_oracle(golden):
    """One application of the CSR MIC(0) (a single PCG step from x0 = 0 with
    tolerance 1 returns x = alpha z0): z0 against the oracle's MIC(0) apply,
    which is bit-exact against the reference header's factor and sweeps."""
    import ctypes
    from shiokaze_b200 import native
    name, g = golden
    n = int(g["rhs"].size)
    if n == 0:
        return
    indptr = np.ascontiguousarray(g["indptr"], np.int64)
    indices = np.ascontiguousarray(g["indices"], np.int64)
    data = np.ascontiguousarray(g["data"], np.float64)
    b = np.ascontiguousarray(g["rhs"], np.float64)
    S = oracle.System(index=None, n=n, indptr=indptr, indices=indices, data=data, rhs=b)
    z, _ = oracle.mic0_apply(S, b)
    cfg = native.default_config()
    cfg.residual = 1e30  # stops after the first step
    cfg.csr_preconditioner = native.PRECOND_MIC0
    ctx = native.Context(cfg)
    x = np.zeros(n, np.float64)
    res = native.Result()
    rc = native.load().shkz_b200_solve_csr(ctx.handle, n, indptr.ctypes.data, indices.ctypes.data, data.ctypes.data,
                                           b.ctypes.data, x.ctypes.data, ctypes.byref(res))
    assert rc == 0 and res.iterations == 1
    # x = alpha z0 with alpha = (z0.b) / (z0.A z0)
    Az = oracle.spmv(S, z)
    alpha = float(z @ b) / float(z @ Az)
    assert np.abs(x - alpha * z).max() <= 1e-12 * np.abs(alpha * z).max()


def test_tile_activity_matches_reference(golden):
    """Tile activity: the pool holds exactly the 8^3 tiles in which the
    reference's pressure grid has an active cell (its allocated tiles)."""
    name, g = golden
    sc = GoldenScene(g)
    s, res, _ = run(sc, Residual=float(g["tol"]))
    act = g["pressure_active"].astype(bool)
    nz, ny, nx = act.shape
    pad = np.zeros(((nz + 7) // 8 * 8, (ny + 7) // 8 * 8, (nx + 7) // 8 * 8), bool)
    pad[:nz, :ny, :nx] = act
    tiles = pad.reshape(pad.shape[0] // 8, 8, pad.shape[1] // 8, 8, pad.shape[2] // 8, 8).any(axis=(1, 3, 5))
    assert res["tiles"] == int(tiles.sum())
    assert res["unknowns"] == int(act.sum())


def test_size_limits_are_errors_not_faults():
    """Grids beyond the documented limits are refused before any device work."""
    import ctypes
    from shiokaze_b200 import native
    ctx = native.Context(native.default_config())
    a = native.ProjectArgs()
    a.nx, a.ny, a.nz, a.dx, a.dt = 70000, 8, 8, 1.0, 1.0
    buf = np.zeros(8, np.float32)
    m = np.zeros(8, np.uint8)
    a.fluid, a.fluid_active = buf.ctypes.data, m.ctypes.data
    for d in range(3):
        a.velocity[d] = buf.ctypes.data
        a.velocity_active[d] = m.ctypes.data
    res = native.Result()
    rc = native.load().shkz_b200_project_device(ctx.handle, ctypes.byref(a), ctypes.byref(res))
    assert rc == -8  # SHKZ_B200_ERR_LIMIT
    a.nx = 0
    rc = native.load().shkz_b200_project_device(ctx.handle, ctypes.byref(a), ctypes.byref(res))
    assert rc == -1  # SHKZ_B200_ERR_ARG


def _csr_solve(indptr, indices, data, b, pre, tol=1e-10):
    import ctypes
    from shiokaze_b200 import native
    cfg = native.default_config()
    cfg.residual = tol
    cfg.csr_preconditioner = pre
    ctx = native.Context(cfg)
    n = len(b)
    x = np.zeros(n, np.float64)
    res = native.Result()
    ip, ix = np.ascontiguousarray(indptr, np.int64), np.ascontiguousarray(indices, np.int64)
    d, bb = np.ascontiguousarray(data, np.float64), np.ascontiguousarray(b, np.float64)
    rc = native.load().shkz_b200_solve_csr(ctx.handle, n, ip.ctypes.data, ix.ctypes.data, d.ctypes.data,
                                           bb.ctypes.data, x.ctypes.data, ctypes.byref(res))
    return rc, res, x


@pytest.mark.parametrize("pre", [0, 1])
def test_solve_csr_edge_cases(pre):
    """The generic CSR solve on degenerate and deep systems, both
    preconditioners: a 1x1 system, a diagonal one (a single level), a zero
    right-hand side (no iteration), and a 1D Laplacian chain of 5,000 rows,
    whose MIC(0) factor has 5,000 levels, against the oracle's PCG."""
    # 1x1
    rc, res, x = _csr_solve([0, 1], [0], [4.0], [2.0], pre)
    assert rc == 0 and res.iterations == 1 and x[0] == 0.5
    # diagonal
    rng = np.random.default_rng(3)
    n = 1000
    dg = rng.uniform(1.0, 3.0, n)
    b = rng.uniform(-1.0, 1.0, n)
    rc, res, x = _csr_solve(np.arange(n + 1), np.arange(n), dg, b, pre)
    assert rc == 0
    if pre == 1:
        # the MIC(0) of a diagonal matrix is exact: one step
        assert res.iterations == 1 and np.abs(x - b / dg).max() <= 1e-12
    else:
        assert np.abs(x - b / dg).max() <= 1e-8
    # zero right-hand side
    rc, res, x = _csr_solve(np.arange(n + 1), np.arange(n), dg, np.zeros(n), pre)
    assert rc == 0 and res.iterations == 0 and not x.any()
    # 1D Laplacian chain: row i couples i-1 and i+1
    n = 5000
    rows = []
    for i in range(n):
        rows.append([(j, v) for j, v in ((i - 1, -1.0), (i, 2.0 + 1e-3), (i + 1, -1.0)) if 0 <= j < n])
    indptr = np.cumsum([0] + [len(r) for r in rows])
    indices = np.array([j for r in rows for j, _ in r])
    data = np.array([v for r in rows for _, v in r])
    b = rng.uniform(-1.0, 1.0, n)
    rc, res, x = _csr_solve(indptr, indices, data, b, pre, tol=1e-9)
    S = oracle.System(index=None, n=n, indptr=indptr.astype(np.int64), indices=indices.astype(np.int64),
                      data=data, rhs=b)
    xo, it_o, _ = oracle.pcg(S, 1e-9, 30000, bool(pre))
    assert rc == 0, rc
    # summation order alone moves long unpreconditioned CG runs by a few percent
    assert abs(res.iterations - it_o) <= max(1, int((0.02 if pre else 0.05) * it_o)), (res.iterations, it_o)
    assert np.abs(x - xo[:n]).max() <= 1e-6 * np.abs(xo).max()


def test_one_context_across_scenes_matches_fresh_contexts():
    """A projection module lives through a simulation whose grid can change
    (a new scene, a resized domain): one context runs scenes of five shapes in
    turn, some twice, growing and shrinking its tile pool, macro tiles and
    wavefront buffers, and every projection is bit-identical (pressure,
    velocities, masks, iteration count) to the same projection on a fresh
    context."""
    from shiokaze_b200 import scenes
    from shiokaze_b200.projection import grids_from_scene
    seq = [scenes.dambreak_sphere(n=48, seed=2, tol=1e-6), scenes.sloshing_tank(n=96, seed=1, tol=1e-6),
           scenes.splash(n=80, seed=4, tol=1e-6, spheres=30), scenes.dambreak_sphere(n=48, seed=2, tol=1e-6),
           scenes.training_scene(n=64, seed=3), scenes.sloshing_tank(n=96, seed=1, tol=1e-6),
           scenes.dambreak_sphere(n=20, seed=5, tol=1e-6)]
    shared = solver(Residual=1e-6)
    for sc in seq:
        shared.initialize((sc.nx, sc.ny, sc.nz), sc.dx)
        vel, solid, svel, fluid = grids_from_scene(sc)
        res = shared.project(sc.dt, vel, solid, svel, fluid)
        fresh, res0, vel0 = run(sc, Residual=1e-6)
        assert res["status"] == 0 and res0["status"] == 0, (res, res0)
        assert res["iterations"] == res0["iterations"], (sc.name, sc.nx, res["iterations"], res0["iterations"])
        p, p0 = shared.get_pressure(), fresh.get_pressure()
        assert np.array_equal(p.active, p0.active)
        assert np.array_equal(p.values.view(np.uint32), p0.values.view(np.uint32)), (sc.name, sc.nx)
        for d in range(3):
            assert np.array_equal(vel.active[d], vel0.active[d])
            assert np.array_equal(vel.values[d].view(np.uint32), vel0.values[d].view(np.uint32)), (sc.name, d)
