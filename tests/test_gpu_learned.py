"""The learned preconditioner's CUDA kernels (tcgen05 convolutions, pooling,
input/weight gradients, Adam) against the CPU restatement in oracle/convnet.py,
and the flexible PCG that uses it. BF16 activations: forward outputs agree to
a few BF16 ulps, gradients to a few per cent (relative Frobenius norm)."""
import numpy as np
import pytest

from oracle import convnet as cn

pytestmark = pytest.mark.gpu


def _projected(n=32, seed=1, **cfg):
    from shiokaze_b200 import scenes
    from shiokaze_b200.projection import MacPressureSolver3, grids_from_scene
    sc = scenes.dambreak_sphere(n=n, seed=seed)
    s = MacPressureSolver3({"Residual": 1e-6, **cfg})
    s.initialize((sc.nx, sc.ny, sc.nz), sc.dx)
    vel, solid, svel, fluid = grids_from_scene(sc)
    res = s.project(sc.dt, vel, solid, svel, fluid)
    return sc, s, res


def _unpack(blob):
    P, off = {}, 0
    for name, lvl, in0, in1, cout, relu in cn.LAYERS:
        cin = in0[1] + (in1[1] if in1 else 0)
        nw = 27 * cout * cin
        P[name + ".w"] = blob[off:off + nw].reshape(27, cout, cin).copy()
        off += nw
        P[name + ".b"] = blob[off:off + cout].copy()
        off += cout
    assert off == blob.size
    return P


def _pool_cells(s, shape_pad):
    unk = s.get_pressure().active.astype(bool)
    nz, ny, nx = unk.shape
    t = unk.reshape(nz // 8, 8, ny // 8, 8, nx // 8, 8).any(axis=(1, 3, 5))
    cells = np.repeat(np.repeat(np.repeat(t, 8, 0), 8, 1), 8, 2)
    pad = np.zeros(shape_pad, bool)
    pad[:nz, :ny, :nx] = cells
    return pad


def test_forward_matches_oracle():
    sc, s, _ = _projected()
    s.learned_init(seed=3)
    rng = np.random.default_rng(0)
    unk = s.get_pressure().active.astype(bool)
    r = np.where(unk, rng.standard_normal(unk.shape), 0).astype(np.float32)
    z = s.learned_apply(r)
    X0 = s.learned_tensor("X0")
    Zg = s.learned_tensor("Z")
    P = _unpack(s.learned_params())
    masks = cn.level_masks(_pool_cells(s, Zg.shape))
    Zo = cn.forward(P, X0, masks)
    scale = np.abs(Zo).max()
    assert scale > 0
    assert np.abs(Zg - Zo).max() / scale < 3e-2
    # z = s * N(r/s) at unknowns, zero elsewhere
    smax = np.abs(r).max()
    nz, ny, nx = unk.shape
    np.testing.assert_allclose(z[unk], (smax * Zg[:nz, :ny, :nx])[unk], rtol=1e-6, atol=1e-6 * smax)
    assert (z[~unk] == 0).all()


def test_gradients_match_oracle():
    sc, s, _ = _projected()
    s.learned_init(seed=4)
    P = _unpack(s.learned_params())
    # nonzero biases so every ReLU pattern is exercised
    rng = np.random.default_rng(1)
    for k in P:
        if k.endswith(".b"):
            P[k] = (0.05 * rng.standard_normal(P[k].shape)).astype(np.float32)
    blob = np.concatenate([np.concatenate([P[n + ".w"].ravel(), P[n + ".b"]]) for n, *_ in cn.LAYERS])
    s.learned_set_params(blob)
    unk = s.get_pressure().active.astype(bool)
    r = np.where(unk, rng.standard_normal(unk.shape), 0).astype(np.float32)
    s.learned_apply(r)
    X0 = s.learned_tensor("X0")
    masks = cn.level_masks(_pool_cells(s, X0.shape[:3]))
    gZ = rng.standard_normal(X0.shape[:3]).astype(np.float32) * masks[0]
    grads_gpu = _unpack(s.learned_backward(gZ))
    P = _unpack(s.learned_params())
    # backward of the oracle on the activations the GPU stored (its ReLU
    # pattern is the GPU's), so the comparison isolates the backward kernels
    T = {name: s.learned_tensor(name) for name in s.TENSORS[:-1]}
    pre = {}
    for name, lvl, in0, in1, cout, relu in cn.LAYERS:
        if relu:
            pre[name] = T[cn.OUTPUT[name]]
    tg = {}
    grads = cn.backward(P, T, pre, masks, gZ, tensor_grads=tg)
    gerr = {}
    for name in s.TENSORS[1:-1]:
        ref = tg[name] * masks[s.TENSORS.index(name) and {"X0": 0, "A1": 0, "S1": 0, "P1": 1, "A2": 1, "S2": 1,
                                                           "P2": 2, "A3": 2, "B3": 2, "C2": 1, "D2": 1, "C1": 0,
                                                           "D1": 0}[name]][..., None]
        got = s.learned_tensor(name, grad=True)
        gerr[name] = float(np.linalg.norm(got - ref) / max(np.linalg.norm(ref), 1e-30))
    print("activation-gradient errors:", {k: round(v, 4) for k, v in gerr.items()})
    errs = {}
    for name, *_ in cn.LAYERS:
        for k in (name + ".w", name + ".b"):
            ref = grads[k]
            den = np.linalg.norm(ref)
            if den == 0:
                continue
            errs[k] = float(np.linalg.norm(grads_gpu[k] - ref) / den)
    bad = {k: v for k, v in errs.items() if v >= 5e-2}
    print("relative gradient errors:", {k: round(v, 4) for k, v in errs.items()})
    assert not bad, sorted(bad)


def test_training_reduces_energy_loss():
    sc, s, _ = _projected()
    s.learned_init(seed=5)
    losses = s.learned_train(60, lr=1e-3, seed=1)
    assert np.isfinite(losses).all()
    first = losses[0:3].mean()
    last = losses[-3:].mean()
    assert last < first, (first, last)


def test_learned_fpcg_converges_to_mic0_solution():
    from shiokaze_b200 import native, scenes
    from shiokaze_b200.projection import MacPressureSolver3, grids_from_scene
    sc, s, res_mic = _projected(n=32, seed=2)
    p_mic = s.get_pressure().values.copy()
    s.learned_init(seed=6)
    s.learned_train(90, lr=1e-3, seed=2)
    s.configure({"B200.Preconditioner": "learned", "B200.StallWindow": 8})
    vel, solid, svel, fluid = grids_from_scene(sc)
    res = s.project(sc.dt, vel, solid, svel, fluid)
    assert res["status"] == 0, res
    assert res["reresid"] <= 1e-6
    p = s.get_pressure().values
    assert np.abs(p - p_mic).max() / np.abs(p_mic).max() < 1e-4


def test_each_layer_matches_oracle():
    """Every layer's stored output against the oracle layer applied to the
    GPU's own stored inputs (isolates each convolution and pooling shape)."""
    sc, s, _ = _projected()
    s.learned_init(seed=7)
    rng = np.random.default_rng(2)
    unk = s.get_pressure().active.astype(bool)
    r = np.where(unk, rng.standard_normal(unk.shape), 0).astype(np.float32)
    s.learned_apply(r)
    T = {name: s.learned_tensor(name) for name in s.TENSORS}
    P = _unpack(s.learned_params())
    masks = cn.level_masks(_pool_cells(s, T["X0"].shape[:3]))
    errs = {}
    for name, lvl, in0, in1, cout, relu in cn.LAYERS:
        x = T[in0[0]]
        if in1:
            x = np.concatenate([x, cn._up(T[in1[0]], x.shape)], axis=-1)
        y = cn.conv(x, P[name + ".w"], P[name + ".b"])
        if relu:
            y = np.maximum(y, 0)
        y = y * masks[lvl][..., None]
        got = T[cn.OUTPUT[name]] if name != "out" else T["Z"][..., None]
        errs[name] = float(np.linalg.norm(got - y) / max(np.linalg.norm(y), 1e-30))
    pool1 = cn.avgpool(T["S1"]) * masks[1][..., None]
    pool2 = cn.avgpool(T["S2"]) * masks[2][..., None]
    errs["P1"] = float(np.linalg.norm(T["P1"] - pool1) / np.linalg.norm(pool1))
    errs["P2"] = float(np.linalg.norm(T["P2"] - pool2) / np.linalg.norm(pool2))
    print("per-layer relative errors:", {k: round(v, 5) for k, v in errs.items()})
    assert all(v < 1e-2 for v in errs.values()), errs


def _step_energy(s, r, z):
    """Energy a conjugate-direction step along z removes, -1/2 (z.r)^2 / z.A z,
    over the same quantity for the exact error direction estimate (larger
    magnitude = better direction)."""
    Az = s.apply_matrix(z).astype(np.float64)
    z64, r64 = z.astype(np.float64), r.astype(np.float64)
    return -0.5 * (z64 * r64).sum() ** 2 / (z64 * Az).sum()


def test_training_gains_over_unpreconditioned_direction():
    """What the trained network gains: after training on the system, the step
    along z = N(r) removes more A-norm error from a residual it was not trained
    on than the step along r itself (unpreconditioned CG's direction) and than
    the untrained network's step."""
    sc, s, _ = _projected(n=32, seed=4)
    mask = s.get_pressure().active.astype(bool)
    rng = np.random.default_rng(11)
    r = np.zeros(mask.shape, np.float32)
    r[mask] = rng.standard_normal(mask.sum()).astype(np.float32)
    r = s.apply_matrix(r)  # a residual of a random error: every frequency present
    r /= np.abs(r).max()
    s.learned_init(seed=3)
    e_untrained = _step_energy(s, r, s.learned_apply(r))
    e_identity = _step_energy(s, r, r)
    s.learned_train(150, lr=3e-4, seed=5)
    e_trained = _step_energy(s, r, s.learned_apply(r))
    assert e_trained < e_identity, (e_trained, e_identity)
    assert e_trained < e_untrained, (e_trained, e_untrained)
