"""CPU restatement of the learned preconditioner network (numpy).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA network kernels (forward,
input/weight gradients, Adam). The product never imports it.

Network (3 levels, 16/32/64 channels, 3^3 kernels, ReLU, BF16 activations and
weights, FP32 accumulation):

    X0 (16 ch: r/s, phi/dx, solid fraction, 13 zero channels)      level 0
    e1a 16->16, e1b 16->16 = S1                                      level 0
    P1 = avgpool2(S1); e2a 16->32, e2b 32->32 = S2                   level 1
    P2 = avgpool2(S2); e3a 32->64, e3b 64->64 = B3                   level 2
    d2a [S2, up(B3)] 96->32, d2b 32->32 = D2                         level 1
    d1a [S1, up(D2)] 48->16, d1b 16->16 = D1                         level 0
    out 16->1 (no ReLU, FP32)                                        level 0

Tensors are dense channels-last arrays (z, y, x, C) per level; level l has
half the extent of level l-1. Activity is per block of 8 (x) x 16 (y) x 8 (z)
voxels of each level; every layer writes zeros outside active blocks, so the
network is defined on the active region only. A 3^3 convolution reads zeros
outside the grid. Tap t = (dz+1)*9 + (dy+1)*3 + (dx+1). up() is nearest
upsampling (voxel v reads v >> 1).
"""
from __future__ import annotations

import numpy as np

LAYERS = [
    # name, level, in0 (name, channels), in1 (name, channels) or None, cout, relu
    ("e1a", 0, ("X0", 16), None, 16, True),
    ("e1b", 0, ("A1", 16), None, 16, True),
    ("e2a", 1, ("P1", 16), None, 32, True),
    ("e2b", 1, ("A2", 32), None, 32, True),
    ("e3a", 2, ("P2", 32), None, 64, True),
    ("e3b", 2, ("A3", 64), None, 64, True),
    ("d2a", 1, ("S2", 32), ("B3", 64), 32, True),
    ("d2b", 1, ("C2", 32), None, 32, True),
    ("d1a", 0, ("S1", 16), ("D2", 32), 16, True),
    ("d1b", 0, ("C1", 16), None, 16, True),
    ("out", 0, ("D1", 16), None, 1, False),
]
OUTPUT = {"e1a": "A1", "e1b": "S1", "e2a": "A2", "e2b": "S2", "e3a": "A3", "e3b": "B3",
          "d2a": "C2", "d2b": "D2", "d1a": "C1", "d1b": "D1", "out": "Z"}
BLOCK = (8, 16, 8)  # x, y, z voxels per activity block


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 to bfloat16 (nearest even), returned as float32."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def init_params(seed: int = 0) -> dict:
    """He-normal weights rounded to BF16, zero biases; W[name] is (27, cout, cin)."""
    rng = np.random.default_rng(seed)
    P = {}
    for name, lvl, in0, in1, cout, relu in LAYERS:
        cin = in0[1] + (in1[1] if in1 else 0)
        fan_in = 27 * (3 if name == "e1a" else cin)
        w = rng.standard_normal((27, cout, cin)).astype(np.float32) * np.float32(np.sqrt(2.0 / fan_in))
        if name == "e1a":
            w[:, :, 3:] = 0.0
        if name == "out":
            w *= 0.1
        P[name + ".w"] = bf16(w)
        P[name + ".b"] = np.zeros(cout, np.float32)
    return P


def level_masks(pool_cells: np.ndarray) -> list:
    """Voxel activity masks (z, y, x) for the three levels from a level-0 cell
    mask (True where the cell belongs to a tile of the pool)."""
    masks = []
    nz, ny, nx = pool_cells.shape
    for lvl in range(3):
        f = 2 ** lvl
        bx, by, bz = BLOCK[0] * f, BLOCK[1] * f, BLOCK[2] * f
        gx, gy, gz = -(-nx // bx), -(-ny // by), -(-nz // bz)
        pad = np.zeros((gz * bz, gy * by, gx * bx), bool)
        pad[:nz, :ny, :nx] = pool_cells
        act = pad.reshape(gz, bz, gy, by, gx, bx).any(axis=(1, 3, 5))
        vox = np.repeat(np.repeat(np.repeat(act, BLOCK[2], 0), BLOCK[1], 1), BLOCK[0], 2)
        lz, ly, lx = nz // f, ny // f, nx // f
        masks.append(vox[:lz, :ly, :lx])
    return masks


def _shift(x: np.ndarray, dz: int, dy: int, dx: int) -> np.ndarray:
    """out[v] = x[v + d] with zeros outside."""
    out = np.zeros_like(x)
    nz, ny, nx = x.shape[:3]
    zs, ze = max(0, -dz), nz - max(0, dz)
    ys, ye = max(0, -dy), ny - max(0, dy)
    xs, xe = max(0, -dx), nx - max(0, dx)
    out[zs:ze, ys:ye, xs:xe] = x[zs + dz:ze + dz, ys + dy:ye + dy, xs + dx:xe + dx]
    return out


def _up(x: np.ndarray, shape) -> np.ndarray:
    return np.repeat(np.repeat(np.repeat(x, 2, 0), 2, 1), 2, 2)[:shape[0], :shape[1], :shape[2]]


def _taps():
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                yield (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1), dz, dy, dx


def conv(xcat: np.ndarray, w: np.ndarray, b: np.ndarray) -> np.ndarray:
    """FP32 3^3 convolution, xcat (z,y,x,cin), w (27,cout,cin) -> (z,y,x,cout)."""
    out = np.zeros(xcat.shape[:3] + (w.shape[1],), np.result_type(xcat, w))
    for t, dz, dy, dx in _taps():
        out += np.einsum("zyxc,oc->zyxo", _shift(xcat, dz, dy, dx), w[t], optimize=True)
    return out + b


def avgpool(x: np.ndarray) -> np.ndarray:
    nz, ny, nx, c = x.shape
    return x.reshape(nz // 2, 2, ny // 2, 2, nx // 2, 2, c).mean(axis=(1, 3, 5))


def forward(P: dict, X0: np.ndarray, masks: list, keep: bool = False):
    """Network output Z (z,y,x) in FP32 from X0 (z,y,x,16); BF16 rounding of
    every stored activation, as the GPU stores them."""
    T = {"X0": bf16(X0 * masks[0][..., None])}
    pre = {}
    for name, lvl, in0, in1, cout, relu in LAYERS:
        if name == "e2a":
            T["P1"] = bf16(avgpool(T["S1"]) * masks[1][..., None])
        if name == "e3a":
            T["P2"] = bf16(avgpool(T["S2"]) * masks[2][..., None])
        x = T[in0[0]]
        if in1:
            x = np.concatenate([x, _up(T[in1[0]], x.shape)], axis=-1)
        y = conv(x, P[name + ".w"], P[name + ".b"])
        pre[name] = y
        if relu:
            y = np.maximum(y, 0.0)
        y = y * masks[lvl][..., None]
        T[OUTPUT[name]] = y if name == "out" else bf16(y)
    Z = T["Z"][..., 0]
    return (Z, T, pre) if keep else Z


def backward(P: dict, T: dict, pre: dict, masks: list, gZ: np.ndarray, tensor_grads: dict | None = None) -> dict:
    """Gradients of sum(gZ * Z) w.r.t. all weights and biases (FP32). If
    tensor_grads is given it receives the gradient w.r.t. every stored
    activation (after the ReLU, before masking), as accumulated."""
    G = {"Z": gZ[..., None] * masks[0][..., None]}
    grads = {}
    for name, lvl, in0, in1, cout, relu in reversed(LAYERS):
        g = G.pop(OUTPUT[name])
        if tensor_grads is not None:
            tensor_grads[OUTPUT[name]] = np.array(g)
        if relu:
            g = g * (pre[name] > 0)
        g = g * masks[lvl][..., None]
        x = T[in0[0]]
        c0 = in0[1]
        if in1:
            x = np.concatenate([x, _up(T[in1[0]], x.shape)], axis=-1)
        w = P[name + ".w"]
        gw = np.zeros_like(w)
        gx = np.zeros(x.shape, np.result_type(x, g))
        for t, dz, dy, dx in _taps():
            xs = _shift(x, dz, dy, dx)
            gw[t] = np.einsum("zyxo,zyxc->oc", g, xs, optimize=True)
            gx += _shift(np.einsum("zyxo,oc->zyxc", g, w[t], optimize=True), -dz, -dy, -dx)
        grads[name + ".w"] = gw
        grads[name + ".b"] = g.sum(axis=(0, 1, 2))
        g0 = gx[..., :c0]
        G[in0[0]] = G.get(in0[0], 0) + g0
        if in1:
            g1 = gx[..., c0:]
            nz, ny, nx = T[in1[0]].shape[:3]
            pad = np.zeros((2 * nz, 2 * ny, 2 * nx, g1.shape[-1]), g1.dtype)
            pad[:g1.shape[0], :g1.shape[1], :g1.shape[2]] = g1
            G[in1[0]] = G.get(in1[0], 0) + pad.reshape(nz, 2, ny, 2, nx, 2, -1).sum(axis=(1, 3, 5))
        if name == "e2a":
            if tensor_grads is not None:
                tensor_grads["P1"] = np.array(G["P1"])
            gp = G.pop("P1") * masks[1][..., None]
            G["S1"] = G.get("S1", 0) + np.repeat(np.repeat(np.repeat(gp, 2, 0), 2, 1), 2, 2) / 8.0
        if name == "e3a":
            if tensor_grads is not None:
                tensor_grads["P2"] = np.array(G["P2"])
            gp = G.pop("P2") * masks[2][..., None]
            G["S2"] = G.get("S2", 0) + np.repeat(np.repeat(np.repeat(gp, 2, 0), 2, 1), 2, 2) / 8.0
    return grads


def adam(P: dict, grads: dict, state: dict, lr: float = 1e-3, b1: float = 0.9, b2: float = 0.999,
         eps: float = 1e-8, master: dict | None = None) -> dict:
    """One Adam step on FP32 master weights; returns the BF16-rounded weights."""
    state["t"] = state.get("t", 0) + 1
    t = state["t"]
    out = {}
    for k, g in grads.items():
        m = state.setdefault("m." + k, np.zeros_like(g))
        v = state.setdefault("v." + k, np.zeros_like(g))
        m[...] = b1 * m + (1 - b1) * g
        v[...] = b2 * v + (1 - b2) * g * g
        mh = m / (1 - b1 ** t)
        vh = v / (1 - b2 ** t)
        w = master[k] if master is not None else P[k]
        w = w - lr * mh / (np.sqrt(vh) + eps)
        if master is not None:
            master[k] = w
        out[k] = bf16(w) if k.endswith(".w") else w.astype(np.float32)
    return out
