"""CPU restatement of the velocity extension the reference runs right after a
projection (macliquid3::extend_both, src/liquid/macliquid3.cpp:330-340).

TEST INFRASTRUCTURE ONLY: the product never imports this module. It is the
checker of the device kernels in ``shiokaze_b200/csrc/extend.cu`` and is
itself pinned bit-exact against the compiled reference (``HarnessExtend`` /
``HarnessConstrain`` of ``oracle/ref/harness.cpp``).

Arrays are dense numpy grids indexed [k, j, i] (x fastest in memory); a face
component d has shape (nz + (d == 2), ny + (d == 1), nx + (d == 0)), the solid
level set is nodal (nz + 1, ny + 1, nx + 1) holding the values the reference's
array3 returns (active value, fill value or background). The arithmetic
follows the reference's types step by step: FP32 sums where it stores into
``Real`` (float), FP64 where it computes in double.
"""
from __future__ import annotations

import numpy as np

# neighbour query order of array_extrapolator3::extrapolate_if
# (include/shiokaze/array/array_extrapolator3.h, the query[] list):
# (i+1), (i-1), (j+1), (j-1), (k-1), (k+1) as (di, dj, dk)
_QUERY = ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, -1), (0, 0, 1))


def _shift(a: np.ndarray, di: int, dj: int, dk: int, fill):
    """out[k, j, i] = a[k + dk, j + dj, i + di], fill outside the grid."""
    out = np.full_like(a, fill)
    D, H, W = a.shape
    src = [slice(max(0, d), n + min(0, d)) for d, n in ((dk, D), (dj, H), (di, W))]
    dst = [slice(max(0, -d), n - max(0, d)) for d, n in ((dk, D), (dj, H), (di, W))]
    out[tuple(dst)] = a[tuple(src)]
    return out


def extrapolate_component(v: np.ndarray, act: np.ndarray, width: int):
    """array_extrapolator3::extrapolate(array, width): ``width`` passes of
    array3::dilate (src/array/dilate3.h): every inactive in-grid cell with an
    active 6-neighbour (in the state before the pass) becomes active with the
    FP32 mean of its active neighbours, summed in the query order above."""
    v = v.astype(np.float32).copy()
    act = act.astype(bool).copy()
    for _ in range(width):
        s = np.zeros_like(v)
        w = np.zeros(v.shape, np.int32)
        for di, dj, dk in _QUERY:
            m = _shift(act, di, dj, dk, False)
            sv = _shift(v, di, dj, dk, np.float32(0))
            s = np.where(m, s + sv, s).astype(np.float32)
            w += m
        new = (~act) & (w > 0)
        v[new] = (s[new] / w[new].astype(np.float32)).astype(np.float32)
        act |= new
    return v, act


def extrapolate(vel: list, vact: list, width: int):
    """macarray_extrapolator3::extrapolate: each component on its own."""
    out = [extrapolate_component(vel[d], vact[d], width) for d in range(3)]
    return [o[0] for o in out], [o[1] for o in out]


def _interp_coef(shape_whd, p):
    """array_interpolator3::interpolate_coef for arrays of points p (N x 3,
    index space): corner indices (N x 8 x 3) and FP64 weights (N x 8)."""
    W, H, D = shape_whd
    x = np.maximum(0.0, np.minimum(W - 1.0, p[:, 0]))
    y = np.maximum(0.0, np.minimum(H - 1.0, p[:, 1]))
    z = np.maximum(0.0, np.minimum(D - 1.0, p[:, 2]))
    i = np.minimum(x, W - 2.0).astype(np.int64)
    j = np.minimum(y, H - 2.0).astype(np.int64)
    k = np.minimum(z, D - 2.0).astype(np.int64)
    fi, fj, fk = i.astype(np.float64), j.astype(np.float64), k.astype(np.float64)
    ax, bx = (fi + 1) - x, x - fi
    ay, by = (fj + 1) - y, y - fj
    az, bz = (fk + 1) - z, z - fk
    idx = np.stack([np.stack([i + (n & 1), j + ((n >> 1) & 1), k + (n >> 2)], 1) for n in range(8)], 1)
    coef = np.stack([az * ax * ay, az * bx * ay, az * ax * by, az * bx * by,
                     bz * ax * ay, bz * bx * ay, bz * ax * by, bz * bx * by], 1)
    deriv = [np.stack([-az * ay, az * ay, -az * by, az * by, -bz * ay, bz * ay, -bz * by, bz * by], 1),
             np.stack([-az * ax, -az * bx, az * ax, az * bx, -bz * ax, -bz * bx, bz * ax, bz * bx], 1),
             np.stack([-ax * ay, -bx * ay, -ax * by, -bx * by, ax * ay, bx * ay, ax * by, bx * by], 1)]
    return idx, coef, deriv


def _gather(a: np.ndarray, idx: np.ndarray) -> np.ndarray:
    return a[idx[..., 2], idx[..., 1], idx[..., 0]]


def _interpolate(a: np.ndarray, p: np.ndarray) -> np.ndarray:
    """array_interpolator3::interpolate (only_actives false): FP32 value,
    ``value += array(corner) * coef`` in FP64 per corner with a non-zero
    weight, rounded to FP32 after each addition."""
    D, H, W = a.shape
    idx, coef, _ = _interp_coef((W, H, D), p)
    vals = _gather(a, idx).astype(np.float64)
    out = np.zeros(p.shape[0], np.float32)
    for n in range(8):
        c = coef[:, n]
        out = np.where(c != 0.0, (out.astype(np.float64) + vals[:, n] * c).astype(np.float32), out)
    return out


def _derivative(a: np.ndarray, p: np.ndarray) -> np.ndarray:
    """array_derivative3::derivative: FP32 gradient (index space), each term
    ``coef * array(corner)`` in FP64 added to the FP32 result."""
    D, H, W = a.shape
    idx, _, deriv = _interp_coef((W, H, D), p)
    vals = _gather(a, idx).astype(np.float64)
    out = np.zeros((p.shape[0], 3), np.float32)
    for d in range(3):
        r = np.zeros(p.shape[0], np.float32)
        for n in range(8):
            r = (r.astype(np.float64) + deriv[d][:, n] * vals[:, n]).astype(np.float32)
        out[:, d] = r
    return out


def constrain_velocity(vel: list, vact: list, solid: np.ndarray, solid_active: np.ndarray, dx: float):
    """macutility3::constrain_velocity (src/utility/macutility3.cpp:61-92)."""
    nz, ny, nx = solid.shape[0] - 1, solid.shape[1] - 1, solid.shape[2] - 1
    save = [np.where(vact[d], vel[d], np.float32(0)).astype(np.float32) for d in range(3)]
    out = [vel[d].astype(np.float32).copy() for d in range(3)]
    # levelset_exist(solid): an active node with a negative value
    # (include/shiokaze/array/array_utility3.h:112-123)
    if np.any(solid_active.astype(bool) & (solid < 0)):
        for d in range(3):
            kk, jj, ii = np.nonzero(vact[d])
            p = np.stack([ii + 0.5 * (d != 0), jj + 0.5 * (d != 1), kk + 0.5 * (d != 2)], 1).astype(np.float64)
            inside = _interpolate(solid, p) < 0.0
            if not inside.any():
                continue
            p, ii, jj, kk = p[inside], ii[inside], jj[inside], kk[inside]
            normal = _derivative(solid, p).astype(np.float64) / dx
            norm2 = normal[:, 0] * normal[:, 0] + normal[:, 1] * normal[:, 1] + normal[:, 2] * normal[:, 2]
            # macarray_interpolator3::interpolate of the saved field at p
            u = np.stack([_interpolate(save[c], p - 0.5 * np.array([c != 0, c != 1, c != 2], np.float64))
                          for c in range(3)], 1).astype(np.float64)
            un = u[:, 0] * normal[:, 0] + u[:, 1] * normal[:, 1] + u[:, 2] * normal[:, 2]
            sel = (norm2 != 0.0) & (un < 0.0)
            newv = (u[:, d] - normal[:, d] * un).astype(np.float32)
            out[d][kk[sel], jj[sel], ii[sel]] = newv[sel]
    # floor and ceiling of the domain: no flow out through y
    a1 = vact[1].astype(bool)
    v1 = out[1]
    lo, hi = v1[:, 0, :], v1[:, ny, :]
    lo[a1[:, 0, :] & (lo < 0)] = np.float32(0)
    hi[a1[:, ny, :] & (hi > 0)] = np.float32(0)
    return out


def extend(vel: list, vact: list, solid, solid_active, dx: float, width: int, constrain: bool = True):
    """extrapolate ``width`` layers, then constrain_velocity (when asked)."""
    v, a = extrapolate(vel, vact, width)
    if constrain:
        if solid is None:
            solid = np.ones((vel[0].shape[0] + 1, vel[0].shape[1] + 1, vel[0].shape[2]), np.float32)
            solid_active = np.zeros(solid.shape, np.uint8)
        v = constrain_velocity(v, a, solid, solid_active, dx)
    return v, a
