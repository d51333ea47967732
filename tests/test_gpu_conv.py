"""The tcgen05 implicit-GEMM 3^3 convolution kernel in isolation, against a
numpy FP32 convolution of the same BF16-rounded operands."""
import numpy as np
import pytest

from oracle import convnet as cn

pytestmark = pytest.mark.gpu


def run_conv(nx, ny, nz, c0, c1, cout, planes, relu=1, seed=0):
    from shiokaze_b200 import native
    rng = np.random.default_rng(seed)
    in0 = cn.bf16(rng.standard_normal((nz, ny, nx, c0)).astype(np.float32))
    in1 = cn.bf16(rng.standard_normal((nz // 2, ny // 2, nx // 2, max(c1, 1))).astype(np.float32)) if c1 else None
    w = cn.bf16((rng.standard_normal((27, cout, c0 + c1)) / np.sqrt(27 * (c0 + c1))).astype(np.float32))
    b = (0.1 * rng.standard_normal(cout)).astype(np.float32)
    out = np.zeros((nz, ny, nx, cout), np.float32)
    L = native.load()
    rc = L.shkz_b200_conv3d(nx, ny, nz, c0, c1, cout, planes, in0.ctypes.data,
                            in1.ctypes.data if c1 else None, w.ctypes.data, b.ctypes.data, relu, out.ctypes.data)
    assert rc == 0
    x = in0 if not c1 else np.concatenate([in0, cn._up(in1, in0.shape)], axis=-1)
    ref = cn.conv(x, w, b)
    if relu:
        ref = np.maximum(ref, 0)
    return out, ref


@pytest.mark.parametrize("shape,c0,c1,cout,planes", [
    ((16, 32, 16), 16, 0, 16, 8),
    ((16, 32, 16), 16, 0, 32, 8),
    ((16, 32, 16), 32, 0, 64, 4),
    ((16, 32, 16), 16, 0, 64, 4),
    ((16, 32, 16), 16, 0, 128, 4),
    ((16, 32, 16), 16, 32, 16, 8),
    ((16, 32, 16), 32, 64, 32, 8),
    ((10, 20, 12), 16, 0, 16, 8),
    ((10, 20, 12), 16, 0, 64, 4),
])
def test_conv_matches_numpy(shape, c0, c1, cout, planes):
    nx, ny, nz = shape
    out, ref = run_conv(nx, ny, nz, c0, c1, cout, planes)
    err = np.linalg.norm(out - ref) / np.linalg.norm(ref)
    assert err < 1e-2, err
