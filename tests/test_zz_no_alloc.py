"""shkz_b200_conv3d_noalloc: the tensor-core convolution for callers that
cannot allocate device memory (an application that owns the whole GPU through
its own allocator, or a loop that must not pay cudaMalloc's device-wide
synchronisation). Its scratch is a fixed array inside the library; the caller
passes device inputs and outputs only. Checked against the allocating entry
point shkz_b200_conv3d on the same data, on two calls in a row (the second
call reuses the array's contents from the first). This file is collected last
on purpose."""
import numpy as np
import pytest

from oracle import convnet as cn

pytestmark = pytest.mark.gpu

TOL = 1e-2  # relative, as for the convolution kernel's own tests


def _bits(a):
    return (np.ascontiguousarray(a, np.float32).view(np.uint32) >> 16).astype(np.uint16)


def _floats(b):
    return (np.ascontiguousarray(b, np.uint16).astype(np.uint32) << 16).view(np.float32)


def test_no_alloc_conv_matches_allocating_entry_point():
    import torch
    from shiokaze_b200 import native
    L = native.load()
    nx, ny, nz, c0, c1, cout, planes = 16, 32, 16, 16, 32, 32, 8
    rng = np.random.default_rng(11)
    in0 = cn.bf16(rng.standard_normal((nz, ny, nx, c0)).astype(np.float32))
    in1 = cn.bf16(rng.standard_normal((nz // 2, ny // 2, nx // 2, c1)).astype(np.float32))
    w = cn.bf16((rng.standard_normal((27, cout, c0 + c1)) / np.sqrt(27 * (c0 + c1))).astype(np.float32))
    b = (0.1 * rng.standard_normal(cout)).astype(np.float32)
    ref = np.zeros((nz, ny, nx, cout), np.float32)
    assert L.shkz_b200_conv3d(nx, ny, nz, c0, c1, cout, planes, in0.ctypes.data, in1.ctypes.data, w.ctypes.data,
                              b.ctypes.data, 1, ref.ctypes.data) == 0
    dev = torch.device("cuda", 0)
    d_in0 = torch.from_numpy(_bits(in0).view(np.int16)).to(dev)
    d_in1 = torch.from_numpy(_bits(in1).view(np.int16)).to(dev)
    d_w = torch.from_numpy(w).to(dev)
    d_b = torch.from_numpy(b).to(dev)
    d_out = torch.zeros((nz, ny, nx, cout), dtype=torch.int16, device=dev)
    torch.cuda.synchronize(dev)
    for call in range(2):
        d_out.zero_()
        torch.cuda.synchronize(dev)
        rc = L.shkz_b200_conv3d_noalloc(nx, ny, nz, c0, c1, cout, planes, d_in0.data_ptr(), d_in1.data_ptr(),
                                        d_w.data_ptr(), d_b.data_ptr(), 1, d_out.data_ptr(), None)
        assert rc == 0, (call, rc)
        got = _floats(d_out.cpu().numpy().view(np.uint16))
        err = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
        assert err <= TOL, (call, err)


def test_no_alloc_rejects_sizes_beyond_the_limit():
    from shiokaze_b200 import native
    L = native.load()
    # cout 256 and c0 + c1 = 144 exceed the fixed scratch; rejected before any GPU work
    dummy = np.zeros(16, np.float32)
    p = dummy.ctypes.data
    assert L.shkz_b200_conv3d_noalloc(16, 16, 16, 16, 0, 256, 4, p, None, p, None, 1, p, None) == -8
    assert L.shkz_b200_conv3d_noalloc(16, 16, 16, 128, 16, 16, 8, p, p, p, None, 1, p, None) == -8
