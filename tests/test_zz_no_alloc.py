"""vox_mv_AN_noalloc: the matvec entry point that allocates nothing.

It is meant for callers that cannot call cudaMalloc where they need the
product (an external memory manager owns all device memory, or allocation is
forbidden in that region).  The test calls it through the C-ABI on device
buffers and checks it against the existing vox_mv_AN_device on two calls in a
row, in both precisions and both products (A and A'), once on a caller's
stream, and that an operator whose intermediates exceed the fixed 64 MiB
array is refused.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

import voxphoton_b200 as vb
from voxphoton_b200 import _lib

pytestmark = pytest.mark.gpu

TOL = {"c128": 1e-12, "c64": 1e-5}


def _op(shape, seed):
    rng = np.random.default_rng(seed)
    L, M, N = shape
    G = rng.standard_normal((L, M, N, 6)) + 1j * rng.standard_normal((L, M, N, 6))
    G[0, :, :, 1:3] = 0
    Mc = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    idx = np.arange(1, 3 * L * M * N + 1)
    return vb.Operator(Mc, 0.8, idx, G=G)


def _call(fn, op, prec, x, y, transp=0, stream=None):
    import torch
    torch.cuda.synchronize()
    _lib.check(fn(op.handle, transp, _lib.PREC[prec], ctypes.c_void_p(x.data_ptr()),
                  ctypes.c_void_p(y.data_ptr()),
                  None if stream is None else ctypes.c_void_p(stream.cuda_stream)))
    torch.cuda.synchronize()


@pytest.mark.parametrize("transp", [0, 1])
@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_noalloc_matches_device_entry_point_twice(prec, transp):
    import torch
    op = _op((20, 9, 6), 0)
    lib = _lib.lib()
    dt = torch.complex128 if prec == "c128" else torch.complex64
    g = torch.Generator(device="cuda").manual_seed(0)
    for _ in range(2):
        x = torch.randn(op.n, dtype=dt, device="cuda", generator=g)
        ref = torch.empty_like(x)
        out = torch.full_like(x, float("nan"))
        _call(lib.vox_mv_AN_device, op, prec, x, ref, transp)
        _call(lib.vox_mv_AN_noalloc, op, prec, x, out, transp)
        err = (torch.linalg.vector_norm(out - ref) / torch.linalg.vector_norm(ref)).item()
        assert err < TOL[prec], err
    op.close()


def test_noalloc_on_a_caller_stream():
    """The product enqueued on a non-default torch stream passed as the stream
    argument equals the device entry point's."""
    import torch
    op = _op((20, 9, 6), 2)
    lib = _lib.lib()
    x = torch.randn(op.n, dtype=torch.complex64, device="cuda")
    ref = torch.empty_like(x)
    out = torch.full_like(x, float("nan"))
    s = torch.cuda.Stream()
    _call(lib.vox_mv_AN_device, op, "c64", x, ref)
    _call(lib.vox_mv_AN_noalloc, op, "c64", x, out, 0, s)
    err = (torch.linalg.vector_norm(out - ref) / torch.linalg.vector_norm(ref)).item()
    assert err < TOL["c64"], err
    op.close()


def test_noalloc_refuses_operators_beyond_the_fixed_scratch():
    import torch
    op = _op((1160, 30, 11), 1)  # complex128 intermediates: 2 x 2560 x 990 x 16 B > 64 MiB
    x = torch.zeros(op.n, dtype=torch.complex128, device="cuda")
    y = torch.empty_like(x)
    with pytest.raises(_lib.VoxError) as e:
        _call(_lib.lib().vox_mv_AN_noalloc, op, "c128", x, y)
    assert "maximum" in str(e.value)
    # the complex64 copy of the same operator fits (2 x 2560 x 990 x 8 B)
    xf = torch.randn(op.n, dtype=torch.complex64, device="cuda")
    ref = torch.empty_like(xf)
    out = torch.empty_like(xf)
    _call(_lib.lib().vox_mv_AN_device, op, "c64", xf, ref)
    _call(_lib.lib().vox_mv_AN_noalloc, op, "c64", xf, out)
    assert (torch.linalg.vector_norm(out - ref) / torch.linalg.vector_norm(ref)).item() < 1e-5
    op.close()
