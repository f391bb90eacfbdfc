"""smadft_r2r3d_noalloc against smadft_r2r3d_device, through the C ABI.

smadft_r2r3d_noalloc is the 3-D r2r transform for callers that cannot allocate device
memory (stream callbacks, memory fully reserved by another allocator, fixed-latency loops
that must not hit cudaMalloc's implicit synchronisation).  Its intermediate field lives in a
fixed device array shared by all calls, so this test runs two calls in a row (different
shapes and inputs, the second reusing what the first left in the array) and compares each
with the context-based entry point at the tolerances the transform tests use.

The file is named to be collected last, so a run that stops at the first failure has
already run every other test; it also passes on its own in a fresh process.
"""
import numpy as np
import pytest

import smadft

pytestmark = pytest.mark.gpu

TOL = {smadft.FP64: 1e-13, smadft.FP32: 3e-6}


def reference_transform(shape, kinds, precision, x):
    import torch
    dt = torch.float64 if precision == smadft.FP64 else torch.float32
    with smadft.Solver(smadft.params(smadft.NOADV, shape, precision=precision)) as s:
        src = torch.from_numpy(x).to("cuda", dt).contiguous()
        dst = torch.empty_like(src)
        torch.cuda.synchronize()
        s.r2r3d_device(src.data_ptr(), dst.data_ptr(), kinds)
        s.sync()
        return dst.double().cpu().numpy()


def noalloc_transform(shape, kinds, precision, x):
    import torch
    dt = torch.float64 if precision == smadft.FP64 else torch.float32
    src = torch.from_numpy(x).to("cuda", dt).contiguous()
    dst = torch.empty_like(src)
    stream = torch.cuda.current_stream().cuda_stream
    rc = smadft.r2r3d_noalloc(src.data_ptr(), dst.data_ptr(), shape, kinds, precision, stream)
    torch.cuda.synchronize()
    assert rc == 0, rc
    return dst.double().cpu().numpy()


@pytest.mark.parametrize("precision", [smadft.FP64, smadft.FP32], ids=["fp64", "fp32"])
def test_noalloc_matches_context_transform_twice(precision):
    calls = [((64, 96, 128), (0, 2, 1)),      # compile-time-length kernels
             ((24, 20, 30), (1, 3, 0))]       # generic kernel, smaller: reuses the scratch
    for n, (shape, kinds) in enumerate(calls):
        x = np.random.default_rng(100 + n).standard_normal(shape)
        want = reference_transform(shape, kinds, precision, x)
        got = noalloc_transform(shape, kinds, precision, x)
        scale = np.max(np.abs(want))
        assert np.max(np.abs(got - want)) <= TOL[precision] * scale, (n, shape)


def test_noalloc_rejects_grids_beyond_its_scratch():
    import torch
    shape = (160, 160, 160)          # 32 MiB of doubles > SMADFT_NOALLOC_MAX_BYTES
    a = torch.empty(shape, device="cuda", dtype=torch.float64)
    rc = smadft.r2r3d_noalloc(a.data_ptr(), a.data_ptr(), shape, (0, 0, 0), smadft.FP64)
    assert rc == -10
    assert smadft.lib().smadft_error_string(-10) == b"grid exceeds the no-alloc scratch maximum"
    assert 160 ** 3 * 8 > smadft.NOALLOC_MAX_BYTES
