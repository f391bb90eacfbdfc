"""smadft_r2r3d_noalloc against smadft_r2r3d_device, through the C ABI.

smadft_r2r3d_noalloc is the 3-D r2r transform for callers that cannot allocate device
memory (device memory fully reserved up front by another allocator, fixed-latency loops that
must not hit cudaMalloc's implicit synchronisation).  Its intermediate field and its twiddle
tables live in fixed device arrays shared by all calls, so these tests run calls in a row
(different shapes and inputs, each reusing what the one before left in the arrays) and
compare each with the context-based entry point at the tolerances the transform tests use:
at the size limit itself, in place (in == out) on a non-default stream, and the rejected
lengths.

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


def noalloc_transform(shape, kinds, precision, x, in_place=False, side_stream=False):
    import torch
    dt = torch.float64 if precision == smadft.FP64 else torch.float32
    src = torch.from_numpy(x).to("cuda", dt).contiguous()
    dst = src if in_place else torch.empty_like(src)
    torch.cuda.synchronize()
    s = torch.cuda.Stream() if side_stream else torch.cuda.current_stream()
    with torch.cuda.stream(s):
        rc = smadft.r2r3d_noalloc(src.data_ptr(), dst.data_ptr(), shape, kinds, precision, s.cuda_stream)
    s.synchronize()
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


@pytest.mark.parametrize("precision", [smadft.FP64, smadft.FP32], ids=["fp64", "fp32"])
def test_noalloc_at_the_limit_in_place_on_a_side_stream(precision):
    """The largest grid the scratch array holds (128^3 doubles are exactly
    SMADFT_NOALLOC_MAX_BYTES; for FP32 the same grid is half of it), then a smaller transform
    in place (in == out) on a non-default stream, then the limit grid again in place."""
    calls = [((128, 128, 128), (0, 0, 1), False, False),
             ((32, 40, 48), (3, 2, 1), True, True),
             ((128, 128, 128), (1, 3, 2), True, True)]
    assert 128 ** 3 * 8 == smadft.NOALLOC_MAX_BYTES
    for n, (shape, kinds, in_place, side) in enumerate(calls):
        x = np.random.default_rng(200 + n).standard_normal(shape)
        want = reference_transform(shape, kinds, precision, x)
        got = noalloc_transform(shape, kinds, precision, x, in_place=in_place, side_stream=side)
        assert np.max(np.abs(got - want)) <= TOL[precision] * np.max(np.abs(want)), (n, shape)


def test_noalloc_rejects_unsupported_lengths():
    """Lengths with a factor 7, odd lengths and lengths above 512 are refused before any work."""
    import torch
    a = torch.empty(1 << 16, device="cuda", dtype=torch.float64)
    for shape in [(14, 16, 16), (16, 15, 16), (16, 16, 1024), (2, 16, 16)]:
        rc = smadft.r2r3d_noalloc(a.data_ptr(), a.data_ptr(), shape, (0, 0, 0), smadft.FP64)
        assert rc == -6, shape
