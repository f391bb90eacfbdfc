"""GPU axis-pass r2r transforms against the oracle (through smadft_r2r3d_device).

Tolerances: FP64 1e-13 and FP32 3e-6 of max|ref|.
"""
import numpy as np
import pytest

import oracle
import smadft

pytestmark = pytest.mark.gpu

KINDS = [(0, 0, 0), (1, 1, 1), (2, 0, 0), (0, 2, 0), (0, 0, 2), (3, 1, 1), (1, 3, 1), (1, 1, 3),
         (2, 2, 2), (3, 3, 3)]
SHAPES = [(16, 12, 20), (64, 64, 64), (96, 32, 160), (8, 30, 10), (40, 24, 48), (128, 64, 40),
          (64, 128, 50), (256, 64, 32),
          (12, 64, 64), (20, 128, 128), (6, 256, 256),
          # register-direct z kernel with a partial last tile (nx * ny not a multiple of 32)
          (6, 10, 64), (4, 10, 256), (10, 6, 128)]


def run_device(shape, kinds, precision, x):
    import torch
    p = smadft.params(smadft.NOADV, shape, precision=precision)
    dt = torch.float64 if precision == smadft.FP64 else torch.float32
    with smadft.Solver(p) as s:
        xin = torch.from_numpy(x).to("cuda", dt).contiguous()
        xout = torch.empty_like(xin)
        s.r2r3d_device(xin.data_ptr(), xout.data_ptr(), kinds)
        s.sync()
        return xout.double().cpu().numpy()


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "x".join(map(str, s)))
@pytest.mark.parametrize("kinds", KINDS, ids=lambda k: "".join(map(str, k)))
@pytest.mark.parametrize("precision,tol", [(smadft.FP64, 1e-13), (smadft.FP32, 3e-6)], ids=["fp64", "fp32"])
def test_r2r3d_matches_oracle(shape, kinds, precision, tol):
    x = np.random.default_rng(hash(shape) % 1000).standard_normal(shape)
    ref = oracle.r2r_3d(x, kinds)
    got = run_device(shape, kinds, precision, x)
    assert np.max(np.abs(got - ref)) <= tol * np.max(np.abs(ref))


@pytest.mark.parametrize("shape", [(12, 64, 64), (20, 128, 128), (6, 256, 256)], ids=lambda s: "x".join(map(str, s)))
@pytest.mark.parametrize("precision", [smadft.FP64, smadft.FP32], ids=["fp64", "fp32"])
def test_plane_kernel_matches_separate_passes(shape, precision, monkeypatch):
    """The fused z + y plane kernel and the three separate axis passes agree (SMADFT_PLANE)."""
    x = np.random.default_rng(17).standard_normal(shape)
    kinds = (0, 3, 2)
    got = {}
    for flag in ("1", "0"):
        monkeypatch.setenv("SMADFT_PLANE", flag)
        got[flag] = run_device(shape, kinds, precision, x)
    tol = 1e-13 if precision == smadft.FP64 else 3e-6
    assert np.max(np.abs(got["1"] - got["0"])) <= tol * np.max(np.abs(got["0"]))


@pytest.mark.parametrize("shape", [(8, 8, 64), (6, 10, 128), (4, 16, 256), (60, 250, 256)],
                         ids=lambda s: "x".join(map(str, s)))
@pytest.mark.parametrize("precision", [smadft.FP64, smadft.FP32], ids=["fp64", "fp32"])
@pytest.mark.parametrize("kinds", [(0, 0, 0), (1, 1, 1), (2, 2, 2), (3, 3, 3)], ids=lambda k: "".join(map(str, k)))
def test_rdz_kernel_matches_staged_z(shape, precision, kinds, monkeypatch):
    """Register-direct z kernel against the staged z kernel (SMADFT_RDZ=0), all four kinds,
    partial last tiles included."""
    x = np.random.default_rng(23).standard_normal(shape)
    got = {}
    for flag in ("1", "0"):
        monkeypatch.setenv("SMADFT_RDZ", flag)
        got[flag] = run_device(shape, kinds, precision, x)
    tol = 1e-13 if precision == smadft.FP64 else 3e-6
    assert np.max(np.abs(got["1"] - got["0"])) <= tol * np.max(np.abs(got["0"]))


def test_r2r3d_in_place_and_roundtrip():
    import torch
    shape = (32, 24, 40)
    x = np.random.default_rng(5).standard_normal(shape)
    p = smadft.params(smadft.NOADV, shape)
    with smadft.Solver(p) as s:
        t = torch.from_numpy(x).cuda()
        s.r2r3d_device(t.data_ptr(), t.data_ptr(), (0, 0, 0))
        s.r2r3d_device(t.data_ptr(), t.data_ptr(), (1, 1, 1))
        s.sync()
        back = t.cpu().numpy() / (8.0 * 32 * 24 * 40)
    assert np.max(np.abs(back - x)) <= 1e-13 * np.max(np.abs(x))
