"""GEMM-form z pass on the tensor cores (tcgen05, r2r_gemm.cuh) against FFTW's r2r definitions.

With SMADFT_GEMM_Z=1 an FP32 context runs its plain z passes of length 128 and 256 as
block-matrix products on the tensor cores (FP16 hi/lo operands, FP32 accumulation) instead
of the FFT-form pass.  The reference is scipy.fft's DCT/DST of types 2 and 3 with
norm=None along z, whose definitions are FFTW's REDFT10/REDFT01/RODFT10/RODFT01 (the oracle's
r2r is pinned to them in tests/test_oracle_r2r.py).  Tolerance: the FP32 pass bar of the
transform tests, 3e-6 of max|ref|.
"""
import numpy as np
import pytest
import scipy.fft as sf

import oracle
import smadft

pytestmark = pytest.mark.gpu

TOL = 3e-6


def ref_z(x, kind):
    if kind in (0, 1):
        return sf.dct(x, type=2 if kind == 0 else 3, axis=2, norm=None)
    return sf.dst(x, type=2 if kind == 2 else 3, axis=2, norm=None)


def run_pass(shape, kind, x, in_place=False):
    import torch
    p = smadft.params(smadft.NOADV, shape, precision=smadft.FP32)
    with smadft.Solver(p) as s:
        src = torch.from_numpy(x).to("cuda", torch.float32).contiguous()
        dst = src if in_place else torch.empty_like(src)
        torch.cuda.synchronize()
        l0 = s.launches
        s.r2r_pass_device(src.data_ptr(), dst.data_ptr(), 2, kind)
        s.sync()
        assert s.launches == l0 + 1
        return dst.double().cpu().numpy()


SHAPES = [(4, 16, 256), (6, 10, 256), (64, 64, 256), (8, 12, 128), (10, 18, 128), (150, 64, 128)]


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "x".join(map(str, s)))
@pytest.mark.parametrize("kind", [0, 1, 2, 3], ids=["dct2", "dct3", "dst2", "dst3"])
def test_gemm_z_pass_matches_r2r_definition(shape, kind, monkeypatch):
    """Every kind at both lengths: whole tiles, a partial last tile (rows not a multiple of
    64), fewer tiles than SMs and more (persistent CTAs taking several tiles)."""
    monkeypatch.setenv("SMADFT_GEMM_Z", "1")
    rng = np.random.default_rng(7 + kind)
    # rows of very different magnitudes: the per-row scaling must keep each one accurate
    x = rng.standard_normal(shape) * np.exp(rng.uniform(-8, 8, size=shape[:2]))[:, :, None]
    got = run_pass(shape, kind, x)
    want = ref_z(x, kind)
    err = np.abs(got - want).max(axis=2) / np.abs(want).max(axis=2)
    assert err.max() <= TOL, err.max()


@pytest.mark.parametrize("kind", [0, 1], ids=["dct2", "dct3"])
def test_gemm_z_pass_in_place_full_grid(kind, monkeypatch):
    """The benchmark's line count (256 x 256 rows of 256) in place."""
    monkeypatch.setenv("SMADFT_GEMM_Z", "1")
    shape = (256, 256, 256)
    x = np.random.default_rng(3).standard_normal(shape).astype(np.float32).astype(np.float64)
    got = run_pass(shape, kind, x, in_place=True)
    want = ref_z(x, kind)
    assert np.abs(got - want).max() <= TOL * np.abs(want).max()


@pytest.mark.parametrize("kinds", [(0, 0, 0), (1, 1, 1), (2, 3, 1), (3, 2, 0), (1, 0, 3), (0, 1, 2)],
                         ids=lambda k: "".join(map(str, k)))
@pytest.mark.parametrize("shape", [(8, 24, 256), (16, 32, 128)], ids=lambda s: "x".join(map(str, s)))
def test_gemm_z_in_3d_transform_matches_oracle(shape, kinds, monkeypatch):
    """A whole 3-D transform (y pass, GEMM-form z pass in place, x pass) against the oracle."""
    import torch
    monkeypatch.setenv("SMADFT_GEMM_Z", "1")
    x = np.random.default_rng(11).standard_normal(shape)
    p = smadft.params(smadft.NOADV, shape, precision=smadft.FP32)
    with smadft.Solver(p) as s:
        src = torch.from_numpy(x).to("cuda", torch.float32).contiguous()
        dst = torch.empty_like(src)
        s.r2r3d_device(src.data_ptr(), dst.data_ptr(), kinds)
        s.sync()
        got = dst.double().cpu().numpy()
    want = oracle.r2r_3d(x, kinds)
    assert np.abs(got - want).max() <= TOL * np.abs(want).max()


def test_gemm_z_adv_step_matches_fft_form(monkeypatch):
    """Whole adv steps with the GEMM-form z passes against the FFT-form FP32 path and the FP64
    oracle: the relative L2 error of psi stays in the FP32 class."""
    shape = (16, 64, 256)
    p = smadft.params(smadft.ADV, shape, precision=smadft.FP32, dt=0.01)
    psi0 = smadft.ic_conics(p, A=1.3, count=3, rmin=1.0, rmax=2.0, noise=1e-3, seed=5)
    out = {}
    for flag in ("0", "1"):
        monkeypatch.setenv("SMADFT_GEMM_Z", flag)
        with smadft.Solver(p) as s:
            s.set_psi(psi0)
            s.step(20)
            out[flag] = s.get("psi")
    o = oracle.Oracle(oracle.ADV, shape, nw=p.nw, dt=p.dt, eps=p.eps, nu=p.nu)
    o.set_psi(psi0)
    o.step(20)
    want = o.get(oracle.F_PSI)
    for flag, got in out.items():
        err = np.linalg.norm(got - want) / np.linalg.norm(want)
        print(f"SMADFT_GEMM_Z={flag}: FP32 psi rel L2 vs oracle after 20 adv steps {err:.3e}")
        assert err <= 2e-5
