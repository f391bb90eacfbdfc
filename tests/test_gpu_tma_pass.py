"""TMA-fed persistent strided passes (r2r_rdt.cuh) against FFTW's r2r definitions.

With SMADFT_TMA_PASS=1 an FP32 context runs its plain x and y passes of length 64, 128 and
256 (and the CN/AB2 update pass, whose input is a plain field) with the tile inputs brought
into shared memory by cp.async.bulk.tensor two tiles ahead.  The reference is scipy.fft's
DCT/DST of types 2 and 3 with norm=None along the axis (FFTW's REDFT10/01, RODFT10/01; the
oracle's r2r is pinned to them).  Tolerance: the FP32 pass bar of the transform tests, 3e-6
of max|ref|.
"""
import numpy as np
import pytest
import scipy.fft as sf

import oracle
import smadft

pytestmark = pytest.mark.gpu

TOL = 3e-6


def ref_axis(x, axis, kind):
    if kind in (0, 1):
        return sf.dct(x, type=2 if kind == 0 else 3, axis=axis, norm=None)
    return sf.dst(x, type=2 if kind == 2 else 3, axis=axis, norm=None)


def run_pass(shape, axis, kind, x, in_place=False):
    import torch
    p = smadft.params(smadft.NOADV, shape, precision=smadft.FP32)
    with smadft.Solver(p) as s:
        src = torch.from_numpy(x).to("cuda", torch.float32).contiguous()
        dst = src if in_place else torch.empty_like(src)
        torch.cuda.synchronize()
        s.r2r_pass_device(src.data_ptr(), dst.data_ptr(), axis, kind)
        s.sync()
        return dst.double().cpu().numpy()


CASES = [((256, 8, 64), 0), ((64, 10, 40), 0), ((128, 6, 96), 0), ((12, 256, 64), 1), ((8, 64, 20), 1),
         ((5 * 2, 128, 48), 1), ((256, 256, 32), 0)]


@pytest.mark.parametrize("shape,axis", CASES, ids=lambda v: "x".join(map(str, v)) if isinstance(v, tuple) else str(v))
@pytest.mark.parametrize("kind", [0, 1, 2, 3], ids=["dct2", "dct3", "dst2", "dst3"])
def test_tma_pass_matches_r2r_definition(shape, axis, kind, monkeypatch):
    """Every kind, x and y, full and partial 32-column tiles (nz = 20, 40, 48), fewer tiles
    than CTAs and more (persistent CTAs taking several tiles)."""
    monkeypatch.setenv("SMADFT_TMA_PASS", "1")
    x = np.random.default_rng(3 + kind).standard_normal(shape)
    got = run_pass(shape, axis, kind, x)
    want = ref_axis(x, axis, kind)
    assert np.abs(got - want).max() <= TOL * np.abs(want).max()


@pytest.mark.parametrize("axis", [0, 1])
def test_tma_pass_in_place_full_grid(axis, monkeypatch):
    monkeypatch.setenv("SMADFT_TMA_PASS", "1")
    shape = (256, 256, 256)
    x = np.random.default_rng(5).standard_normal(shape).astype(np.float32).astype(np.float64)
    got = run_pass(shape, axis, 1, x, in_place=True)
    want = ref_axis(x, axis, 1)
    assert np.abs(got - want).max() <= TOL * np.abs(want).max()


@pytest.mark.parametrize("model", [smadft.NOADV, smadft.ADV], ids=["noadv", "adv"])
def test_tma_pass_steps_match_oracle(model, monkeypatch):
    """Whole FP32 steps with the TMA-fed passes (plain x passes and the update storer) against
    the FP64 oracle, in the FP32 error class of the default path."""
    shape = (128, 64, 64)
    p = smadft.params(model, shape, precision=smadft.FP32, dt=0.01)
    psi0 = smadft.ic_conics(p, A=1.3, count=3, rmin=1.0, rmax=2.0, noise=1e-3, seed=9)
    o = oracle.Oracle(oracle.ADV if model == smadft.ADV else oracle.NOADV, shape, nw=p.nw, dt=p.dt, eps=p.eps,
                      nu=p.nu)
    o.set_psi(psi0)
    o.step(10)
    want = o.get(oracle.F_PSI)
    for flag in ("0", "1"):
        monkeypatch.setenv("SMADFT_TMA_PASS", flag)
        with smadft.Solver(p) as s:
            s.set_psi(psi0)
            s.step(10)
            err = np.linalg.norm(s.get("psi") - want) / np.linalg.norm(want)
        print(f"SMADFT_TMA_PASS={flag}: FP32 psi rel L2 vs oracle after 10 steps {err:.3e}")
        assert err <= 1e-5
