"""Adjoint of the advected step (smadft_adjoint on an adv run): gradients of the mean
interface position with respect to eps, alpha, beta, gamma, nu and the initial psi against
central differences of the FP64 forward, and the FP32 adjoint against the FP64 adjoint.

The reverse sweep runs through the transposed Stokes projection (with its truncated modes),
the index-shifted gradient spectra and the mixed DCT/DST transforms; 20 steps with
checkpoints every 6 leave a shorter last segment.  As for the diffusive adjoint, the
difference step is 1e-6, small enough that no tracked crossing changes cell between +h and
-h (the loss is piecewise smooth)."""
import numpy as np
import pytest

import smadft

pytestmark = pytest.mark.gpu

STEPS, K = 20, 6
TRACK = dict(axis=0, mode=smadft.TRACK_BUMP, hi=0.6, lo=0.1)
BASE = dict(eps=-0.7, alpha=1.0, beta=2.0, gamma=1.0, nu=1.3, dt=0.02)
H = 1e-6


def make(shape, precision=smadft.FP64, **over):
    kw = dict(BASE)
    kw.update(over)
    return smadft.params(smadft.ADV, shape, precision=precision, **kw)


def psi_init(shape):
    return smadft.ic_interface(make(shape), A=1.328, bump=0.5 * 2 * np.pi, noise=1e-3, seed=31)


def forward_loss(shape, psi0, **over):
    p = make(shape, **over)
    with smadft.Solver(p) as s:
        s.set_psi(psi0)
        s.step(STEPS)
        idx, pos = s.track(**TRACK)
    m = (idx >= 0) & np.isfinite(pos)
    return pos[m].mean() / p.nw, int(m.sum())


def direction(shape):
    x = np.arange(shape[0])[:, None, None]
    y = np.arange(shape[1])[None, :, None]
    z = np.arange(shape[2])[None, None, :]
    return np.cos(0.3 * x) * np.sin(0.4 * y + 0.2) * np.cos(0.5 * z) + 0.3 * np.cos(0.2 * x + 0.1 * z)


def adjoint_of(shape, precision=smadft.FP64):
    psi0 = psi_init(shape)
    with smadft.Solver(make(shape, precision=precision)) as s:
        s.set_psi(psi0)
        g = s.adjoint(STEPS, checkpoint_every=K, **TRACK)
        after = {f: s.get(f) for f in ("psi", "vx", "gz")}
    return psi0, g, after


SMALL = (32, 16, 24)      # generic passes
GROUPED = (48, 64, 64)    # register-direct y/z passes, grouped multi-component transforms


@pytest.fixture(scope="module")
def adj64():
    return adjoint_of(SMALL)


def test_adv_adjoint_loss_and_state(adj64):
    psi0, g, after = adj64
    loss, found = forward_loss(SMALL, psi0)
    assert g["found"] == found and found > SMALL[1] * SMALL[2] // 2
    assert abs(g["loss"] - loss) <= 1e-12 * abs(loss)
    with smadft.Solver(make(SMALL)) as s:          # the run continues as a plain run would
        s.set_psi(psi0)
        s.step(STEPS)
        for f, v in after.items():
            assert np.array_equal(s.get(f), v), f


@pytest.mark.parametrize("name", ["eps", "alpha", "beta", "gamma", "nu"])
def test_adv_adjoint_parameter_gradient_matches_central_difference(adj64, name):
    psi0, g, _ = adj64
    jp, fp = forward_loss(SMALL, psi0, **{name: BASE[name] + H})
    jm, fm = forward_loss(SMALL, psi0, **{name: BASE[name] - H})
    assert fp == fm == g["found"]
    fd = (jp - jm) / (2 * H)
    assert abs(g[name] - fd) <= 1e-4 * abs(fd) + 1e-8, (name, g[name], fd)


def test_adv_adjoint_initial_condition_gradient_matches_central_difference(adj64):
    psi0, g, _ = adj64
    d = direction(SMALL)
    jp, fp = forward_loss(SMALL, psi0 + H * d)
    jm, fm = forward_loss(SMALL, psi0 - H * d)
    assert fp == fm == g["found"]
    fd = (jp - jm) / (2 * H)
    ad = float(np.sum(g["psi0"] * d))
    assert abs(ad - fd) <= 1e-4 * abs(fd) + 1e-8, (ad, fd)


def test_adv_fp32_adjoint_matches_fp64_adjoint(adj64):
    _, g64, _ = adj64
    _, g32, _ = adjoint_of(SMALL, smadft.FP32)
    assert g32["found"] == g64["found"]
    for name in ("eps", "alpha", "beta", "gamma", "nu"):
        assert abs(g32[name] - g64[name]) <= 1e-3 * abs(g64[name]) + 1e-7, name
    rel = np.linalg.norm(g32["psi0"] - g64["psi0"]) / np.linalg.norm(g64["psi0"])
    assert rel <= 1e-3


def test_adv_adjoint_on_the_grouped_passes():
    psi0, g, _ = adjoint_of(GROUPED)
    for name in ("eps", "nu"):
        jp, fp = forward_loss(GROUPED, psi0, **{name: BASE[name] + H})
        jm, fm = forward_loss(GROUPED, psi0, **{name: BASE[name] - H})
        assert fp == fm == g["found"]
        fd = (jp - jm) / (2 * H)
        assert abs(g[name] - fd) <= 1e-4 * abs(fd) + 1e-8, (name, g[name], fd)
    d = direction(GROUPED)
    jp, _ = forward_loss(GROUPED, psi0 + H * d)
    jm, _ = forward_loss(GROUPED, psi0 - H * d)
    fd = (jp - jm) / (2 * H)
    ad = float(np.sum(g["psi0"] * d))
    assert abs(ad - fd) <= 1e-4 * abs(fd) + 1e-8, (ad, fd)
    _, g32, _ = adjoint_of(GROUPED, smadft.FP32)
    for name in ("eps", "alpha", "beta", "gamma", "nu"):
        assert abs(g32[name] - g[name]) <= 1e-3 * abs(g[name]) + 1e-7, name
