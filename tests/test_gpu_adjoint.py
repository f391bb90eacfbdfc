"""Adjoint of the diffusive step (smadft_adjoint): gradients of the mean interface position
against central differences of the FP64 forward, and the FP32 adjoint against the FP64
adjoint.

The loss is piecewise smooth: each column's position is a linear interpolation inside one
grid cell, and its derivative jumps where a crossing moves to the next cell.  A difference
step must therefore be small enough that no crossing changes cell between +h and -h: with
h = 1e-4 about one of the 384 columns does (the difference then misses the gradient by
~1e-3 in eps and by a factor ~3 in the initial-psi direction), with h = 1e-6 none does."""
import numpy as np
import pytest

import smadft

pytestmark = pytest.mark.gpu

SHAPE = (32, 16, 24)
STEPS, K = 30, 10
TRACK = dict(axis=0, mode=smadft.TRACK_BUMP, hi=0.6, lo=0.1)
BASE = dict(eps=-0.7, alpha=1.0, beta=2.0, gamma=1.0, dt=0.05)


def make(precision=smadft.FP64, **over):
    kw = dict(BASE)
    kw.update(over)
    return smadft.params(smadft.NOADV, SHAPE, precision=precision, **kw)


def psi_init():
    p = make()
    return smadft.ic_interface(p, A=1.328, bump=0.5 * 2 * np.pi, noise=1e-3, seed=31)


def forward_loss(psi0, **over):
    p = make(**over)
    with smadft.Solver(p) as s:
        s.set_psi(psi0)
        s.step(STEPS)
        idx, pos = s.track(**TRACK)
    m = (idx >= 0) & np.isfinite(pos)
    return pos[m].mean() / p.nw, int(m.sum())


@pytest.fixture(scope="module")
def adj64():
    psi0 = psi_init()
    with smadft.Solver(make()) as s:
        s.set_psi(psi0)
        g = s.adjoint(STEPS, checkpoint_every=K, **TRACK)
        after = s.get("psi")
    return psi0, g, after


def test_adjoint_loss_and_state(adj64):
    psi0, g, after = adj64
    loss, found = forward_loss(psi0)
    assert g["found"] == found and found > SHAPE[1] * SHAPE[2] // 2
    assert abs(g["loss"] - loss) <= 1e-12 * abs(loss)
    with smadft.Solver(make()) as s:          # the run continues from the final state
        s.set_psi(psi0)
        s.step(STEPS)
        assert np.array_equal(s.get("psi"), after)


@pytest.mark.parametrize("name", ["eps", "alpha", "beta", "gamma"])
def test_adjoint_parameter_gradient_matches_central_difference(adj64, name):
    psi0, g, _ = adj64
    h = 1e-6
    jp, fp = forward_loss(psi0, **{name: BASE[name] + h})
    jm, fm = forward_loss(psi0, **{name: BASE[name] - h})
    assert fp == fm == g["found"]
    fd = (jp - jm) / (2 * h)
    assert abs(g[name] - fd) <= 1e-4 * abs(fd) + 1e-8, (name, g[name], fd)


def test_adjoint_initial_condition_gradient_matches_central_difference(adj64):
    psi0, g, _ = adj64
    x = np.arange(SHAPE[0])[:, None, None]
    y = np.arange(SHAPE[1])[None, :, None]
    z = np.arange(SHAPE[2])[None, None, :]
    d = np.cos(0.3 * x) * np.sin(0.4 * y + 0.2) * np.cos(0.5 * z) + 0.3 * np.cos(0.2 * x + 0.1 * z)
    h = 1e-6
    jp, fp = forward_loss(psi0 + h * d)
    jm, fm = forward_loss(psi0 - h * d)
    assert fp == fm == g["found"]
    fd = (jp - jm) / (2 * h)
    ad = float(np.sum(g["psi0"] * d))
    assert abs(ad - fd) <= 1e-4 * abs(fd) + 1e-8, (ad, fd)


def test_fp32_adjoint_matches_fp64_adjoint(adj64):
    psi0, g64, _ = adj64
    with smadft.Solver(make(precision=smadft.FP32)) as s:
        s.set_psi(psi0)
        g32 = s.adjoint(STEPS, checkpoint_every=K, **TRACK)
    assert g32["found"] == g64["found"]
    for name in ("eps", "alpha", "beta", "gamma"):
        assert abs(g32[name] - g64[name]) <= 1e-3 * abs(g64[name]) + 1e-7, name
    rel = np.linalg.norm(g32["psi0"] - g64["psi0"]) / np.linalg.norm(g64["psi0"])
    assert rel <= 1e-3


def test_adjoint_needs_initial_state_and_a_supported_model():
    psi0 = psi_init()
    with smadft.Solver(make()) as s:
        s.set_psi(psi0)
        s.step(1)
        with pytest.raises(smadft.SmadftError) as e:
            s.adjoint(5, checkpoint_every=5, **TRACK)
        assert e.value.code == -8
    p = smadft.params(smadft.QUASI, (16, 16, 16))
    with smadft.Solver(p) as s:
        s.set_psi(np.zeros((16, 16, 16)))
        with pytest.raises(smadft.SmadftError) as e:
            s.adjoint(5, checkpoint_every=5, **TRACK)
        assert e.value.code == -6
