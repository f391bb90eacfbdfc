"""The adv step's gradient fields through psi's own y and z passes.

grad psi is the transform of index-shifted, scaled copies of psihat along one axis, and
that shift-and-scale commutes with the transforms along the other axes, so the step takes
gz from psi's y-pass output and gx from psi's y + z output (SMADFT_SHARE_GRAD=1, the
default where the y length has the register-direct grouped pass) instead of transforming
three scaled copies of psihat (SMADFT_SHARE_GRAD=0, the reference's order).  The two orders
differ only in rounding: FP64 fields agree to 1e-12 of their norm, and both stay on the
oracle's trajectory.
"""
import numpy as np
import pytest

import oracle
import smadft

pytestmark = pytest.mark.gpu

FIELDS = ("psi", "gx", "gy", "gz", "vx", "vy", "vz")
OF = dict(psi=oracle.F_PSI, gx=oracle.F_GX, gy=oracle.F_GY, gz=oracle.F_GZ, vx=oracle.F_VX, vy=oracle.F_VY,
          vz=oracle.F_VZ)


def run(shape, prec, flag, steps, monkeypatch, psi0, dt):
    monkeypatch.setenv("SMADFT_SHARE_GRAD", flag)
    p = smadft.params(smadft.ADV, shape, precision=prec, dt=dt)
    with smadft.Solver(p) as s:
        s.set_psi(psi0)
        s.step(steps)
        return {f: s.get(f) for f in FIELDS}


@pytest.mark.parametrize("shape", [(16, 64, 48), (12, 128, 40), (8, 256, 64)],
                         ids=lambda v: "x".join(map(str, v)))
@pytest.mark.parametrize("prec", [smadft.FP64, smadft.FP32], ids=["fp64", "fp32"])
def test_shared_gradients_match_reference_order_and_oracle(shape, prec, monkeypatch):
    steps, dt = 6, 0.01
    p = smadft.params(smadft.ADV, shape, dt=dt)
    psi0 = smadft.ic_conics(p, A=1.3, count=3, rmin=1.0, rmax=2.0, noise=1e-3, seed=17)
    shared = run(shape, prec, "1", steps, monkeypatch, psi0, dt)
    plain = run(shape, prec, "0", steps, monkeypatch, psi0, dt)
    o = oracle.Oracle(oracle.ADV, shape, nw=p.nw, dt=p.dt, eps=p.eps, nu=p.nu)
    o.set_psi(psi0)
    o.step(steps)
    tol_pair = 1e-12 if prec == smadft.FP64 else 2e-5
    tol_oracle = 1e-11 if prec == smadft.FP64 else 2e-5
    for f in FIELDS:
        a, b, want = shared[f], plain[f], o.get(OF[f])
        nrm = np.linalg.norm(want)
        d_pair = np.linalg.norm(a - b) / nrm
        d_oracle = np.linalg.norm(a - want) / nrm
        print(f"{f}: shared vs reference order {d_pair:.2e}, shared vs oracle {d_oracle:.2e}")
        assert d_pair <= tol_pair, f
        assert d_oracle <= tol_oracle, f
