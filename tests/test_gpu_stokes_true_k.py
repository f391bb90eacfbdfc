"""Force spectra stored by true wavenumber and the aligned Stokes projection (LdStokesK).

With SMADFT_STOKES_K=1 (the default where all three lengths have the register-direct
kernels) the sine-axis pass of each force component stores its output one index up along
its axis, the projection reads the three spectra of one wavenumber at one index, and v_z's
sine z pass reads its spectrum one index up.  The operands and operations are the
reference-indexed ones (SMADFT_STOKES_K=0), so velocities and whole steps agree to rounding
(the passes that store or read one index up are separate instantiations of the same
transforms); both stay on the oracle's trajectory.
"""
import numpy as np
import pytest

import oracle
import smadft

pytestmark = pytest.mark.gpu

FIELDS = ("psi", "vx", "vy", "vz", "gx", "gy", "gz")
OF = dict(psi=oracle.F_PSI, gx=oracle.F_GX, gy=oracle.F_GY, gz=oracle.F_GZ, vx=oracle.F_VX, vy=oracle.F_VY,
          vz=oracle.F_VZ)


def run(p, psi0, steps, flag, monkeypatch):
    monkeypatch.setenv("SMADFT_STOKES_K", flag)
    with smadft.Solver(p) as s:
        s.set_psi(psi0)
        s.step(steps)
        return {f: s.get(f) for f in FIELDS}


@pytest.mark.parametrize("shape", [(64, 64, 64), (128, 64, 256), (64, 256, 128)],
                         ids=lambda v: "x".join(map(str, v)))
@pytest.mark.parametrize("prec", [smadft.FP64, smadft.FP32], ids=["fp64", "fp32"])
def test_true_k_stokes_matches_the_reference_indexing(shape, prec, monkeypatch):
    p = smadft.params(smadft.ADV, shape, precision=prec, dt=0.01)
    psi0 = smadft.ic_conics(p, A=1.3, count=3, rmin=1.0, rmax=2.0, noise=1e-3, seed=23)
    a = run(p, psi0, 4, "1", monkeypatch)
    b = run(p, psi0, 4, "0", monkeypatch)
    if prec == smadft.FP64:
        for f in FIELDS:
            d = np.linalg.norm(a[f] - b[f]) / np.linalg.norm(b[f])
            print(f"{f}: true-k vs reference indexing {d:.2e}")
            assert d <= 1e-13, f
        return
    # FP32: the projection subtracts nearly equal terms, so rounding differences in the spectra
    # show up magnified in v (both orders sit about 5e-6 from FP64 there).  The true-k order
    # must be as close to the FP64 result as the reference order is.
    c = run(smadft.params(smadft.ADV, shape, dt=0.01), psi0, 4, "0", monkeypatch)
    for f in FIELDS:
        ea = np.linalg.norm(a[f] - c[f]) / np.linalg.norm(c[f])
        eb = np.linalg.norm(b[f] - c[f]) / np.linalg.norm(c[f])
        print(f"{f}: FP32 vs FP64, true-k {ea:.2e}, reference indexing {eb:.2e}")
        assert ea <= 2 * eb + 1e-7, f


@pytest.mark.parametrize("prec", [smadft.FP64, smadft.FP32], ids=["fp64", "fp32"])
def test_true_k_stokes_matches_oracle(prec, monkeypatch):
    shape, steps = (64, 64, 128), 6
    p = smadft.params(smadft.ADV, shape, precision=prec, dt=0.01)
    psi0 = smadft.ic_conics(p, A=1.3, count=3, rmin=1.0, rmax=2.0, noise=1e-3, seed=29)
    got = run(p, psi0, steps, "1", monkeypatch)
    o = oracle.Oracle(oracle.ADV, shape, nw=p.nw, dt=p.dt, eps=p.eps, nu=p.nu)
    o.set_psi(psi0)
    o.step(steps)
    tol = 1e-11 if prec == smadft.FP64 else 2e-5
    for f in FIELDS:
        want = o.get(OF[f])
        err = np.linalg.norm(got[f] - want) / np.linalg.norm(want)
        print(f"{f}: rel L2 vs oracle {err:.2e}")
        assert err <= tol, f


@pytest.mark.parametrize("prec", [smadft.FP64, smadft.FP32], ids=["fp64", "fp32"])
def test_true_k_stokes_in_batch_groups_matches_solo_runs(prec):
    """A batch group of adv members runs the same order with its z passes over the pool."""
    cases = [smadft.params(smadft.ADV, (64, 64, 64), precision=prec, dt=0.01, eps=-0.7 - 0.05 * i) for i in range(2)]
    ics = [smadft.ic_conics(p, A=1.3, count=2, rmin=1.0, rmax=2.0, noise=1e-3, seed=40 + i)
           for i, p in enumerate(cases)]
    solo = []
    for p, ic in zip(cases, ics):
        with smadft.Solver(p) as s:
            s.set_psi(ic)
            s.step(5)
            solo.append({f: s.get(f) for f in ("psi", "vx", "vy", "vz")})
    with smadft.Batch(cases) as b:
        assert b.groups == 1
        for i, ic in enumerate(ics):
            b.members[i].set_psi(ic)
        b.step(5)
        b.sync()
        for i in range(len(cases)):
            for f in ("psi", "vx", "vy", "vz"):
                got, want = b.members[i].get(f), solo[i][f]
                d = np.linalg.norm(got - want) / np.linalg.norm(want)
                print(f"member {i} {f}: group vs solo {d:.2e}")
                assert d <= (1e-12 if prec == smadft.FP64 else 1e-5), (i, f)
