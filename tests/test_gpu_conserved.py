"""Conserved dynamics (smadft_params.conserved = 1) on the GPU against the oracle.

The reference's conserved variants are no-adv/cosNoAdvConserv.cpp (operator and N weighted
by q^2: C1,2 = 1 +- dt/2 q^2 L, N = q^2 REDFT10^3(beta psi^3 - gamma psi^5), the pre-loop N
weighted too) and adv/cosAdvConSingle.cpp (C1,2 = 1 +- dt/2 q^2 L, Sp2 still from L,
N = q^2 REDFT10^3(beta psi^3 - gamma psi^5) - REDFT10^3(v . grad psi), the pre-loop N
unweighted).  The oracle is pinned bit-exact to both (tests/test_oracle_pin.py).

The q^2-weighted explicit term is stiffer than the non-conserved one: at nw = 8 these runs
use dt = 0.005 (the reference runs dt = 0.0005 at nw = 16).
"""
import numpy as np
import pytest

import oracle
import smadft

pytestmark = pytest.mark.gpu

OMODEL = {smadft.NOADV: oracle.NOADV, smadft.ADV: oracle.ADV}
KW = {smadft.NOADV: dict(dt=0.005, eps=-0.7), smadft.ADV: dict(dt=0.005, eps=-0.7, nu=1.0)}


def rel_max(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def make(model, shape, precision=smadft.FP64, **over):
    kw = dict(KW[model])
    kw.update(over)
    return smadft.params(model, shape, precision=precision, conserved=1, **kw)


def ic(p, seed=7):
    return smadft.ic_interface(p, A=1.328, bump=0.5, noise=1e-3, seed=seed)


@pytest.mark.parametrize("model", [smadft.NOADV, smadft.ADV])
@pytest.mark.parametrize("shape,steps", [
    ((16, 12, 20), 40),      # generic Stockham passes
    ((24, 64, 64), 20),      # register-direct y/z passes, grouped y transforms (adv)
    ((64, 32, 128), 15),     # register-direct x pass with the conserved update storer
])
def test_fp64_matches_oracle(model, shape, steps):
    p = make(model, shape)
    psi0 = ic(p)
    with smadft.Solver(p) as s:
        s.set_psi(psi0)
        s.step(steps - 1)
        d = s.step_diag()
        got = {"psi": s.get("psi"), "nhat": s.get("nhat")}
        if model == smadft.ADV:
            got["vx"] = s.get("vx")
            got["gz"] = s.get("gz")
    o = oracle.Oracle(OMODEL[model], shape, conserved=1, **KW[model])
    o.set_psi(psi0)
    o.step(steps)
    assert rel_max(got["psi"], o.get(oracle.F_PSI)) <= 1e-10
    assert rel_max(got["nhat"], o.get(oracle.F_NHAT)) <= 1e-10
    if model == smadft.ADV:
        assert rel_max(got["vx"], o.get(oracle.F_VX)) <= 1e-10
        assert rel_max(got["gz"], o.get(oracle.F_GZ)) <= 1e-10
    assert abs(d["l1"] - o.diag()["l1"]) <= 1e-10 * abs(o.diag()["l1"])


@pytest.mark.parametrize("model", [smadft.NOADV, smadft.ADV])
def test_fp32_tracks_fp64(model):
    shape = (64, 64, 64)
    out = {}
    for prec in (smadft.FP64, smadft.FP32):
        p = make(model, shape, precision=prec)
        with smadft.Solver(p) as s:
            s.set_psi(ic(p, seed=3))
            s.step(200)
            out[prec] = s.get("psi")
    assert rel_l2(out[smadft.FP32], out[smadft.FP64]) <= 1e-5


@pytest.mark.parametrize("precision,tol", [(smadft.FP64, 1e-13), (smadft.FP32, 1e-6)])
def test_noadv_conserved_keeps_the_mean(precision, tol):
    # the q = 0 mode has C1 = C2 = 1 and a zero-weighted N: psihat(0) never changes, so the
    # mean of psi is conserved to the rounding of the inverse transform (the oracle is not
    # needed at this size)
    p = make(smadft.NOADV, (128, 128, 128), precision=precision)
    psi0 = ic(p, seed=5)
    m0 = psi0.mean()
    with smadft.Solver(p) as s:
        s.set_psi(psi0)
        means = []
        for _ in range(3):
            s.step(99)
            means.append(s.step_diag()["mean"])
        psi = s.get("psi")
    rms = np.sqrt(np.mean(psi ** 2))
    assert np.max(np.abs(np.array(means) - m0)) <= tol * rms
    assert abs(psi.mean() - m0) <= tol * rms
    assert rel_l2(psi, psi0) > 1e-3          # the field itself did evolve


def test_conserved_runs_have_no_surface_output_or_adjoint():
    for model in (smadft.NOADV, smadft.ADV):
        p = make(model, (16, 16, 16))
        with smadft.Solver(p) as s:
            s.set_psi(ic(p))
            with pytest.raises(smadft.SmadftError) as e:
                s.step_surface()
            assert e.value.code == -6
            if model == smadft.NOADV:
                with pytest.raises(smadft.SmadftError) as e:
                    s.adjoint(4, checkpoint_every=2, axis=0, mode=smadft.TRACK_BUMP, hi=0.6, lo=0.1)
                assert e.value.code == -6


def test_checkpoint_keeps_the_conserved_flag(tmp_path):
    path = str(tmp_path / "c.ck")
    pc = make(smadft.NOADV, (16, 12, 20))
    with smadft.Solver(pc) as s:
        s.set_psi(ic(pc))
        s.step(5)
        s.save(path)
        s.step(5)
        want = s.get("psi")
    with smadft.Solver(pc) as s:
        s.load(path)
        s.step(5)
        assert np.array_equal(s.get("psi"), want)
    pn = smadft.params(smadft.NOADV, (16, 12, 20), **KW[smadft.NOADV])
    with smadft.Solver(pn) as s:
        with pytest.raises(smadft.SmadftError) as e:
            s.load(path)
        assert e.value.code == -1


def test_batch_with_conserved_members_matches_solo_runs():
    cases = [make(smadft.NOADV, (32, 24, 40)), make(smadft.ADV, (16, 64, 64), precision=smadft.FP32),
             smadft.params(smadft.NOADV, (32, 24, 40), dt=0.005, eps=-0.7)]
    solo = []
    for i, p in enumerate(cases):
        with smadft.Solver(p) as s:
            s.set_psi(ic(p, seed=20 + i))
            s.step(6)
            solo.append(s.get("psi"))
    with smadft.Batch(cases) as b:
        for i, p in enumerate(cases):
            b.members[i].set_psi(ic(p, seed=20 + i))
        b.step(6)
        b.sync()
        for i in range(len(cases)):
            assert np.array_equal(b.members[i].get("psi"), solo[i]), i
    assert not np.array_equal(solo[0], solo[2])   # conserved and non-conserved runs differ
