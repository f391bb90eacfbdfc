"""The compressible model (SMADFT_MODEL_COMP) on the GPU against the oracle.

The oracle restates compressible/compressible.cpp and is pinned bit-exact to it
(tests/test_oracle_pin.py).  The runs cross the relaxation switch (divv_switch): before it
rho follows the filtered amplitude, shifted up by rho_up planes; after it rho has its own
mass balance.  FP64 matches the oracle to 1e-10 relative on every field; FP32 states its
relative error against FP64.
"""
import numpy as np
import pytest

import oracle
import smadft

pytestmark = pytest.mark.gpu

BASE = dict(nw=8.0, dt=0.001, eps=-0.75, nu=1.0, rho0=0.01, zeta=0.001)
FIELDS = {"psi": oracle.F_PSI, "psihat": oracle.F_PSIHAT, "rho": oracle.F_RHO, "amp": oracle.F_AMP,
          "divv": oracle.F_DIVV, "mu": oracle.F_MU, "vx": oracle.F_VSOLX, "vy": oracle.F_VSOLY,
          "vz": oracle.F_VSOLZ, "virrx": oracle.F_VIRRX, "virry": oracle.F_VIRRY, "virrz": oracle.F_VIRRZ,
          "frho": oracle.F_FRHO, "nhat": oracle.F_NHAT, "gx": oracle.F_GX}


def rel_max(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def ic(shape, seed=3):
    """Smectic layers behind an x-normal interface, with a small seeded perturbation."""
    nx, ny, nz = shape
    x = np.arange(nx)[:, None, None]
    z = np.arange(nz)[None, None, :] * 2 * np.pi / 8
    rng = np.random.default_rng(seed)
    return 1.3 * np.cos(z) * 0.5 * (1 - np.tanh((x - nx / 2) / 4.0)) * np.ones((1, ny, 1)) + \
        0.01 * rng.standard_normal(shape)


def make(shape, precision=smadft.FP64, **over):
    kw = dict(BASE)
    kw.update(over)
    return smadft.params(smadft.COMP, shape, precision=precision, **kw)


@pytest.mark.parametrize("shape,steps,divv,rho_up", [
    ((16, 12, 20), 30, 10, 16),      # generic passes, relaxation then independent rho
    ((24, 64, 64), 12, 5, 8),        # register-direct y/z passes, 8-component grouped transforms
    ((64, 32, 128), 8, 3, 0),        # register-direct x pass, no z shift of rho
])
def test_fp64_matches_oracle(shape, steps, divv, rho_up):
    psi0 = ic(shape)
    p = make(shape, divv_switch=divv, rho_up=rho_up)
    with smadft.Solver(p) as s:
        s.set_psi(psi0)
        s.step(steps - 1)
        d = s.step_diag()
        got = {k: s.get(k) for k in FIELDS}
    kw = dict(BASE)
    o = oracle.Oracle(oracle.COMP, shape, divv_switch=divv, rho_up=rho_up, **kw)
    o.set_psi(psi0)
    o.step(steps)
    for k, f in FIELDS.items():
        assert rel_max(got[k], o.get(f)) <= 1e-10, k
    od = o.diag()
    for k in ("l1", "mass", "energy"):
        assert abs(d[k] - od[k]) <= 1e-10 * abs(od[k]), k


def test_fp32_tracks_fp64():
    shape = (32, 64, 64)
    out = {}
    for prec in (smadft.FP64, smadft.FP32):
        with smadft.Solver(make(shape, precision=prec, divv_switch=20, rho_up=8)) as s:
            s.set_psi(ic(shape, seed=5))
            s.step(60)
            out[prec] = (s.get("psi"), s.get("rho"))
    for a, b in zip(out[smadft.FP32], out[smadft.FP64]):
        assert np.linalg.norm(a - b) / np.linalg.norm(b) <= 1e-5


def test_checkpoint_resume_is_bit_exact(tmp_path):
    shape = (16, 12, 20)
    path = str(tmp_path / "comp.ck")
    p = make(shape, divv_switch=6, rho_up=4)
    with smadft.Solver(p) as s:
        s.set_psi(ic(shape))
        s.step(4)
        s.save(path)
        s.step(6)
        want = (s.get("psi"), s.get("rho"))
    with smadft.Solver(p) as s:
        s.load(path)
        s.step(6)
        assert np.array_equal(s.get("psi"), want[0])
        assert np.array_equal(s.get("rho"), want[1])


def test_comp_has_no_surface_output_or_adjoint():
    shape = (16, 12, 20)
    with smadft.Solver(make(shape)) as s:
        s.set_psi(ic(shape))
        with pytest.raises(smadft.SmadftError) as e:
            s.step_surface()
        assert e.value.code == -6
        with pytest.raises(smadft.SmadftError) as e:
            s.adjoint(4, checkpoint_every=2)
        assert e.value.code == -6


def test_batch_with_comp_members_matches_solo_runs():
    cases = [make((16, 12, 20), divv_switch=3, rho_up=4), make((24, 64, 64), precision=smadft.FP32, divv_switch=2),
             smadft.params(smadft.ADV, (16, 64, 64), dt=0.01)]
    solo = []
    for i, p in enumerate(cases):
        with smadft.Solver(p) as s:
            s.set_psi(ic((p.nx, p.ny, p.nz), seed=30 + i))
            s.step(5)
            solo.append(s.get("psi"))
    with smadft.Batch(cases) as b:
        for i, p in enumerate(cases):
            b.members[i].set_psi(ic((p.nx, p.ny, p.nz), seed=30 + i))
        b.step(2)
        b.step(3)
        b.sync()
        for i in range(len(cases)):
            assert np.array_equal(b.members[i].get("psi"), solo[i]), i


def test_autotune_keeps_a_comp_run():
    # ny = nz = 64 offers the fused plane path too; the in-place inverse group then goes
    # through the scratch field
    shape = (16, 64, 64)
    p = make(shape, divv_switch=2, rho_up=4)
    psi0 = ic(shape, seed=9)
    with smadft.Solver(p) as a:
        a.set_psi(psi0)
        a.step(3)
        rep = a.autotune(2)
        a.step(4)
        got = a.get("psi"), a.get("rho")
    with smadft.Solver(p) as b:
        b.set_psi(psi0)
        b.step(7)
        want = b.get("psi"), b.get("rho")
    assert rep["chosen"] in rep["ms_per_step"] and len(rep["ms_per_step"]) >= 4
    for g, w in zip(got, want):
        assert np.max(np.abs(g - w)) <= 1e-11 * np.max(np.abs(w))
