"""Batched runs (smadft_batch_*) and the kernel-path autotuner (smadft_autotune).

A batch member runs the same kernels as a context of its own, so after the same number of
steps its fields are bit-identical to a solo run; the autotuner restores the state after its
trials, so a run continues as without the call (up to the rounding of a different kernel
path, if it picks one).
"""
import numpy as np
import pytest

import smadft

pytestmark = pytest.mark.gpu


def member_cases():
    return [
        (smadft.params(smadft.NOADV, (32, 24, 40)), 1.3),
        (smadft.params(smadft.ADV, (16, 64, 64), dt=0.01), 1.3),
        (smadft.params(smadft.QUASI, (24, 20, 32), dt=0.002, kp=0.3, divv_switch=3), 1.3),
        (smadft.params(smadft.ADV, (24, 32, 40), precision=smadft.FP32, dt=0.01), 1.3),
        (smadft.params(smadft.NOADV, (96, 96, 96), precision=smadft.FP32, eps=-0.7), 1.3),
    ]


def ic(p, seed):
    return smadft.ic_conics(p, A=1.3, count=2, rmin=1.0, rmax=2.0, noise=1e-3, seed=seed)


def test_batch_members_match_solo_runs():
    cases = member_cases()
    steps = 7
    solo = []
    for i, (p, _) in enumerate(cases):
        with smadft.Solver(p) as s:
            s.set_psi(ic(p, i))
            s.step(steps)
            solo.append((s.get("psi"), s.get("vx") if p.model != smadft.NOADV else None))
    with smadft.Batch([p for p, _ in cases]) as b:
        for i, (p, _) in enumerate(cases):
            b.members[i].set_psi(ic(p, i))
        b.step(3)
        b.step(steps - 3)
        b.sync()
        for i, (p, _) in enumerate(cases):
            assert np.array_equal(b.members[i].get("psi"), solo[i][0]), i
            if solo[i][1] is not None:
                assert np.array_equal(b.members[i].get("vx"), solo[i][1]), i


def test_batch_interleaves_with_member_calls():
    cases = member_cases()[:3]
    with smadft.Batch([p for p, _ in cases]) as b:
        for i, (p, _) in enumerate(cases):
            b.members[i].set_psi(ic(p, 10 + i))
        b.step(2)
        b.members[1].step(3)                 # one member alone
        d = b.members[0].step_diag()         # diagnostics step of another
        b.step(2)
        got = [m.get("psi") for m in b.members]
    ref = []
    for i, (p, _) in enumerate(cases):
        with smadft.Solver(p) as s:
            s.set_psi(ic(p, 10 + i))
            s.step(2)
            if i == 1:
                s.step(3)
            if i == 0:
                s.step_diag()
            s.step(2)
            ref.append(s.get("psi"))
    assert d["rc"] == 0
    for i in range(3):
        assert np.array_equal(got[i], ref[i]), i


def test_batch_needs_initial_conditions():
    p = smadft.params(smadft.NOADV, (16, 16, 16))
    with smadft.Batch([p, p]) as b:
        b.members[0].set_psi(ic(p, 0))
        with pytest.raises(smadft.SmadftError) as e:
            b.step(1)
        assert e.value.code == -8


@pytest.mark.parametrize("model,shape,kw", [
    (smadft.ADV, (16, 64, 64), dict(dt=0.01)),
    (smadft.QUASI, (8, 64, 64), dict(dt=0.002, kp=0.3, divv_switch=4)),
])
def test_autotune_keeps_the_run(model, shape, kw):
    p = smadft.params(model, shape, **kw)
    psi0 = ic(p, 3)
    with smadft.Solver(p) as a:
        a.set_psi(psi0)
        a.step(3)
        rep = a.autotune(2)
        a.step(5)
        got = a.get("psi")
    with smadft.Solver(p) as b:
        b.set_psi(psi0)
        b.step(8)
        want = b.get("psi")
    assert len(rep["ms_per_step"]) >= 4          # plane, staged, ungrouped, ... on ny = nz = 64
    assert rep["chosen"] in rep["ms_per_step"]
    assert np.max(np.abs(got - want)) <= 1e-11 * np.max(np.abs(want))


def test_autotune_times_the_gemm_form_z_pass_for_fp32():
    """The tensor-core GEMM-form z pass is an autotuner candidate for FP32 contexts whose z
    length is 128 or 256 (and only there): it is timed beside the FFT-form paths and kept only
    when it measures faster."""
    gemm = "GEMM-form z passes on the tensor cores"
    for prec, shape, timed in ((smadft.FP32, (8, 32, 256), True), (smadft.FP64, (8, 32, 256), False),
                               (smadft.FP32, (8, 32, 64), False)):
        p = smadft.params(smadft.ADV, shape, precision=prec, dt=0.01)
        with smadft.Solver(p) as s:
            s.set_psi(ic(p, 5))
            rep = s.autotune(2)
            s.step(2)
            assert np.all(np.isfinite(s.get("psi")))
        assert (gemm in rep["ms_per_step"]) == timed, (prec, shape, rep)


def test_batch_groups_match_solo_runs():
    """Members with the same model (noadv / adv), grid and precision form groups whose plain
    axis passes run as one launch over pooled fields; with different parameters per member
    (eps, gamma) each still follows its solo run (FP64 to 1e-12, FP32 to 1e-5 relative: the
    grouped x passes are other instantiations of the same kernels), also interleaved with a
    member stepped alone, and with grouping off the batch reproduces the solo runs exactly."""
    cases = [smadft.params(smadft.ADV, (16, 64, 64), precision=smadft.FP32, dt=0.01, eps=-0.7 - 0.05 * i,
                           gamma=1.0 + 0.1 * i) for i in range(3)]
    cases += [smadft.params(smadft.NOADV, (32, 24, 40), eps=-0.75 + 0.03 * i) for i in range(3)]
    cases += [smadft.params(smadft.ADV, (8, 96, 96), precision=smadft.FP32, dt=0.01, eps=-0.7 - 0.1 * i)
              for i in range(2)]
    cases += [smadft.params(smadft.QUASI, (24, 20, 32), dt=0.002, kp=0.3, divv_switch=3)]
    steps = 6
    solo = []
    for i, p in enumerate(cases):
        with smadft.Solver(p) as s:
            s.set_psi(ic(p, 20 + i))
            s.step(2)
            if i == 1:
                s.step(1)
            s.step(steps - 2)
            solo.append((s.get("psi"), s.get("vx") if p.model != smadft.NOADV else None))
    with smadft.Batch(cases) as b:
        assert b.groups == 3
        for i, p in enumerate(cases):
            b.members[i].set_psi(ic(p, 20 + i))
        b.step(2)
        b.members[1].step(1)                 # a grouped member alone, on its pooled fields
        b.step(steps - 2)
        b.sync()
        for i, p in enumerate(cases):
            tol = 1e-12 if p.precision == smadft.FP64 else 1e-5
            got, want = b.members[i].get("psi"), solo[i][0]
            assert np.max(np.abs(got - want)) <= tol * np.max(np.abs(want)), i
            if solo[i][1] is not None:
                gv, wv = b.members[i].get("vx"), solo[i][1]
                assert np.max(np.abs(gv - wv)) <= 10 * tol * np.max(np.abs(wv)), i


def test_batch_without_groups_is_exact(monkeypatch):
    monkeypatch.setenv("SMADFT_BATCH_GROUP", "0")
    cases = [smadft.params(smadft.ADV, (16, 64, 64), precision=smadft.FP32, dt=0.01, eps=-0.7 - 0.05 * i)
             for i in range(2)]
    solo = []
    for i, p in enumerate(cases):
        with smadft.Solver(p) as s:
            s.set_psi(ic(p, 30 + i))
            s.step(4)
            solo.append(s.get("psi"))
    with smadft.Batch(cases) as b:
        assert b.groups == 0
        for i, p in enumerate(cases):
            b.members[i].set_psi(ic(p, 30 + i))
        b.step(4)
        b.sync()
        for i in range(2):
            assert np.array_equal(b.members[i].get("psi"), solo[i]), i
