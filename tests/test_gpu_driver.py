"""The reference-style driver (sma-dft_b200/smadft_run) end to end: its output files against
the oracle stepping the same initial condition.

L1.dat gets one line per `l1every` steps (no-adv/cosNoAdvTrackSing.cpp:789-795); on the save
iteration surfPsi.dat / velSurf.dat / curvH.dat / curvK.dat get one line per (i, j) column
(:1004-1021, adv/cosAdvTrackMult.cpp:1578-1585).
"""
import os
import subprocess

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

DRIVER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "sma-dft_b200", "smadft_run")


def read(path):
    with open(path) as f:
        return np.array([float(x) for x in f.read().split()])


@pytest.mark.parametrize("model,omodel,extra", [
    ("noadv", oracle.NOADV, dict(dt=0.05)),
    ("adv", oracle.ADV, dict(dt=0.02, nu=1.0)),
])
def test_driver_outputs_match_oracle(tmp_path, model, omodel, extra):
    if not os.path.exists(DRIVER):
        pytest.skip("smadft_run not built")
    shape = (16, 12, 20)
    z = np.arange(shape[2]) * 2 * np.pi / 8
    rng = np.random.default_rng(11)
    psi0 = (1.3 * np.cos(z)[None, None, :] * np.ones((shape[0], shape[1], 1))
            + 0.05 * np.sin(np.arange(shape[0]) * 0.7)[:, None, None] * np.cos(np.arange(shape[1]) * 0.5)[None, :, None]
            + 0.01 * rng.standard_normal(shape))
    ic = tmp_path / "ic.txt"
    np.savetxt(ic, psi0.reshape(-1), fmt="%.17g")
    args = [DRIVER, model, f"nx={shape[0]}", f"ny={shape[1]}", f"nz={shape[2]}", "nw=8", "eps=-0.7",
            "steps=20", "l1every=10", "saveevery=2", f"ic=file:{ic}", f"out={tmp_path}"]
    args += [f"{k}={v}" for k, v in extra.items()]
    subprocess.run(args, check=True, capture_output=True, text=True)

    o = oracle.Oracle(omodel, shape, nw=8, eps=-0.7, **extra)
    o.set_psi(psi0)
    o.step(10)
    l1_10 = o.diag()["l1"]
    o.step(9)
    idx, vel, h, k = o.step_surface()
    l1_20 = o.diag()["l1"]

    l1 = read(tmp_path / "L1.dat")
    assert l1.size == 2
    assert np.allclose(l1, [l1_10, l1_20], rtol=1e-10, atol=0)
    surf = read(tmp_path / "surfPsi.dat")
    found = idx.reshape(-1) >= 0
    assert found.sum() > found.size // 2
    assert np.array_equal(surf, idx.reshape(-1).astype(float))
    for name, want in (("velSurf.dat", vel), ("curvH.dat", h), ("curvK.dat", k)):
        got = read(tmp_path / name)
        w = want.reshape(-1)
        assert np.max(np.abs(got[found] - w[found])) <= 1e-9 * np.max(np.abs(w[found])), name
    final = read(tmp_path / "psi0.dat").reshape(shape)
    assert np.max(np.abs(final - o.get(oracle.F_PSI))) <= 1e-10 * np.max(np.abs(final))


@pytest.mark.parametrize("model,omodel,extra", [
    ("noadv", oracle.NOADV, dict(dt=0.005)),
    ("adv", oracle.ADV, dict(dt=0.005, nu=1.0)),
])
def test_driver_conserved_run_matches_oracle(tmp_path, model, omodel, extra):
    if not os.path.exists(DRIVER):
        pytest.skip("smadft_run not built")
    shape = (16, 12, 20)
    z = np.arange(shape[2]) * 2 * np.pi / 8
    rng = np.random.default_rng(12)
    psi0 = 1.3 * np.cos(z)[None, None, :] * np.ones((shape[0], shape[1], 1)) + 0.01 * rng.standard_normal(shape)
    ic = tmp_path / "ic.txt"
    np.savetxt(ic, psi0.reshape(-1), fmt="%.17g")
    args = [DRIVER, model, f"nx={shape[0]}", f"ny={shape[1]}", f"nz={shape[2]}", "nw=8", "eps=-0.7",
            "conserved=1", "steps=20", "l1every=10", "saveevery=2", f"ic=file:{ic}", f"out={tmp_path}"]
    args += [f"{k}={v}" for k, v in extra.items()]
    subprocess.run(args, check=True, capture_output=True, text=True)

    o = oracle.Oracle(omodel, shape, nw=8, eps=-0.7, conserved=1, **extra)
    o.set_psi(psi0)
    o.step(10)
    l1_10 = o.diag()["l1"]
    o.step(10)
    l1_20 = o.diag()["l1"]
    assert np.allclose(read(tmp_path / "L1.dat"), [l1_10, l1_20], rtol=1e-10, atol=0)
    idx, _ = o.track(axis=2, mode=0, hi=0.7, lo=0.0)
    assert np.array_equal(read(tmp_path / "surfPsi.dat"), idx.reshape(-1).astype(float))
    assert read(tmp_path / "velSurf.dat").size == 0      # no conserved surface diagnostics
    final = read(tmp_path / "psi0.dat").reshape(shape)
    assert np.max(np.abs(final - o.get(oracle.F_PSI))) <= 1e-10 * np.max(np.abs(final))


def test_driver_comp_run_matches_oracle(tmp_path):
    if not os.path.exists(DRIVER):
        pytest.skip("smadft_run not built")
    shape = (16, 12, 20)
    x = np.arange(shape[0])[:, None, None]
    z = np.arange(shape[2])[None, None, :] * 2 * np.pi / 8
    psi0 = 1.3 * np.cos(z) * 0.5 * (1 - np.tanh((x - 8) / 4.0)) * np.ones((1, shape[1], 1))
    ic = tmp_path / "ic.txt"
    np.savetxt(ic, psi0.reshape(-1), fmt="%.17g")
    args = [DRIVER, "comp", f"nx={shape[0]}", f"ny={shape[1]}", f"nz={shape[2]}", "nw=8", "eps=-0.75",
            "dt=0.001", "divv=30", "rhoup=4", "steps=100", "l1every=50", "saveevery=2", f"ic=file:{ic}",
            f"out={tmp_path}"]
    subprocess.run(args, check=True, capture_output=True, text=True)
    o = oracle.Oracle(oracle.COMP, shape, nw=8, eps=-0.75, dt=0.001, nu=1.0, rho0=0.01, zeta=0.001,
                      divv_switch=30, rho_up=4)
    o.set_psi(psi0)
    want = []
    for _ in range(2):
        o.step(50)
        want.append(o.diag())
    for name, key in (("L1.dat", "l1"), ("mass.dat", "mass"), ("energy.dat", "energy")):
        assert np.allclose(read(tmp_path / name), [w[key] for w in want], rtol=1e-10, atol=0), name
    assert np.max(np.abs(read(tmp_path / "rho0.dat").reshape(shape) - o.get(oracle.F_RHO))) <= 1e-10
    final = read(tmp_path / "psi0.dat").reshape(shape)
    assert np.max(np.abs(final - o.get(oracle.F_PSI))) <= 1e-10 * np.max(np.abs(final))
    assert read(tmp_path / "amp.dat").size == shape[0] * shape[2]


def quasi_ic(shape, seed=13):
    z = np.arange(shape[2]) * 2 * np.pi / 8
    x = np.arange(shape[0])[:, None, None]
    rng = np.random.default_rng(seed)
    return (1.3 * np.cos(z)[None, None, :] * 0.5 * (1 - np.tanh((x - shape[0] / 2) / 4.0)) * np.ones((1, shape[1], 1))
            + 0.01 * rng.standard_normal(shape))


def mid(f, shape):
    """The reference's saveMid slice: j = Ny/2, written i-major, k fastest (quasi/quasi.cpp:91-126)."""
    return f[:, shape[1] // 2, :].reshape(-1)


QUASI_KW = dict(dt=0.002, kp=0.3755, divv=10)


def test_driver_quasi_mid_slices_match_oracle(tmp_path):
    """quasi's save iteration: divv.dat (div v in real space), p.dat, rho.dat and energyMid.dat
    mid slices (quasi/quasi.cpp:2417-2487), text with the reference's default 6 significant
    digits, against the oracle after the same 20 steps (past the div v switch at 10)."""
    if not os.path.exists(DRIVER):
        pytest.skip("smadft_run not built")
    shape = (16, 12, 20)
    psi0 = quasi_ic(shape)
    ic = tmp_path / "ic.txt"
    np.savetxt(ic, psi0.reshape(-1), fmt="%.17g")
    args = [DRIVER, "quasi", f"nx={shape[0]}", f"ny={shape[1]}", f"nz={shape[2]}", "nw=8", "eps=-0.7",
            "steps=20", "l1every=10", "saveevery=2", f"ic=file:{ic}", f"out={tmp_path}"]
    args += [f"{k}={v}" for k, v in QUASI_KW.items()]
    subprocess.run(args, check=True, capture_output=True, text=True)
    o = oracle.Oracle(oracle.QUASI, shape, nw=8, eps=-0.7, dt=QUASI_KW["dt"], kp=QUASI_KW["kp"],
                      divv_switch=QUASI_KW["divv"])
    o.set_psi(psi0)
    o.step(20)
    scale = 1.0 / (8.0 * shape[0] * shape[1] * shape[2])
    want = {"divv.dat": scale * oracle.r2r_3d(o.get(oracle.F_DIVV), (1, 1, 1)),
            "p.dat": o.get(oracle.F_P), "rho.dat": o.get(oracle.F_RHO), "energyMid.dat": o.get(oracle.F_ENERGY)}
    for name, f in want.items():
        got = read(tmp_path / name)
        w = mid(f, shape)
        assert got.size == w.size, name
        # 6 significant digits in the text file
        assert np.max(np.abs(got - w)) <= 1e-5 * np.max(np.abs(w)), name
    assert np.abs(want["divv.dat"]).max() > 0


def test_driver_quasi_mid_slices_match_reference_build(tmp_path):
    """The same files against the ones the reference's own quasi source writes (built with the
    single-rank shim in oracle/_ref) on its save iteration, step 500 (stepL1 = 50, every 10th)."""
    if not os.path.exists(DRIVER):
        pytest.skip("smadft_run not built")
    if not oracle.reference_available("quasi"):
        pytest.skip("shimmed reference build absent")
    shape = (16, 12, 20)
    psi0 = quasi_ic(shape, seed=14)
    steps = 500
    kw = dict(QUASI_KW, dt=0.001)     # dt = 0.002 goes non-finite before step 500 on this grid
    _, texts, _ = oracle.run_reference("quasi", shape, steps, psi0=psi0, nw=8, dt=kw["dt"], eps=-0.7,
                                       nu=1.0, kp=kw["kp"], rho0=1.0, divv=kw["divv"])
    ic = tmp_path / "ic.txt"
    np.savetxt(ic, psi0.reshape(-1), fmt="%.17g")
    args = [DRIVER, "quasi", f"nx={shape[0]}", f"ny={shape[1]}", f"nz={shape[2]}", "nw=8", "eps=-0.7",
            f"steps={steps}", "l1every=50", "saveevery=10", f"ic=file:{ic}", f"out={tmp_path}"]
    args += [f"{k}={v}" for k, v in kw.items()]
    subprocess.run(args, check=True, capture_output=True, text=True)
    for name in ("divv.dat", "p.dat", "rho.dat", "energyMid.dat"):
        ref = np.array([float(x) for x in texts[name].split()])
        got = read(tmp_path / name)
        assert got.size == ref.size == shape[0] * shape[2], name
        assert np.max(np.abs(got - ref)) <= 2e-5 * np.max(np.abs(ref)), name
