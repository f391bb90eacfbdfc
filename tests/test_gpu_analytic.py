"""Single-mode and projection identities of the discrete model, on the GPU path.

1. With N = 0 (beta = gamma = 0) a single DCT-II mode cos(pi a (i+1/2)/nx) ... is an
   eigenvector of every step: psi_n = (C1/C2)^n psi_0 with C1,2 = 1 +- dt/2 L(q)
   (no-adv/cosNoAdvTrackSing.cpp:594-602), and with q^2 L in place of L for conserved runs
   (no-adv/cosNoAdvConserv.cpp:646-650).
2. The Stokes projection (adv/cosAdvTrackMult.cpp:1103-1274) is divergence-free in the
   discrete DST/DCT sense: the velocity spectra of one physical wavevector
   K = (pi I/Lx, pi J/Ly, pi K/Lz) sit at vx-hat[I-1, J, K], vy-hat[I, J-1, K],
   vz-hat[I, J, K-1], and K . v-hat = 0 except where the reference's truncations zero a
   component (vy-hat, vz-hat at j = ny-1 or k = nz-1).
3. Quasi with kp = 0 has uniform density: rho = rho_0 and div v = 0 (quasi/quasi.cpp:1322-1377).
"""
import numpy as np
import pytest

import oracle
import smadft

pytestmark = pytest.mark.gpu


def mode(shape, a, b, c, amp=0.8):
    i, j, k = (np.arange(n) + 0.5 for n in shape)
    return amp * (np.cos(np.pi * a * i / shape[0])[:, None, None] * np.cos(np.pi * b * j / shape[1])[None, :, None]
                  * np.cos(np.pi * c * k / shape[2])[None, None, :])


@pytest.mark.parametrize("precision,tol", [(smadft.FP64, 1e-12), (smadft.FP32, 2e-6)])
@pytest.mark.parametrize("conserved", [0, 1])
def test_single_mode_decays_by_the_cn_factor(precision, tol, conserved):
    shape, (a, b, c) = (16, 12, 20), (3, 2, 5)
    dt, steps = 0.02 if conserved else 0.05, 40
    p = smadft.params(smadft.NOADV, shape, precision=precision, beta=0.0, gamma=0.0, eps=-0.3, dt=dt,
                      conserved=conserved)
    q2 = sum((m * p.q0 * p.nw / (2 * n)) ** 2 for m, n in zip((a, b, c), shape))   # (pi m / L)^2, L = n 2 pi/(q0 nw)
    L = p.eps - p.alpha * (q2 - p.q0 ** 2) ** 2
    if conserved:
        L = q2 * L
    g = (1 + dt / 2 * L) / (1 - dt / 2 * L)
    psi0 = mode(shape, a, b, c)
    with smadft.Solver(p) as s:
        s.set_psi(psi0)
        s.step(steps)
        got = s.get("psi")
    want = g ** steps * psi0
    assert np.max(np.abs(got - want)) <= tol * np.max(np.abs(psi0))
    assert g ** steps < 0.9          # the mode did decay


def test_stokes_velocity_is_divergence_free():
    shape = (16, 12, 20)
    p = smadft.params(smadft.ADV, shape, dt=0.02)
    psi0 = smadft.ic_conics(p, A=1.3, count=2, rmin=1.0, rmax=2.0, noise=1e-2, seed=4)
    with smadft.Solver(p) as s:
        s.set_psi(psi0)
        s.step(3)
        v = [s.get(f) for f in ("vx", "vy", "vz")]
    n = np.prod(shape)
    R10, S10 = oracle.REDFT10, oracle.RODFT10
    # forward kinds of each component (sine along its own axis); iST then ST scales by 8 n
    vh = [oracle.r2r_3d(v[0], (S10, R10, R10)) / (8 * n), oracle.r2r_3d(v[1], (R10, S10, R10)) / (8 * n),
          oracle.r2r_3d(v[2], (R10, R10, S10)) / (8 * n)]
    nx, ny, nz = shape
    qx, qy, qz = (np.arange(m) * p.q0 * p.nw / (2 * m) for m in shape)   # pi I / L
    div = np.zeros(shape)
    div[1:, :, :] += qx[1:, None, None] * vh[0][:-1, :, :]
    div[:, 1:, :] += qy[None, 1:, None] * vh[1][:, :-1, :]
    div[:, :, 1:] += qz[None, None, 1:] * vh[2][:, :, :-1]
    scale = max(np.max(np.abs(h)) for h in vh) * np.sqrt(qx[-1] ** 2 + qy[-1] ** 2 + qz[-1] ** 2)
    inner = div[:, : ny - 1, : nz - 1]               # outside the truncated modes
    assert np.max(np.abs(inner)) <= 1e-11 * scale
    assert np.max(np.abs(div)) > 1e-6 * scale       # the truncations do leave a divergence


def test_quasi_without_density_coupling_keeps_rho_uniform():
    shape = (16, 12, 20)
    p = smadft.params(smadft.QUASI, shape, dt=0.002, kp=0.0, rho0=1.0, divv_switch=2)
    psi0 = smadft.ic_interface(p, A=1.3, noise=1e-3, seed=8)
    with smadft.Solver(p) as s:
        s.set_psi(psi0)
        s.step(6)
        rho, divv = s.get("rho"), s.get("divv")
        d = s.step_diag()
    assert np.max(np.abs(rho - 1.0)) <= 1e-13
    assert np.max(np.abs(divv)) / (8 * np.prod(shape)) <= 1e-11   # REDFT10^3 of div v (unnormalised)
    assert abs(d["mass"] - np.prod(shape) * (2 * np.pi / 8) ** 3) <= 1e-10 * d["mass"]
