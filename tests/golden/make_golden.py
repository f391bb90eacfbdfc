"""Generate tests/golden/*.npz from the reference's own sources.

The reference has no tests or golden files of its own, so the vectors here come from the
reference loop bodies themselves: oracle/build_ref.sh compiles no-adv/cosNoAdvTrackSing.cpp,
no-adv/cosNoAdvTrackBump.cpp, no-adv/cosNoAdvConserv.cpp, adv/cosAdvTrackMult.cpp,
adv/cosAdvConSingle.cpp, quasi/quasi.cpp and compressible/compressible.cpp with a single-rank
MPI shim and an FFTW-r2r shim (oracle/r2r.c), and this script runs them on small seeded
grids, recording the initial condition, the final fields and the text diagnostics.

    python tests/golden/make_golden.py [name ...]   # needs oracle/_ref/ (run oracle/build_ref.sh)

Each case is (model, shape, steps, IC amplitude, interface normal, parameters).  The shapes are deliberately not cubic so
that axis mix-ups show.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402

CASES = {
    # name: (reference binary, shape, steps, IC amplitude, interface normal, params)
    "noadv_16x12x20_s40": ("noadv", (16, 12, 20), 40, 0.5, 0, dict(nw=8, dt=0.05, eps=-0.75)),
    "noadv_24x16x20_s100": ("noadv", (24, 16, 20), 100, 1.328, 0, dict(nw=8, dt=0.05, eps=-0.75)),
    "adv_16x12x20_s20": ("adv", (16, 12, 20), 20, 1.328, 0, dict(nw=8, dt=0.02, eps=-0.75, nu=1.0)),
    "adv_20x16x12_s100": ("adv", (20, 16, 12), 100, 1.328, 0, dict(nw=8, dt=0.02, eps=-0.75, nu=1.0)),
    "quasi_16x12x20_s20_kp0": ("quasi", (16, 12, 20), 20, 1.328, 0,
                               dict(nw=8, dt=0.005, eps=-0.75, nu=1.0, kp=0.0, rho0=1.0, divv=200)),
    "quasi_16x12x20_s60_kp": ("quasi", (16, 12, 20), 60, 1.328, 0,
                              dict(nw=8, dt=0.002, eps=-0.75, nu=1.0, kp=0.3755, rho0=1.0, divv=20)),
    "bump_16x12x32_s1000": ("bump", (16, 12, 32), 1000, 1.328, 2, dict(nw=8, dt=0.05, eps=-0.7)),
    # conserved dynamics (no-adv/cosNoAdvConserv.cpp, adv/cosAdvConSingle.cpp): the q^2-weighted
    # explicit term needs a smaller step than the non-conserved runs at nw = 8
    "noadvc_16x12x20_s200": ("noadvc", (16, 12, 20), 200, 1.328, 0, dict(nw=8, dt=0.005, eps=-0.75)),
    "advc_16x12x20_s100": ("advc", (16, 12, 20), 100, 1.328, 0, dict(nw=8, dt=0.005, eps=-0.75, nu=1.0)),
    # compressible/compressible.cpp: 40 relaxation steps (rho from the amplitude, shifted up
    # by rho_up) then the independent density
    "comp_16x12x20_s100": ("comp", (16, 12, 20), 100, 1.3, 0,
                           dict(nw=8, dt=0.001, eps=-0.75, nu=1.0, rho0=0.01, zeta=0.001, rho_up=16, divv=40)),
}


def seeded_ic(shape, seed, A=0.5, normal=0, nw=8.0, q0=1.0):
    """Smectic layers A cos(q0 z) behind an interface, plus U(-1e-3, 1e-3) (numpy PCG64).

    normal=0: x-normal interface, envelope 1/2 (1 - tanh((x - L/2)/(2 lambda0))) (the configs').
    normal=2: z-normal interface at z0 = Lz/2 + lambda0 sin(2 pi x / Lx) (smectic below, as the
    reference's bump tracker expects; it scans z from the top).
    """
    nx, ny, nz = shape
    dx = 2 * np.pi / (q0 * nw)
    lam = 2 * np.pi / q0
    x = np.arange(nx) * dx
    z = np.arange(nz) * dx
    layers = np.cos(q0 * z)[None, None, :]
    if normal == 0:
        env = 0.5 * (1 - np.tanh((x - nx * dx / 2) / (2 * lam)))[:, None, None]
    else:
        z0 = nz * dx / 2 + lam * np.sin(2 * np.pi * x / (nx * dx))
        env = 0.5 * (1 - np.tanh((z[None, :] - z0[:, None]) / (2 * lam)))[:, None, :]
    psi = A * layers * env * np.ones((1, ny, 1))
    rng = np.random.default_rng(seed)
    return psi + rng.uniform(-1e-3, 1e-3, shape)


def parse_dat(text: str) -> np.ndarray:
    vals = [float(t) for t in text.split()]
    return np.array(vals, dtype=np.float64)


def make(name: str) -> str:
    which, shape, steps, amp, normal, params = CASES[name]
    psi0 = seeded_ic(shape, seed=1234 + list(CASES).index(name), A=amp, normal=normal)
    fields, texts, _ = oracle.run_reference(which, shape, steps, psi0=psi0, **params)
    out = dict(psi0=psi0, shape=np.array(shape), steps=np.array(steps),
               which=np.array(which), params_keys=np.array(list(params.keys())),
               params_vals=np.array([float(v) for v in params.values()]))
    for k, v in fields.items():
        out["f_" + k] = v
    for fn, txt in texts.items():
        arr = parse_dat(txt)
        if arr.size:
            out["t_" + fn.replace(".dat", "")] = arr
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **out)
    return path


def main():
    if not all(oracle.reference_available(w) for w in oracle.REF_BINARIES):
        raise SystemExit("oracle/_ref is not built: run oracle/build_ref.sh first")
    for name in sys.argv[1:] or CASES:
        p = make(name)
        print("wrote", p, os.path.getsize(p), "bytes")


if __name__ == "__main__":
    main()
