"""The bounds-check build (libsmadft_check.so, SMADFT_CHECK_BOUNDS) over the models' steps.

Every element index an axis-pass kernel hands to its loader or storer is checked against
the field size; an index outside it sets a device word instead of touching memory.  Each
case runs in a fresh process with SMADFT_LIB=libsmadft_check.so over grids that reach the
register-direct, staged and generic kernels (full and partial tiles, lengths 64/96/128/160 and
odd tile remainders), then asserts that no index was out of range and that the checked
library gives the field of the normal one (to rounding: the extra code changes how the
compiler contracts and schedules the arithmetic).
"""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHECK_LIB = os.path.join(ROOT, "sma-dft_b200", "libsmadft_check.so")

RUN = r"""
import json, sys
import numpy as np
import smadft
out = {}
cases = [
    ("noadv", smadft.NOADV, (16, 12, 40), smadft.FP64, {}),
    ("adv", smadft.ADV, (12, 64, 64), smadft.FP32, dict(dt=0.01)),
    ("adv96", smadft.ADV, (8, 96, 20), smadft.FP32, dict(dt=0.01)),
    ("adv160", smadft.ADV, (6, 160, 36), smadft.FP64, dict(dt=0.01)),
    ("adv128x", smadft.ADV, (128, 6, 40), smadft.FP32, dict(dt=0.01)),
    ("quasi", smadft.QUASI, (8, 64, 64), smadft.FP64, dict(dt=0.002, kp=0.3, divv_switch=2)),
    ("comp", smadft.COMP, (16, 12, 20), smadft.FP32, dict(divv_switch=2, rho_up=4)),
    ("noadvc", smadft.NOADV, (24, 20, 32), smadft.FP32, dict(conserved=1, dt=0.005)),
]
for name, model, shape, prec, kw in cases:
    p = smadft.params(model, shape, precision=prec, **kw)
    z = np.arange(shape[2]) * 2 * np.pi / 8
    x = np.arange(shape[0])[:, None, None]
    psi0 = 1.3 * np.cos(z) * 0.5 * (1 - np.tanh((x - shape[0] / 2) / 4.0)) * np.ones((1, shape[1], 1))
    with smadft.Solver(p) as s:
        s.set_psi(psi0)
        s.step(4)
        d = s.step_diag()
        psi = s.get("psi")
        bad = smadft.bounds_status(s)
    out[name] = {"bad": bad, "psi_sum": float(np.sum(psi * psi)), "rc": d["rc"], "fp32": prec == smadft.FP32}
print(json.dumps(out))
"""


def run(lib):
    env = dict(os.environ, SMADFT_LIB=lib)
    r = subprocess.run([sys.executable, "-c", RUN], cwd=os.path.join(ROOT, "sma-dft_b200"), env=env,
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_bounds_check_build_sees_no_out_of_range_index():
    if not os.path.exists(CHECK_LIB):
        pytest.skip("libsmadft_check.so not built (make -C sma-dft_b200 check)")
    checked = run("libsmadft_check.so")
    normal = run("libsmadft.so")
    for name, r in checked.items():
        assert r["bad"] == 0, name
        assert r["rc"] == 0, name
        tol = 1e-6 if r["fp32"] else 1e-12
        assert abs(r["psi_sum"] - normal[name]["psi_sum"]) <= tol * abs(normal[name]["psi_sum"]), name
    assert all(r["bad"] == -6 for r in normal.values())   # the normal build does not check
