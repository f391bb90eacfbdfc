"""Distinct contexts driven from different host threads at the same time: each run's result
is bit-identical to the same run made alone (the C ABI releases the GIL through ctypes, so
the calls overlap; a single context is not shared between threads)."""
import threading

import numpy as np
import pytest

import smadft

pytestmark = pytest.mark.gpu

CASES = [
    (smadft.ADV, (32, 64, 64), dict(dt=0.01)),
    (smadft.NOADV, (48, 40, 36), dict()),
    (smadft.QUASI, (16, 64, 64), dict(dt=0.002, kp=0.3, divv_switch=2)),
    (smadft.COMP, (24, 32, 40), dict(divv_switch=2, rho_up=4)),
]


def run(case, steps=6, precision=smadft.FP32):
    model, shape, kw = case
    p = smadft.params(model, shape, precision=precision, **kw)
    psi0 = smadft.ic_conics(p, A=1.3, count=2, rmin=1.0, rmax=2.0, noise=1e-3, seed=11)
    with smadft.Solver(p) as s:
        s.set_psi(psi0)
        s.step(steps - 1)
        s.step_diag()
        return s.get("psi")


def test_contexts_on_separate_threads_match_solo_runs():
    rounds = []
    for _ in range(2):                  # the concurrent round first: it takes the first launches
        got = [None] * len(CASES)
        errs = []

        def work(i):
            try:
                got[i] = run(CASES[i])
            except Exception as e:      # reported below
                errs.append(e)
        threads = [threading.Thread(target=work, args=(i,)) for i in range(len(CASES))]
        for t in threads:
            t.start()
        for t in threads:
            t.join(timeout=300)
        assert not errs, errs
        rounds.append(got)
    solo = [run(c) for c in CASES]
    for got in rounds:
        for i in range(len(CASES)):
            assert np.array_equal(got[i], solo[i]), i
