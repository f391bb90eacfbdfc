"""Host-side pieces of bench.py (no GPU): the numpy initial condition both arms use, and the
reference arm's independence from the product library."""
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_numpy_ic_matches_the_library_builder():
    """bench.make_ic restates smadft_ic_conics (same SplitMix64 counter stream, same blend);
    the two agree to rounding (libm and numpy transcendental functions differ in the last bit)."""
    sys.path.insert(0, ROOT)
    import bench
    import smadft
    for shape, rr in (((16, 12, 20), (1.0, 2.0)), ((40, 24, 32), (1.5, 2.5))):
        p = smadft.params(smadft.ADV, shape, **bench.CFG)
        want = smadft.ic_conics(p, A=1.328, count=4, rmin=rr[0], rmax=rr[1], noise=1e-3, seed=20240601)
        got = bench.make_ic(shape, rmin=rr[0], rmax=rr[1])
        assert got.shape == want.shape
        assert np.max(np.abs(got - want)) <= 1e-14


def test_reference_arm_never_loads_the_product_library():
    """--impl reference prints its line without importing smadft (the reference's own timing
    is replaced by a stub here: it takes minutes at 256^3)."""
    code = (
        "import sys, json, types; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '2', '--warmup', '1'];"
        "import bench;"
        "calls = [];"
        "bench.cpu_reference_run = lambda steps, psi0, threads: (calls.append(steps) or (1.0, float(steps), 'reference', 'stub'));"
        "bench.main();"
        "assert calls == [3, 2], calls;"
        "assert 'smadft' not in sys.modules;"
        "print('ok')"
    )
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    import json
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["steps"] == 2 and d["warmup"] == 3   # warm-up is at least 3
    assert r.stdout.strip().endswith("ok")
