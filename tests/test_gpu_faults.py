"""Failures made on the host (no GPU fault is ever provoked): an allocation that reports
out-of-memory, and damaged checkpoint files.  Each must return its error code and leave
the device and the run as they were.
"""
import os

import numpy as np
import pytest

import smadft

pytestmark = pytest.mark.gpu


def test_failed_allocation_cleans_up(monkeypatch):
    import torch
    p = smadft.params(smadft.ADV, (128, 128, 128))        # 15 fields of 16 MiB
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for k in (0, 4, 14):
        for _ in range(4):
            monkeypatch.setenv("SMADFT_FAIL_ALLOC", str(k))
            with pytest.raises(smadft.SmadftError) as e:
                smadft.Solver(p)
            assert e.value.code == -3
    monkeypatch.delenv("SMADFT_FAIL_ALLOC")
    torch.cuda.synchronize()
    assert abs(torch.cuda.mem_get_info()[0] - free0) < 64 << 20     # nothing left behind
    with smadft.Solver(smadft.params(smadft.NOADV, (16, 12, 20))) as s:   # and the library still works
        s.set_psi(np.cos(np.arange(20) * 2 * np.pi / 8) * np.ones((16, 12, 20)))
        s.step(3)
        assert np.all(np.isfinite(s.get("psi")))


def _run_with_damaged_checkpoint(tmp_path, damage, code):
    shape = (16, 12, 20)
    p = smadft.params(smadft.ADV, shape, dt=0.01)
    psi0 = smadft.ic_conics(p, A=1.3, count=2, rmin=1.0, rmax=2.0, seed=2)
    good = str(tmp_path / "good.ck")
    with smadft.Solver(p) as s:
        s.set_psi(psi0)
        s.step(4)
        s.save(good)
    raw = bytearray(open(good, "rb").read())
    bad = str(tmp_path / "bad.ck")
    open(bad, "wb").write(damage(raw))
    with smadft.Solver(p) as a, smadft.Solver(p) as b:
        a.set_psi(psi0)
        b.set_psi(psi0)
        a.step(2)
        b.step(2)
        with pytest.raises(smadft.SmadftError) as e:
            a.load(bad)
        assert e.value.code == code
        a.step(3)                      # the run goes on from its own state
        b.step(3)
        assert np.array_equal(a.get("psi"), b.get("psi"))


def test_truncated_checkpoint_leaves_the_run(tmp_path):
    _run_with_damaged_checkpoint(tmp_path, lambda raw: bytes(raw[: len(raw) * 2 // 3]), -7)


def test_checkpoint_with_bad_magic_is_rejected(tmp_path):
    _run_with_damaged_checkpoint(tmp_path, lambda raw: b"NOTACKPT" + bytes(raw[8:]), -7)


def test_checkpoint_with_a_foreign_slot_is_rejected(tmp_path):
    def relabel(raw):
        # header: magic(8) version(4) params steps(8) n(8) nslots(4); then per slot id(4) + data
        import ctypes
        off = 8 + 4 + ctypes.sizeof(smadft.Params) + 8 + 8 + 4
        raw[off:off + 4] = (999).to_bytes(4, "little")
        return bytes(raw)
    _run_with_damaged_checkpoint(tmp_path, relabel, -7)


def test_checkpoint_holding_nan_is_rejected(tmp_path):
    def plant_nan(raw):
        raw[-8:] = np.array([np.nan]).tobytes()      # last element of the last slot
        return bytes(raw)
    _run_with_damaged_checkpoint(tmp_path, plant_nan, -4)
