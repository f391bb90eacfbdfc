"""C-ABI surface and host logic (no GPU needed).

* libsmadft.so loads and exports every function include/smadft.h declares;
* parameter validation and error strings;
* the host-only initial-condition builders;
* without a CUDA device, smadft_create fails loudly (SMADFT_ERR_NODEVICE), never falls back.
"""
import ctypes
import os
import re

import numpy as np
import pytest

import smadft

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "smadft.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(smadft_\w+)\s*\(", text)))


def test_header_declares_core_entry_points():
    names = declared_functions()
    for must in ("smadft_create", "smadft_step", "smadft_set_psi", "smadft_get_psi",
                 "smadft_step_diag", "smadft_track", "smadft_destroy"):
        assert must in names


def test_library_exports_every_declared_symbol(smadft_lib):
    missing = [n for n in declared_functions() if not hasattr(smadft_lib, n)]
    assert not missing, missing


def test_python_mirror_binds_every_declared_symbol():
    bound = {name for name, _, _ in smadft.SIGNATURES}
    assert set(declared_functions()) <= bound


def test_params_defaults_and_check(smadft_lib):
    p = smadft.params(smadft.NOADV, (64, 64, 64))
    assert p.alpha == 1.0 and p.beta == 2.0 and p.gamma == 1.0 and p.eps == -0.75 and p.nw == 8.0
    assert p.dt == 0.05
    assert smadft_lib.smadft_params_check(ctypes.byref(p)) == 0
    assert smadft.params(smadft.ADV).dt == 0.02


@pytest.mark.parametrize("field,value,code", [
    ("nx", 7, -6), ("nx", 14, -6), ("ny", 2, -1), ("nz", 2048, -6), ("dt", 0.0, -1),
    ("nw", -1.0, -1), ("precision", 5, -1), ("model", 9, -1),
])
def test_params_check_rejects(smadft_lib, field, value, code):
    p = smadft.params(smadft.ADV, (32, 32, 32))
    setattr(p, field, value)
    assert smadft_lib.smadft_params_check(ctypes.byref(p)) == code


def test_quasi_and_adv_need_positive_viscosity(smadft_lib):
    p = smadft.params(smadft.ADV, (16, 16, 16), nu=0.0)
    assert smadft_lib.smadft_params_check(ctypes.byref(p)) == -1
    p = smadft.params(smadft.NOADV, (16, 16, 16), nu=0.0)
    assert smadft_lib.smadft_params_check(ctypes.byref(p)) == 0


def test_conserved_flag_only_for_noadv_and_adv(smadft_lib):
    for model in (smadft.NOADV, smadft.ADV):
        p = smadft.params(model, (16, 16, 16), conserved=1)
        assert smadft_lib.smadft_params_check(ctypes.byref(p)) == 0
        p.conserved = 2
        assert smadft_lib.smadft_params_check(ctypes.byref(p)) == -1
    p = smadft.params(smadft.QUASI, (16, 16, 16), conserved=1)
    assert smadft_lib.smadft_params_check(ctypes.byref(p)) == -1
    assert ctypes.sizeof(smadft.Params) == 176       # conserved and rho_up in reserved ints, then zeta


def test_comp_parameter_checks(smadft_lib):
    p = smadft.params(smadft.COMP, (16, 16, 24))
    assert (p.dt, p.rho0, p.zeta, p.rho_up) == (0.001, 0.01, 0.001, 16)
    assert smadft_lib.smadft_params_check(ctypes.byref(p)) == 0
    p.rho_up = 24                        # must stay below nz
    assert smadft_lib.smadft_params_check(ctypes.byref(p)) == -1
    p.rho_up = 16
    p.loaded = 1                         # the reference's load branch also reads rho from files
    assert smadft_lib.smadft_params_check(ctypes.byref(p)) == -6


def test_error_strings(smadft_lib):
    assert smadft_lib.smadft_error_string(-4) == b"non-finite field"
    assert smadft_lib.smadft_abi_version() == 1


def test_ic_interface_formula(smadft_lib):
    p = smadft.params(smadft.NOADV, (16, 12, 20))
    psi = smadft.ic_interface(p, A=0.5, bump=0.0, noise=0.0)
    dx = 2 * np.pi / 8
    x = np.arange(16) * dx
    z = np.arange(20) * dx
    ref = 0.5 * np.cos(z)[None, None, :] * (0.5 * (1 - np.tanh((x - 8 * dx) / (4 * np.pi))))[:, None, None]
    assert np.allclose(psi, np.broadcast_to(ref, psi.shape), rtol=0, atol=1e-15)


def test_ic_noise_is_seeded_and_bounded(smadft_lib):
    p = smadft.params(smadft.NOADV, (8, 8, 8))
    a = smadft.ic_interface(p, A=0.0, noise=1e-3, seed=5)
    b = smadft.ic_interface(p, A=0.0, noise=1e-3, seed=5)
    c = smadft.ic_interface(p, A=0.0, noise=1e-3, seed=6)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    assert np.abs(a).max() <= 1e-3 and np.abs(a).max() > 5e-4
    assert abs(a.mean()) < 2e-4


def test_ic_bump_moves_interface(smadft_lib):
    p = smadft.params(smadft.NOADV, (32, 32, 16))
    flat = smadft.ic_interface(p, A=1.0, bump=0.0, noise=0.0)
    bump = smadft.ic_interface(p, A=1.0, bump=2 * 2 * np.pi, noise=0.0)
    assert not np.allclose(flat, bump)
    assert np.allclose(flat[:, 0], bump[:, 0])          # sin(0) = 0 at j = 0


def test_ic_conics_seeded(smadft_lib):
    p = smadft.params(smadft.ADV, (24, 24, 24))
    a = smadft.ic_conics(p, count=4, seed=1)
    b = smadft.ic_conics(p, count=4, seed=1)
    c = smadft.ic_conics(p, count=4, seed=2)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    assert np.abs(a).max() <= 0.5 + 1e-3 + 1e-12


def test_create_without_device_fails_loudly(smadft_lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    p = smadft.params(smadft.NOADV, (16, 16, 16))
    with pytest.raises(smadft.SmadftError) as e:
        smadft.Solver(p)
    assert e.value.code == -9
