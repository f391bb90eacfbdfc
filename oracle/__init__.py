"""FP64 CPU oracle for sma-dft's time-step loop -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import
this package; the product library never does.

* :class:`Oracle` wraps ``liboracle.so`` (oracle.c / r2r.c), the clean C restatement of
  the reference's loop bodies (no-adv/cosNoAdvTrackSing.cpp:681-1074,
  adv/cosAdvTrackMult.cpp:824-1744, quasi/quasi.cpp:1099-2498).
* :func:`run_reference` runs the reference's own sources, compiled by ``build_ref.sh``
  into ``oracle/_ref/`` against a single-rank MPI / FFTW-r2r shim, and returns its final
  fields; it pins the oracle (tests/test_oracle_pin.py) and produced tests/golden/.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

NOADV, ADV, QUASI, COMP = 0, 1, 2, 3
F_PSI, F_PSIHAT, F_VX, F_VY, F_VZ, F_GX, F_GY, F_GZ = range(8)
F_RHO, F_P, F_DIVV, F_MU, F_ENERGY, F_NHAT = range(8, 14)
F_AMP, F_VSOLX, F_VSOLY, F_VSOLZ, F_VIRRX, F_VIRRY, F_VIRRZ, F_FRHO = range(14, 22)
REDFT10, REDFT01, RODFT10, RODFT01 = 0, 1, 2, 3


class OrcParams(ctypes.Structure):
    _fields_ = [
        ("model", ctypes.c_int),
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("nw", ctypes.c_double), ("dt", ctypes.c_double),
        ("alpha", ctypes.c_double), ("beta", ctypes.c_double), ("gamma", ctypes.c_double),
        ("eps", ctypes.c_double), ("q0", ctypes.c_double),
        ("nu", ctypes.c_double),
        ("rho0", ctypes.c_double), ("kp", ctypes.c_double), ("amp", ctypes.c_double),
        ("divv_switch", ctypes.c_int), ("loaded", ctypes.c_int),
        ("conserved", ctypes.c_int),
        ("zeta", ctypes.c_double), ("rho_up", ctypes.c_int),
    ]


_lib = None


def build() -> str:
    """Compile liboracle.so in place (gcc with OpenMP)."""
    subprocess.run(["make", "-s", "-C", HERE, "CC_OMP=gcc"], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.POINTER(OrcParams)]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_set_psi.argtypes = [ctypes.c_void_p, dp]
        L.orc_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_get.argtypes = [ctypes.c_void_p, ctypes.c_int, dp]
        L.orc_diag.argtypes = [ctypes.c_void_p, dp]
        L.orc_free_energy.argtypes = [ctypes.c_void_p]
        L.orc_free_energy.restype = ctypes.c_double
        L.orc_track.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                ctypes.c_double, ctypes.c_double,
                                ctypes.POINTER(ctypes.c_int), dp]
        L.orc_step_surface.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), dp, dp, dp]
        L.orc_r2r_1d.argtypes = [dp, dp, ctypes.c_int, ctypes.c_int]
        L.orc_r2r_3d.argtypes = [dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                 ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_get_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def get_threads() -> int:
    return int(lib().orc_get_threads())


def r2r_1d(x, kind: int) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty_like(x)
    lib().orc_r2r_1d(_dp(x), _dp(y), x.size, kind)
    return y


def r2r_3d(x, kinds) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty_like(x)
    lib().orc_r2r_3d(_dp(x), _dp(y), x.shape[0], x.shape[1], x.shape[2], *kinds)
    return y


DEFAULTS = dict(nw=8.0, dt=0.05, alpha=1.0, beta=2.0, gamma=1.0, eps=-0.75, q0=1.0, nu=1.0,
                rho0=1.0, kp=0.0, amp=1.34164, divv_switch=200, loaded=0, conserved=0,
                zeta=0.001, rho_up=16)


class Oracle:
    """One FP64 CPU run of a model on an (nx, ny, nz) grid."""

    def __init__(self, model: int, shape, **kw):
        p = dict(DEFAULTS)
        p.update(kw)
        self.shape = tuple(int(s) for s in shape)
        ints = {name for name, t in OrcParams._fields_ if t is ctypes.c_int}
        self.params = OrcParams(model=int(model), nx=self.shape[0], ny=self.shape[1], nz=self.shape[2],
                                **{k: (int(p[k]) if k in ints else p[k]) for k in DEFAULTS})
        self._c = lib().orc_create(ctypes.byref(self.params))
        if not self._c:
            raise ValueError("orc_create rejected the parameters")

    def __del__(self):
        c = getattr(self, "_c", None)
        if c:
            lib().orc_destroy(c)
            self._c = None

    def set_psi(self, psi) -> None:
        a = np.ascontiguousarray(psi, dtype=np.float64).reshape(self.shape)
        lib().orc_set_psi(self._c, _dp(a))

    def step(self, n: int = 1) -> None:
        if lib().orc_step(self._c, int(n)) != 0:
            raise RuntimeError("orc_step failed (no initial condition?)")

    def get(self, field: int = F_PSI) -> np.ndarray:
        out = np.empty(self.shape, dtype=np.float64)
        if lib().orc_get(self._c, int(field), _dp(out)) != 0:
            raise ValueError(f"field {field} not available for this model")
        return out

    def diag(self) -> dict:
        d = np.zeros(5)
        lib().orc_diag(self._c, _dp(d))
        return dict(l1=d[0], mass=d[1], energy=d[2], mean=d[3], steps=int(d[4]))

    def free_energy(self) -> float:
        return float(lib().orc_free_energy(self._c))

    def track(self, axis: int = 2, mode: int = 0, hi: float = 0.7, lo: float = 0.0,
              field: int = F_PSI):
        dims = [s for a, s in enumerate(self.shape) if a != axis]
        idx = np.empty(dims, dtype=np.int32)
        pos = np.empty(dims, dtype=np.float64)
        lib().orc_track(self._c, field, axis, mode, hi, lo,
                        idx.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _dp(pos))
        return idx, pos

    def step_surface(self):
        """One step with the surface diagnostics: per (i, j) column the interface index
        along z (-1: none), normal velocity, 2H and K (NaN: none)."""
        shp = (self.shape[0], self.shape[1])
        idx = np.empty(shp, dtype=np.int32)
        vel, h, k = (np.empty(shp) for _ in range(3))
        rc = lib().orc_step_surface(self._c, idx.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _dp(vel), _dp(h),
                                    _dp(k))
        if rc:
            raise RuntimeError("orc_step_surface failed")
        return idx, vel, h, k


# ----------------------------------------------------------------------------------
# The reference itself, compiled from its sources by build_ref.sh (single-rank shims).
# ----------------------------------------------------------------------------------
REF_BINARIES = {"noadv": "noadv_ref", "bump": "bump_ref", "adv": "adv_ref", "quasi": "quasi_ref",
                "noadvc": "noadvc_ref", "advc": "advc_ref", "comp": "comp_ref"}
REF_DUMPS = {
    "noadv": ["psi", "nq"],
    "noadvc": ["psi", "nq"],
    "advc": ["psi", "vx", "vy", "vz", "gx", "gy", "gz", "nq"],
    "comp": ["psi", "rho", "psiq", "amp", "divv", "mu", "vsolx", "vsoly", "vsolz", "virrx", "virry", "virrz",
             "nl", "frho"],
    "bump": ["psi"],
    "adv": ["psi", "vx", "vy", "vz", "gx", "gy", "gz", "nq"],
    "quasi": ["psi", "rho", "p", "vx", "vy", "vz", "mu", "energy", "psiq"],
}


def reference_available(which: str = "noadv") -> bool:
    return os.path.exists(os.path.join(REF_DIR, REF_BINARIES[which]))


def run_reference(which: str, shape, steps: int, psi0=None, workdir: str | None = None,
                  threads: int | None = None, **params):
    """Run the shimmed reference build; returns (fields dict, text outputs dict, stdout).

    ``params`` keys: nw, dt, eps, alpha, beta, gamma, nu, kp, rho0, divv (quasi switch).
    ``psi0`` replaces the reference's own IC after its IC block (None keeps its IC).
    """
    exe = os.path.join(REF_DIR, REF_BINARIES[which])
    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    own = workdir is None
    tmp = tempfile.TemporaryDirectory() if own else None
    wd = tmp.name if own else workdir
    try:
        env = dict(os.environ)
        nx, ny, nz = shape
        env.update(REFSHIM_NX=str(nx), REFSHIM_NY=str(ny), REFSHIM_NZ=str(nz),
                   REFSHIM_STEPS=str(int(steps)), REFSHIM_DIR=wd)
        if threads:
            env["OMP_NUM_THREADS"] = str(int(threads))
        for k, v in params.items():
            env["REFSHIM_" + k.upper()] = repr(float(v))
        if psi0 is not None:
            ic = os.path.join(wd, "ic.bin")
            np.ascontiguousarray(psi0, dtype=np.float64).tofile(ic)
            env["REFSHIM_IC"] = ic
        else:
            env.pop("REFSHIM_IC", None)
        argv = [exe]
        if which == "adv":
            argv += ["1", "75", "10", "0"]          # nu e0d radius load
            os.makedirs(os.path.join(wd, "r1-e0d75-r10"), exist_ok=True)
        elif which == "quasi":
            argv += ["1", "75", "10", "0"]
            os.makedirs(os.path.join(wd, "r1-e0d75"), exist_ok=True)
        elif which == "comp":
            argv += ["1", "75", "10", "0"]          # nu e0d radius load
        elif which == "noadvc":
            argv += ["75", "10", str(nx), "0"]      # e0d radius N load
            os.makedirs(os.path.join(wd, "r75-r10"), exist_ok=True)
        elif which == "advc":
            argv += ["1", "75", "10", str(nx), "0"]  # nu e0d radius N load
            os.makedirs(os.path.join(wd, "r1-e0d75-r10"), exist_ok=True)
        r = subprocess.run(argv, cwd=wd, env=env, capture_output=True, text=True, check=True)
        fields = {}
        for name in REF_DUMPS[which]:
            fp = os.path.join(wd, name + ".bin")
            fields[name] = np.fromfile(fp, dtype=np.float64).reshape(shape)
        texts = {}
        for root, _, files in os.walk(wd):
            for fn in files:
                if fn.endswith(".dat") and not fn.startswith("psi"):
                    with open(os.path.join(root, fn)) as fh:
                        texts[fn] = fh.read()
        return fields, texts, r.stdout
    finally:
        if tmp is not None:
            tmp.cleanup()
