"""Python mirror of the smadft C ABI (include/smadft.h), via ctypes.

The reference's per-step loop body (no-adv/cosNoAdvTrackSing.cpp:681-1074,
adv/cosAdvTrackMult.cpp:824-1744, quasi/quasi.cpp:1099-2498) is replaced by calls into
``libsmadft.so``; this module only marshals arguments.  It never falls back to a CPU
implementation: if the library (or a CUDA device) is missing, calls raise.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# SMADFT_LIB selects another build of the library in this directory (libsmadft_check.so: the
# bounds-check build)
LIB_PATH = os.path.join(PKG_DIR, os.environ.get("SMADFT_LIB", "libsmadft.so"))

NOADV, ADV, QUASI, COMP = 0, 1, 2, 3
FP64, FP32 = 0, 1
FIELD = dict(psi=0, psihat=1, vx=2, vy=3, vz=4, gx=5, gy=6, gz=7, rho=8, p=9, divv=10, mu=11,
             energy=12, nhat=13, amp=14, virrx=15, virry=16, virrz=17, frho=18, divv_real=19)
TRACK_FLAT, TRACK_BUMP, TRACK_LEVEL = 0, 1, 2
REDFT10, REDFT01, RODFT10, RODFT01 = 0, 1, 2, 3

ERRORS = {0: "ok", -1: "invalid argument", -2: "CUDA error", -3: "out of memory",
          -4: "non-finite field", -5: "device wait timed out", -6: "unsupported grid length",
          -7: "checkpoint I/O error", -8: "call out of order", -9: "no CUDA device",
          -10: "grid exceeds the no-alloc scratch maximum"}
NOALLOC_MAX_BYTES = 16 << 20


class SmadftError(RuntimeError):
    def __init__(self, code: int, msg: str = ""):
        self.code = code
        super().__init__(f"smadft error {code} ({ERRORS.get(code, '?')}){': ' + msg if msg else ''}")


class Params(ctypes.Structure):
    """Mirror of ``smadft_params``."""
    _fields_ = [
        ("model", ctypes.c_int), ("precision", ctypes.c_int),
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("nw", ctypes.c_double), ("dt", ctypes.c_double),
        ("alpha", ctypes.c_double), ("beta", ctypes.c_double), ("gamma", ctypes.c_double),
        ("eps", ctypes.c_double), ("q0", ctypes.c_double), ("nu", ctypes.c_double),
        ("rho0", ctypes.c_double), ("kp", ctypes.c_double), ("amp", ctypes.c_double),
        ("divv_switch", ctypes.c_int), ("loaded", ctypes.c_int), ("device", ctypes.c_int),
        ("conserved", ctypes.c_int), ("rho_up", ctypes.c_int), ("reserved", ctypes.c_int * 3),
        ("zeta", ctypes.c_double), ("reserved_d", ctypes.c_double * 3),
    ]


class Diag(ctypes.Structure):
    """Mirror of ``smadft_diag``."""
    _fields_ = [("l1", ctypes.c_double), ("mass", ctypes.c_double), ("energy", ctypes.c_double),
                ("mean", ctypes.c_double), ("steps", ctypes.c_longlong),
                ("nonfinite", ctypes.c_int), ("reserved", ctypes.c_int)]

    def as_dict(self) -> dict:
        return dict(l1=self.l1, mass=self.mass, energy=self.energy, mean=self.mean,
                    steps=int(self.steps), nonfinite=int(self.nonfinite))


class AdjOpts(ctypes.Structure):
    """smadft_adj_opts"""
    _fields_ = [("steps", ctypes.c_int), ("checkpoint_every", ctypes.c_int), ("axis", ctypes.c_int),
                ("mode", ctypes.c_int), ("hi", ctypes.c_double), ("lo", ctypes.c_double)]


class Grads(ctypes.Structure):
    """smadft_grads"""
    _fields_ = [("loss", ctypes.c_double), ("found", ctypes.c_int), ("d_eps", ctypes.c_double),
                ("d_alpha", ctypes.c_double), ("d_beta", ctypes.c_double), ("d_gamma", ctypes.c_double),
                ("d_nu", ctypes.c_double)]


class TuneReport(ctypes.Structure):
    """smadft_tune_report"""
    _fields_ = [("configs", ctypes.c_int), ("chosen", ctypes.c_int), ("ms", ctypes.c_double * 8)]


# (name, restype, argtypes) of every exported entry point declared in include/smadft.h
_P = ctypes.POINTER
_dp = _P(ctypes.c_double)
_vp = ctypes.c_void_p
SIGNATURES = [
    ("smadft_abi_version", ctypes.c_int, []),
    ("smadft_error_string", ctypes.c_char_p, [ctypes.c_int]),
    ("smadft_params_init", None, [_P(Params), ctypes.c_int]),
    ("smadft_params_check", ctypes.c_int, [_P(Params)]),
    ("smadft_create", ctypes.c_int, [_P(Params), _P(_vp)]),
    ("smadft_destroy", ctypes.c_int, [_vp]),
    ("smadft_last_error", ctypes.c_char_p, [_vp]),
    ("smadft_set_psi", ctypes.c_int, [_vp, _dp, ctypes.c_size_t]),
    ("smadft_get_psi", ctypes.c_int, [_vp, _dp, ctypes.c_size_t]),
    ("smadft_get_field", ctypes.c_int, [_vp, ctypes.c_int, _dp, ctypes.c_size_t]),
    ("smadft_step", ctypes.c_int, [_vp, ctypes.c_int]),
    ("smadft_step_diag", ctypes.c_int, [_vp, _P(Diag)]),
    ("smadft_sync", ctypes.c_int, [_vp]),
    ("smadft_track", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                    ctypes.c_double, _P(ctypes.c_int), _dp]),
    ("smadft_free_energy", ctypes.c_int, [_vp, _dp]),
    ("smadft_step_surface", ctypes.c_int, [_vp, _P(ctypes.c_int), _dp, _dp, _dp, _P(Diag)]),
    ("smadft_save_checkpoint", ctypes.c_int, [_vp, ctypes.c_char_p]),
    ("smadft_load_checkpoint", ctypes.c_int, [_vp, ctypes.c_char_p]),
    ("smadft_r2r3d_device", ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    ("smadft_r2r_pass_device", ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int]),
    ("smadft_step_host", ctypes.c_int, [_vp, _dp, ctypes.c_size_t, ctypes.c_int]),
    ("smadft_get_stream", ctypes.c_int, [_vp, _P(_vp)]),
    ("smadft_launch_count", ctypes.c_int, [_vp, _P(ctypes.c_longlong)]),
    ("smadft_r2r3d_noalloc", ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp]),
    ("smadft_batch_create", ctypes.c_int, [_P(Params), ctypes.c_int, _P(_vp)]),
    ("smadft_batch_destroy", ctypes.c_int, [_vp]),
    ("smadft_batch_size", ctypes.c_int, [_vp, _P(ctypes.c_int)]),
    ("smadft_batch_member", ctypes.c_int, [_vp, ctypes.c_int, _P(_vp)]),
    ("smadft_batch_step", ctypes.c_int, [_vp, ctypes.c_int]),
    ("smadft_batch_sync", ctypes.c_int, [_vp]),
    ("smadft_bounds_status", ctypes.c_int, [_vp, _P(ctypes.c_int)]),
    ("smadft_batch_get_stream", ctypes.c_int, [_vp, _P(_vp)]),
    ("smadft_batch_groups", ctypes.c_int, [_vp, _P(ctypes.c_int)]),
    ("smadft_batch_last_error", ctypes.c_char_p, [_vp]),
    ("smadft_autotune", ctypes.c_int, [_vp, ctypes.c_int, _P(TuneReport)]),
    ("smadft_adjoint", ctypes.c_int, [_vp, _P(AdjOpts), _P(Grads), _dp]),
    ("smadft_tune_config_name", ctypes.c_char_p, [ctypes.c_int]),
    ("smadft_ic_interface", ctypes.c_int, [_P(Params), ctypes.c_double, ctypes.c_double,
                                           ctypes.c_double, ctypes.c_ulonglong, _dp]),
    ("smadft_ic_focal_conic", ctypes.c_int, [_P(Params), ctypes.c_double, ctypes.c_double, _dp]),
    ("smadft_ic_conics", ctypes.c_int, [_P(Params), ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_double, ctypes.c_ulonglong, _dp]),
]

_lib = None


def build() -> str:
    """Compile libsmadft.so in place (nvcc -gencode arch=compute_100a,code=sm_100a)."""
    subprocess.run(["make", "-s", "-C", PKG_DIR, "libsmadft.so"], check=True)
    return LIB_PATH


def lib():
    """Load libsmadft.so (raises if it is missing: there is no CPU fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} is not built; run smadft.build() or make -C sma-dft_b200")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def params(model: int, shape=(64, 64, 64), precision: int = FP64, **kw) -> Params:
    p = Params()
    lib().smadft_params_init(ctypes.byref(p), int(model))
    p.nx, p.ny, p.nz = (int(s) for s in shape)
    p.precision = int(precision)
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _check(rc: int, ctx=None):
    if rc != 0:
        msg = ""
        if ctx:
            m = lib().smadft_last_error(ctx)
            msg = m.decode() if m else ""
        raise SmadftError(rc, msg)


def ic_interface(p: Params, A=0.5, bump=0.0, noise=1e-3, seed=20240601) -> np.ndarray:
    out = np.empty((p.nx, p.ny, p.nz), dtype=np.float64)
    _check(lib().smadft_ic_interface(ctypes.byref(p), A, bump, noise, seed, _dptr(out)))
    return out


def ic_focal_conic(p: Params, A=1.328, radius=10.0) -> np.ndarray:
    out = np.empty((p.nx, p.ny, p.nz), dtype=np.float64)
    _check(lib().smadft_ic_focal_conic(ctypes.byref(p), A, radius, _dptr(out)))
    return out


def ic_conics(p: Params, A=0.5, count=4, rmin=3.0, rmax=6.0, noise=1e-3, seed=20240601) -> np.ndarray:
    out = np.empty((p.nx, p.ny, p.nz), dtype=np.float64)
    _check(lib().smadft_ic_conics(ctypes.byref(p), A, count, rmin, rmax, noise, seed, _dptr(out)))
    return out


def bounds_status(solver) -> int:
    """1 if the bounds-check build saw an out-of-range index in this context, 0 if not; the
    normal build returns SMADFT_ERR_UNSUPPORTED (-6)."""
    bad = ctypes.c_int()
    rc = lib().smadft_bounds_status(solver._h, ctypes.byref(bad))
    return rc if rc else bad.value


def r2r3d_noalloc(src_ptr: int, dst_ptr: int, shape, kinds, precision: int = FP64, stream: int = 0) -> int:
    """smadft_r2r3d_noalloc on device pointers; returns the status code (0 = ok)."""
    nx, ny, nz = (int(s) for s in shape)
    return int(lib().smadft_r2r3d_noalloc(_vp(src_ptr), _vp(dst_ptr), nx, ny, nz,
                                          *[int(k) for k in kinds], int(precision), _vp(stream)))


class Solver:
    """One simulation context on one GPU (``smadft_ctx``)."""

    def __init__(self, p: Params):
        self.p = p
        self.shape = (p.nx, p.ny, p.nz)
        self.n = p.nx * p.ny * p.nz
        h = _vp()
        rc = lib().smadft_create(ctypes.byref(p), ctypes.byref(h))
        _check(rc)
        self._h = h

    def close(self):
        h = getattr(self, "_h", None)
        if h:
            lib().smadft_destroy(h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_psi(self, psi) -> None:
        a = np.ascontiguousarray(psi, dtype=np.float64)
        if a.size != self.n:
            raise ValueError("psi has the wrong size")
        _check(lib().smadft_set_psi(self._h, _dptr(a), a.size), self._h)

    def step(self, n: int = 1) -> None:
        _check(lib().smadft_step(self._h, int(n)), self._h)

    def step_diag(self) -> dict:
        d = Diag()
        rc = lib().smadft_step_diag(self._h, ctypes.byref(d))
        if rc not in (0, -4):
            _check(rc, self._h)
        out = d.as_dict()
        out["rc"] = rc
        return out

    def sync(self) -> None:
        _check(lib().smadft_sync(self._h), self._h)

    def get(self, field="psi") -> np.ndarray:
        out = np.empty(self.shape, dtype=np.float64)
        fid = FIELD[field] if isinstance(field, str) else int(field)
        _check(lib().smadft_get_field(self._h, fid, _dptr(out), out.size), self._h)
        return out

    def free_energy(self) -> float:
        e = ctypes.c_double()
        _check(lib().smadft_free_energy(self._h, ctypes.byref(e)), self._h)
        return e.value

    def track(self, axis=2, mode=TRACK_FLAT, hi=0.7, lo=0.0, field="psi"):
        dims = [s for a, s in enumerate(self.shape) if a != axis]
        idx = np.empty(dims, dtype=np.int32)
        pos = np.empty(dims, dtype=np.float64)
        _check(lib().smadft_track(self._h, FIELD[field], axis, mode, hi, lo,
                                  idx.ctypes.data_as(_P(ctypes.c_int)), _dptr(pos)), self._h)
        return idx, pos

    def step_surface(self):
        """One step with the interface diagnostics: per (i, j) column the interface index
        along z (-1: none), normal velocity, 2H and K (NaN: none), shaped (nx, ny)."""
        shp = (self.shape[0], self.shape[1])
        idx = np.empty(shp, dtype=np.int32)
        vel, h, k = (np.empty(shp) for _ in range(3))
        d = Diag()
        _check(lib().smadft_step_surface(self._h, idx.ctypes.data_as(_P(ctypes.c_int)), _dptr(vel), _dptr(h),
                                         _dptr(k), ctypes.byref(d)), self._h)
        self.last_diag = d.as_dict()
        return idx, vel, h, k

    def save(self, path: str) -> None:
        _check(lib().smadft_save_checkpoint(self._h, path.encode()), self._h)

    def load(self, path: str) -> None:
        _check(lib().smadft_load_checkpoint(self._h, path.encode()), self._h)

    def step_host(self, psi: np.ndarray, n: int = 1) -> None:
        """Per-step call with psi in host memory (in/out, float64, C-contiguous)."""
        if psi.dtype != np.float64 or not psi.flags.c_contiguous or psi.size != self.n:
            raise ValueError("psi must be a C-contiguous float64 array of the grid size")
        _check(lib().smadft_step_host(self._h, _dptr(psi), psi.size, int(n)), self._h)

    @property
    def stream(self) -> int:
        s = _vp()
        _check(lib().smadft_get_stream(self._h, ctypes.byref(s)), self._h)
        return s.value or 0

    @property
    def launches(self) -> int:
        c = ctypes.c_longlong()
        _check(lib().smadft_launch_count(self._h, ctypes.byref(c)), self._h)
        return c.value

    def r2r_pass_device(self, src_ptr: int, dst_ptr: int, axis: int, kind: int) -> None:
        _check(lib().smadft_r2r_pass_device(self._h, _vp(src_ptr), _vp(dst_ptr), int(axis), int(kind)),
               self._h)

    def adjoint(self, steps: int, checkpoint_every: int = 50, axis: int = 0, mode: int = TRACK_BUMP,
                hi: float = 0.6, lo: float = 0.1, want_dpsi0: bool = True) -> dict:
        """Interface-loss gradients of `steps` noadv or adv loop bodies from the initial
        condition (nu: adv only, 0 for noadv)."""
        o = AdjOpts(int(steps), int(checkpoint_every), int(axis), int(mode), float(hi), float(lo))
        g = Grads()
        dpsi = np.empty(self.shape, dtype=np.float64) if want_dpsi0 else None
        _check(lib().smadft_adjoint(self._h, ctypes.byref(o), ctypes.byref(g),
                                    _dptr(dpsi) if dpsi is not None else None), self._h)
        return dict(loss=g.loss, found=g.found, eps=g.d_eps, alpha=g.d_alpha, beta=g.d_beta, gamma=g.d_gamma,
                    nu=g.d_nu, psi0=dpsi)

    def autotune(self, steps: int = 5) -> dict:
        """Time each applicable kernel path on this run and keep the fastest (state kept)."""
        r = TuneReport()
        _check(lib().smadft_autotune(self._h, int(steps), ctypes.byref(r)), self._h)
        ms = {lib().smadft_tune_config_name(i).decode(): r.ms[i] for i in range(8) if r.ms[i] > 0}
        return {"chosen": lib().smadft_tune_config_name(r.chosen).decode(), "ms_per_step": ms}

    def r2r3d_device(self, src_ptr: int, dst_ptr: int, kinds) -> None:
        _check(lib().smadft_r2r3d_device(self._h, _vp(src_ptr), _vp(dst_ptr), *[int(k) for k in kinds]),
               self._h)


class _Member(Solver):
    """A batch member: a context owned by its batch (closing it is a no-op)."""

    def __init__(self, handle, p: Params):
        self.p = p
        self.shape = (p.nx, p.ny, p.nz)
        self.n = p.nx * p.ny * p.nz
        self._h = handle

    def close(self):
        self._h = None


class Batch:
    """Independent runs advanced together (``smadft_batch``): one CUDA graph per step for all."""

    def __init__(self, plist):
        arr = (Params * len(plist))(*plist)
        h = _vp()
        _check(lib().smadft_batch_create(arr, len(plist), ctypes.byref(h)))
        self._h = h
        self.members = []
        for i, p in enumerate(plist):
            m = _vp()
            _check(lib().smadft_batch_member(h, i, ctypes.byref(m)))
            self.members.append(_Member(m, p))

    def step(self, n: int = 1) -> None:
        rc = lib().smadft_batch_step(self._h, int(n))
        if rc:
            raise SmadftError(rc, lib().smadft_batch_last_error(self._h).decode())

    def sync(self) -> None:
        _check(lib().smadft_batch_sync(self._h))

    @property
    def stream(self) -> int:
        """The batch's cudaStream_t (every batch step is ordered on it)."""
        s = _vp()
        _check(lib().smadft_batch_get_stream(self._h, ctypes.byref(s)))
        return s.value or 0

    @property
    def groups(self) -> int:
        """Number of member groups stepped with pooled fields."""
        g = ctypes.c_int()
        _check(lib().smadft_batch_groups(self._h, ctypes.byref(g)))
        return g.value

    def close(self):
        h = getattr(self, "_h", None)
        if h:
            for m in self.members:
                m._h = None
            lib().smadft_batch_destroy(h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
