"""ctypes wrapper of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the mose_b200 package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
GC = 2


class orc_config(C.Structure):
    _fields_ = [("n_rk", C.c_int32), ("cfl", C.c_double), ("time_accurate", C.c_int32),
                ("limiter", C.c_int32), ("riemann", C.c_int32), ("integration", C.c_int32),
                ("ndir", C.c_int32), ("gamma", C.c_double), ("rgas", C.c_double),
                ("ramp_iter", C.c_int32), ("res_diter", C.c_int32), ("minf", C.c_double),
                ("irs_beta", C.c_double), ("sd_limiter", C.c_int32), ("model", C.c_int32), ("mu", C.c_double),
                ("kappa", C.c_double), ("vnn", C.c_double)]


_LIBS: dict = {}


def build() -> None:
    """Compiles the oracle libraries with the Makefile beside this file."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def build_native(dest: str | os.PathLike) -> dict:
    """Builds the host-tuned timing builds (-march=native, IEEE and
    -ffast-math) into dest on the machine that runs them; returns their paths."""
    subprocess.run(["make", "-s", "-C", str(HERE), "native", f"NATIVE_DIR={dest}"], check=True)
    return {"native": Path(dest) / "liboracle_native.so", "fastmath": Path(dest) / "liboracle_fastmath.so"}


def load(omp: bool = False, path: str | os.PathLike | None = None) -> C.CDLL:
    name = str(path) if path is not None else ("liboracle_omp.so" if omp else "liboracle.so")
    if name in _LIBS:
        return _LIBS[name]
    path = Path(path) if path is not None else HERE / name
    if not path.exists():
        build()
    lib = C.CDLL(str(path))
    D = C.c_void_p
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int32)
    lib.orc_create.restype = D
    lib.orc_create.argtypes = [C.POINTER(orc_config), C.c_int]
    lib.orc_destroy.argtypes = [D]
    lib.orc_add_block.argtypes = [D, C.c_int, C.c_int, C.c_int, dp]
    lib.orc_set_bcs.argtypes = [D, ip, dp, C.c_int]
    lib.orc_setup_metrics.argtypes = [D]
    for f in ("orc_set_prim", "orc_set_prim_old", "orc_set_dtlocal"):
        getattr(lib, f).argtypes = [D, C.c_int, dp]
    for f in ("orc_get_prim", "orc_get_residual", "orc_get_dtlocal"):
        getattr(lib, f).argtypes = [D, C.c_int, dp]
    lib.orc_get_metrics.argtypes = [D, C.c_int, dp, dp, dp]
    lib.orc_get_faces.argtypes = [D, C.c_int, C.c_int, dp, dp]
    lib.orc_set_metrics.argtypes = [D, C.c_int, dp, dp, dp]
    lib.orc_set_faces.argtypes = [D, C.c_int, C.c_int, dp, dp]
    for f in ("orc_fill_ghost_cell", "orc_fluxes", "orc_bc_fluxes", "orc_copy_state", "orc_set_global_dt"):
        getattr(lib, f).argtypes = [D]
    lib.orc_rk_newstate.argtypes = [D, C.c_int]
    lib.orc_compute_dt.argtypes = [D, dp]
    lib.orc_explicit_step.argtypes = [D, dp, dp]
    lib.orc_compute_residual.argtypes = [D, dp]
    lib.orc_set_time.argtypes = [D, C.c_double, C.c_int]
    lib.orc_set_dtglobal.argtypes = [D, C.c_double]
    lib.orc_get_time.argtypes = [D]
    lib.orc_get_time.restype = C.c_double
    lib.orc_last_error.argtypes = [D, ip, ip, ip, ip]
    lib.orc_limiter.argtypes = [C.c_int, C.c_double, C.c_double]
    lib.orc_limiter.restype = C.c_double
    lib.orc_riemann.argtypes = [D, dp, dp, dp, dp]
    lib.orc_add_series.argtypes = [D, dp, dp, C.c_int, C.c_int]
    lib.orc_series_eval.argtypes = [D, C.c_int, C.c_double]
    lib.orc_series_eval.restype = C.c_double
    _LIBS[name] = lib
    return lib


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_double))


LIMITERS = {"first-order": 0, "none": 0, "minmod": 1, "vanleer": 2, "vanalbada": 3, "mc": 4, "superbee": 5}
RIEMANN = {"HLLC": 0, "AUSM+": 1, "SLAU": 2, "SLAU2": 3, "HLLE": 4, "HLLEM": 5, "LLF": 6, "Rusanov": 6,
           "PLLF": 7, "Hanel": 8, "AUSM+-up": 9, "AUSM+-up2": 10, "HLLC+": 11, "HLLE++": 12,
           "HLLC Rotated": 13, "exact": 14, "Exact": 14}


class Oracle:
    """One oracle domain built from a mose_b200.cases.Case (or the same fields)."""

    def __init__(self, case, nthreads: int = 1, omp: bool = False, ndir: int = 0, lib_path=None):
        self.lib = load(omp, lib_path)
        cfg = orc_config(n_rk=case.n_rk, cfl=case.cfl, time_accurate=int(case.time_accurate),
                         limiter=LIMITERS[case.limiter], riemann=RIEMANN[case.riemann],
                         integration={"cons": 0, "prim": 1}[getattr(case, "integration", "cons")],
                         ndir=ndir, gamma=case.gamma, rgas=case.rgas, ramp_iter=int(getattr(case, "ramp_iter", 0)),
                         res_diter=1,
                         minf=getattr(case, "minf", 0.0), irs_beta=getattr(case, "irs_beta", 0.0),
                         sd_limiter=int(getattr(case, "sd_limiter", False)), model=int(getattr(case, "model", 0)),
                         mu=float(getattr(case, "mu", 0.0)), kappa=float(getattr(case, "kappa", 0.0)),
                         vnn=float(getattr(case, "vnn", 0.5)))
        self.h = self.lib.orc_create(C.byref(cfg), nthreads)
        self.dims = []
        for nd in case.nodes:
            nk, nj, ni = nd.shape[0] - 1, nd.shape[1] - 1, nd.shape[2] - 1
            self.dims.append((ni, nj, nk))
            arr = np.ascontiguousarray(nd, dtype=np.float64)
            self._check(self.lib.orc_add_block(self.h, ni, nj, nk, _dp(arr)), "add_block")
        for t, v, periodic in getattr(case, "series", []):
            t = np.ascontiguousarray(t, dtype=np.float64)
            v = np.ascontiguousarray(v, dtype=np.float64)
            sid = self.lib.orc_add_series(self.h, _dp(t), _dp(v), len(t), int(periodic))
            if sid < 0:
                raise RuntimeError("oracle add_series failed")
        rec = np.ascontiguousarray(case.bc_rec, dtype=np.int32)
        data = np.ascontiguousarray(case.bc_data, dtype=np.float64)
        self._check(self.lib.orc_set_bcs(self.h, rec.ctypes.data_as(C.POINTER(C.c_int32)), _dp(data),
                                         len(rec)), "set_bcs")
        self._check(self.lib.orc_setup_metrics(self.h), "setup_metrics")
        from mose_b200.cases import to_ref_layout
        for b, p in enumerate(case.prim, start=1):
            self.set_prim(b, to_ref_layout(p))

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    @staticmethod
    def _check(rc, what):
        if rc != 0:
            raise RuntimeError(f"oracle {what} failed with code {rc}")

    def _shape(self, b):
        ni, nj, nk = self.dims[b - 1]
        return (nk + 2 * GC, nj + 2 * GC, ni + 2 * GC, 5)

    def series_eval(self, sid, time):
        return self.lib.orc_series_eval(self.h, sid, time)

    def set_prim(self, b, P):
        P = np.ascontiguousarray(P, dtype=np.float64)
        assert P.shape == self._shape(b)
        self._check(self.lib.orc_set_prim(self.h, b, _dp(P)), "set_prim")

    def set_prim_old(self, b, P):
        P = np.ascontiguousarray(P, dtype=np.float64)
        self._check(self.lib.orc_set_prim_old(self.h, b, _dp(P)), "set_prim_old")

    def get_prim(self, b):
        out = np.empty(self._shape(b))
        self._check(self.lib.orc_get_prim(self.h, b, _dp(out)), "get_prim")
        return out

    def get_residual(self, b):
        out = np.empty(self._shape(b))
        self._check(self.lib.orc_get_residual(self.h, b, _dp(out)), "get_residual")
        return out

    def get_dtlocal(self, b):
        ni, nj, nk = self.dims[b - 1]
        out = np.empty((nk, nj, ni))
        self._check(self.lib.orc_get_dtlocal(self.h, b, _dp(out)), "get_dtlocal")
        return out

    def set_dtlocal(self, b, dt):
        dt = np.ascontiguousarray(dt, dtype=np.float64)
        self._check(self.lib.orc_set_dtlocal(self.h, b, _dp(dt)), "set_dtlocal")

    def get_metrics(self, b):
        ni, nj, nk = self.dims[b - 1]
        g = (nk + 4, nj + 4, ni + 4)
        vol = np.empty(g)
        dl = np.empty(g + (3,))
        M = np.empty(g + (3, 3))
        self._check(self.lib.orc_get_metrics(self.h, b, _dp(vol), _dp(dl), _dp(M)), "get_metrics")
        return vol, dl, M

    def get_faces(self, b, direction):
        ni, nj, nk = self.dims[b - 1]
        shape = {1: (nk, nj, ni + 1), 2: (nk, nj + 1, ni), 3: (nk + 1, nj, ni)}[direction]
        N = np.empty(shape + (3,))
        A = np.empty(shape)
        self._check(self.lib.orc_get_faces(self.h, b, direction, _dp(N), _dp(A)), "get_faces")
        return N, A

    def set_metrics(self, b, vol, dl, M):
        ni, nj, nk = self.dims[b - 1]
        g = (nk + 4, nj + 4, ni + 4)
        arrs = [np.ascontiguousarray(x, dtype=np.float64) for x in (vol, dl, M)]
        assert arrs[0].shape == g and arrs[1].shape == g + (3,) and arrs[2].shape == g + (3, 3)
        self._check(self.lib.orc_set_metrics(self.h, b, *(_dp(x) for x in arrs)), "set_metrics")

    def set_faces(self, b, direction, N, A):
        N = np.ascontiguousarray(N, dtype=np.float64)
        A = np.ascontiguousarray(A, dtype=np.float64)
        assert N.shape == A.shape + (3,)
        self._check(self.lib.orc_set_faces(self.h, b, direction, _dp(N), _dp(A)), "set_faces")

    # phases of Explicit_Step
    def fill_ghost_cell(self):
        self.lib.orc_fill_ghost_cell(self.h)

    def fluxes(self):
        return self.lib.orc_fluxes(self.h)

    def bc_fluxes(self):
        return self.lib.orc_bc_fluxes(self.h)

    def rk_newstate(self, irk):
        return self.lib.orc_rk_newstate(self.h, irk)

    def copy_state(self):
        self.lib.orc_copy_state(self.h)

    def compute_dt(self, dtglobal_start=1e5):
        """Compute_dt with the minimum started from dtglobal_start (the
        explicit step passes 1d5, Mod_Explicit.f90:44)."""
        out = C.c_double(0.0)
        self.lib.orc_set_dtglobal(self.h, dtglobal_start)
        self.lib.orc_compute_dt(self.h, C.byref(out))
        return out.value

    def set_global_dt(self, dtglobal=None):
        if dtglobal is not None:
            self.lib.orc_set_dtglobal(self.h, dtglobal)
        self.lib.orc_set_global_dt(self.h)

    def step(self):
        dt, t = C.c_double(0.0), C.c_double(0.0)
        rc = self.lib.orc_explicit_step(self.h, C.byref(dt), C.byref(t))
        if rc != 0:
            raise RuntimeError(f"oracle step failed: {rc} at {self.last_error()}")
        return dt.value, t.value

    def residual_norms(self):
        out = np.zeros(5)
        self.lib.orc_compute_residual(self.h, _dp(out))
        return out

    def last_error(self):
        b, i, j, k = (C.c_int32() for _ in range(4))
        code = self.lib.orc_last_error(self.h, C.byref(b), C.byref(i), C.byref(j), C.byref(k))
        return code, (b.value, i.value, j.value, k.value)

    @property
    def time(self):
        return self.lib.orc_get_time(self.h)

    def set_time(self, time, it=0):
        self.lib.orc_set_time(self.h, time, it)
