"""Host-side mirror of MOSE's explicit-step driver over the C ABI.

`Solver` exposes the phases of Explicit_Step
(src/lib/numerics/time/explicit/Mod_Explicit.f90:40-113) under the reference's
names and argument meanings, with the state resident on the GPU:

  fill_ghost_cell()        Fill_Ghost_Cell      (numerics/space/Lib_Ghost.f90:11)
  fluxes_and_bc_fluxes()   Fluxes + BC_Fluxes   (numerics/fluxes/Mod_Fluxes.f90:10,
                                                  numerics/fluxes/bc/Mod_BC_Fluxes.f90:10)
  rk_newstate(irk)         RK_Newstate          (numerics/time/explicit/Lib_Newstate.f90:13)
  compute_dt(...)          Compute_dt           (numerics/time/Mod_dt.f90:10)
  set_global_dt(dt)        Set_Global_dt        (numerics/time/Mod_dt.f90:110)
  copy_state()             Copy_State           (Mod_Explicit.f90:149)
  explicit_step()          Explicit_Step, fused: one kernel per RK stage
  compute_residual()       Compute_Residual     (diagnostic/Mod_Diagnostic.f90:13)

Errors raise MoseError carrying the C-ABI status; device-detected failures
(non-physical interface state, NaN or p < 0) report the offending (b,i,j,k)
like the reference's `stop` messages.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .cases import Case, LIMITERS, RIEMANN, to_ref_layout

GC = 2


class MoseError(RuntimeError):
    def __init__(self, code: int, msg: str, where=None):
        super().__init__(f"[{code}] {msg}")
        self.code = code
        self.where = where


def _dp(a: np.ndarray):
    if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
        raise ValueError("arrays crossing the C ABI must be C-contiguous float64")
    return a.ctypes.data_as(C.POINTER(C.c_double))


def pack_metrics(vol, dl, M, faces) -> np.ndarray:
    """A block's Setup_Metrics output in the layout mose_gpu_add_block takes:
    vol, dl%c(3) and M%c(3,3) over the ghosted cells (each in its Fortran
    memory order: arrays shaped (nk+4, nj+4, ni+4[, ...]) C-contiguous), then
    for each direction d = 1..3 the faces dir(d)%f as (N(3), A) per face;
    faces = [(N_d, A_d)] with N_d shaped A_d.shape + (3,)."""
    parts = [np.ascontiguousarray(x, dtype=np.float64).ravel() for x in (vol, dl, M)]
    for N, A in faces:
        N = np.asarray(N, dtype=np.float64).reshape(-1, 3)
        A = np.asarray(A, dtype=np.float64).reshape(-1, 1)
        parts.append(np.concatenate([N, A], axis=1).ravel())
    return np.ascontiguousarray(np.concatenate(parts))


class Solver:
    """A GPU context holding one multi-block domain.  metrics: optional, per
    block a pack_metrics() array (or None) of precomputed metrics to use
    instead of the ones the device forms from the nodes."""

    def __init__(self, case: Case, precision: int = _lib.PRECISION_FP64_EXACT, device: int = 0,
                 upload: bool = True, metrics=None):
        self.lib = _lib.load()
        cfg = _lib.Config()
        self.lib.mose_gpu_default_config(C.byref(cfg))
        cfg.n_rk = case.n_rk
        cfg.cfl = case.cfl
        cfg.time_accurate = int(case.time_accurate)
        cfg.limiter = LIMITERS[case.limiter]
        cfg.riemann = RIEMANN[case.riemann]
        cfg.precision = precision
        cfg.gamma = case.gamma
        cfg.rgas = case.rgas
        cfg.ramp_iter = int(getattr(case, "ramp_iter", 0))
        cfg.integration = {"cons": 0, "prim": 1}[getattr(case, "integration", "cons")]
        cfg.device = device
        h = C.c_void_p()
        rc = self.lib.mose_gpu_create(C.byref(cfg), C.byref(h))
        if rc != 0:
            raise MoseError(rc, "mose_gpu_create failed (no sm_100 device, or unsupported configuration)")
        self.h = h
        self.case = case
        if getattr(case, "minf", 0.0):
            self._check(self.lib.mose_gpu_set_riemann_minf(self.h, float(case.minf)))
        if getattr(case, "sd_limiter", False):
            self._check(self.lib.mose_gpu_set_sd_limiter(self.h, 1))
        if getattr(case, "irs_beta", 0.0):
            self._check(self.lib.mose_gpu_set_irs_beta(self.h, float(case.irs_beta)))
        if getattr(case, "model", 0):
            self._check(self.lib.mose_gpu_set_viscous(self.h, int(case.model), float(case.mu), float(case.kappa),
                                                      float(case.vnn)))
        self.dims = []
        for b, nd in enumerate(case.nodes, start=1):
            nk, nj, ni = nd.shape[0] - 1, nd.shape[1] - 1, nd.shape[2] - 1
            self.dims.append((ni, nj, nk))
            mb = metrics[b - 1] if metrics is not None else None
            if mb is not None:
                mb = np.ascontiguousarray(mb, dtype=np.float64)
                NG = (ni + 4) * (nj + 4) * (nk + 4)
                want = 13 * NG + 4 * ((ni + 1) * nj * nk + ni * (nj + 1) * nk + ni * nj * (nk + 1))
                if mb.size != want:
                    raise ValueError(f"block {b}: precomputed metrics hold {mb.size} values, the layout {want}")
            self._check(self.lib.mose_gpu_add_block(self.h, b, ni, nj, nk, _dp(np.ascontiguousarray(nd)),
                                                    _dp(mb) if mb is not None else None))
        for t, v, periodic in getattr(case, "series", []):
            sid = C.c_int32()
            t = np.ascontiguousarray(t, dtype=np.float64)
            v = np.ascontiguousarray(v, dtype=np.float64)
            if t.shape != v.shape or t.ndim != 1:
                raise ValueError("a time table is two 1-D arrays of equal length")
            self._check(self.lib.mose_gpu_add_series(self.h, _dp(t), _dp(v), len(t), int(bool(periodic)),
                                                     C.byref(sid)))
        rec = np.ascontiguousarray(case.bc_rec, dtype=np.int32)
        data = np.ascontiguousarray(case.bc_data, dtype=np.float64)
        self._check(self.lib.mose_gpu_set_bcs(self.h, rec.ctypes.data_as(C.POINTER(C.c_int32)), _dp(data),
                                              len(rec)))
        self._check(self.lib.mose_gpu_setup(self.h))
        if upload:
            for b, p in enumerate(case.prim, start=1):
                self.upload_prim(b, to_ref_layout(p))

    def close(self):
        if getattr(self, "h", None):
            self.lib.mose_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc):
        if rc != 0:
            msg = self.lib.mose_gpu_last_error(self.h).decode()
            loc = [C.c_int32() for _ in range(4)]
            self.lib.mose_gpu_error_location(self.h, *(C.byref(x) for x in loc))
            raise MoseError(rc, msg, tuple(x.value for x in loc))

    def _shape(self, b):
        ni, nj, nk = self.dims[b - 1]
        return (nk + 2 * GC, nj + 2 * GC, ni + 2 * GC, 5)

    # ---- state transfer (reference layout) -----------------------------------
    def upload_prim(self, b: int, P: np.ndarray):
        P = np.ascontiguousarray(P, dtype=np.float64)
        if P.shape != self._shape(b):
            raise ValueError(f"block {b}: expected {self._shape(b)}, got {P.shape}")
        self._check(self.lib.mose_gpu_upload_prim(self.h, b, _dp(P)))

    def upload_prim_old(self, b: int, P: np.ndarray):
        P = np.ascontiguousarray(P, dtype=np.float64)
        self._check(self.lib.mose_gpu_upload_prim_old(self.h, b, _dp(P)))

    def download_prim(self, b: int, out: np.ndarray | None = None) -> np.ndarray:
        out = np.empty(self._shape(b)) if out is None else out
        self._check(self.lib.mose_gpu_download_prim(self.h, b, _dp(out)))
        return out

    # ---- discrete adjoint (2-D, HLLC) -------------------------------------------
    def set_inflow_mach(self, mach: float):
        """Mach number of every 405 supersonic-inflow face."""
        self._check(self.lib.mose_gpu_set_inflow_mach(self.h, float(mach)))

    def adjoint_forward(self, nsteps: int, interval: int, block: int = 1, face: int = 3) -> float:
        """nsteps fused steps with a checkpoint every `interval` steps; returns
        J = sum over the cells of face `face` of block `block` of p * A."""
        J = C.c_double()
        self._check(self.lib.mose_gpu_adjoint_forward(self.h, nsteps, interval, block, face, C.byref(J)))
        return J.value

    def adjoint_backward(self) -> float:
        """Reverse sweep of the last adjoint_forward: dJ/dP0 stays in the
        adjoint state (download_adjoint); returns dJ/dMach."""
        d = C.c_double()
        self._check(self.lib.mose_gpu_adjoint_backward(self.h, C.byref(d)))
        return d.value

    def adjoint_step(self) -> float:
        """lambda <- (dP^{n+1}/dP^n)^T lambda at the current state; returns
        lambda . dP^{n+1}/dMach."""
        d = C.c_double()
        self._check(self.lib.mose_gpu_adjoint_step(self.h, C.byref(d)))
        return d.value

    def upload_adjoint(self, b: int, lam: np.ndarray):
        lam = np.ascontiguousarray(lam, dtype=np.float64)
        if lam.shape != self._shape(b):
            raise ValueError(f"block {b}: expected {self._shape(b)}, got {lam.shape}")
        self._check(self.lib.mose_gpu_upload_adjoint(self.h, b, _dp(lam)))

    def download_adjoint(self, b: int) -> np.ndarray:
        out = np.empty(self._shape(b))
        self._check(self.lib.mose_gpu_download_adjoint(self.h, b, _dp(out)))
        return out

    def download_residual(self, b: int) -> np.ndarray:
        out = np.empty(self._shape(b))
        self._check(self.lib.mose_gpu_download_residual(self.h, b, _dp(out)))
        return out

    def upload_residual(self, b: int, R: np.ndarray):
        self._check(self.lib.mose_gpu_upload_residual(self.h, b, _dp(np.ascontiguousarray(R))))

    def download_dt(self, b: int) -> np.ndarray:
        ni, nj, nk = self.dims[b - 1]
        out = np.empty((nk, nj, ni))
        self._check(self.lib.mose_gpu_download_dt(self.h, b, _dp(out)))
        return out

    def upload_dt(self, b: int, dt: np.ndarray):
        self._check(self.lib.mose_gpu_upload_dt(self.h, b, _dp(np.ascontiguousarray(dt, dtype=np.float64))))

    # ---- phases of Explicit_Step ----------------------------------------------
    def compute_dt(self, cfl: float | None = None, iter: int = 0, ramp_iter: int = 0,
                   dtglobal: float = 1e5) -> float:
        v = C.c_double(dtglobal)
        self._check(self.lib.mose_gpu_compute_dt(self.h, self.case.cfl if cfl is None else cfl, iter, ramp_iter,
                                                 C.byref(v)))
        return v.value

    def set_global_dt(self, dtglobal: float):
        self._check(self.lib.mose_gpu_set_global_dt(self.h, dtglobal))

    def copy_state(self):
        self._check(self.lib.mose_gpu_copy_state(self.h))

    def fill_ghost_cell(self):
        self._check(self.lib.mose_gpu_fill_ghosts(self.h))

    def fluxes_and_bc_fluxes(self):
        self._check(self.lib.mose_gpu_residual(self.h))

    def rk_newstate(self, irk: int):
        self._check(self.lib.mose_gpu_rk_stage(self.h, irk))

    def synchronize(self):
        self._check(self.lib.mose_gpu_synchronize(self.h))

    def explicit_step(self):
        dt, t = C.c_double(), C.c_double()
        self._check(self.lib.mose_gpu_step(self.h, C.byref(dt), C.byref(t)))
        return dt.value, t.value

    def advance(self, nsteps: int):
        dt, t = C.c_double(), C.c_double()
        self._check(self.lib.mose_gpu_advance(self.h, nsteps, C.byref(dt), C.byref(t)))
        return dt.value, t.value

    def compute_residual(self) -> np.ndarray:
        out = np.zeros(5)
        self._check(self.lib.mose_gpu_residual_norms(self.h, _dp(out)))
        return out

    # ---- 2-D work-list tiling -----------------------------------------------
    TILING_KEYS = ("rows_per_item", "strip_width", "order", "ctas_per_sm")

    def tiling(self) -> dict:
        t = (C.c_int32 * 4)()
        self._check(self.lib.mose_gpu_get_tiling(self.h, t))
        return dict(zip(self.TILING_KEYS, list(t)))

    def set_tiling(self, rows_per_item=0, strip_width=62, order=0, ctas_per_sm=0):
        t = (C.c_int32 * 4)(rows_per_item, strip_width, order, ctas_per_sm)
        self._check(self.lib.mose_gpu_set_tiling(self.h, t))

    def autotune(self, steps: int = 3) -> dict:
        """Times candidate tilings of the 2-D work list on this domain and
        keeps the fastest; the state is unchanged.  Returns the tiling and
        the measured ms per step of it and of the default."""
        t = (C.c_int32 * 4)()
        best, default = C.c_double(), C.c_double()
        self._check(self.lib.mose_gpu_autotune(self.h, steps, t, C.byref(best), C.byref(default)))
        out = dict(zip(self.TILING_KEYS, list(t)))
        out.update(ms_per_step=best.value, default_ms_per_step=default.value)
        return out

    def set_time(self, time: float, it: int = 0):
        self._check(self.lib.mose_gpu_set_time(self.h, time, it))

    @property
    def time(self) -> float:
        t, it = C.c_double(), C.c_int32()
        self._check(self.lib.mose_gpu_get_time(self.h, C.byref(t), C.byref(it)))
        return t.value

    @property
    def uniform_metrics(self) -> bool:
        return bool(self.lib.mose_gpu_uniform_metrics(self.h))

    @property
    def launch_count(self) -> int:
        return int(self.lib.mose_gpu_launch_count(self.h))

    @property
    def stream_handle(self) -> int:
        """The context's cudaStream_t, e.g. for torch.cuda.ExternalStream."""
        return int(self.lib.mose_gpu_stream(self.h) or 0)

    def time_kernels(self, nsteps: int):
        """Device ms per kernel class (dt+bookkeeping, ghost fill, stage) and launch counts."""
        ms = np.zeros(3)
        n = (C.c_int32 * 3)()
        self._check(self.lib.mose_gpu_time_kernels(self.h, nsteps, _dp(ms), n))
        return ms, list(n)

    def download_metrics(self, b: int):
        ni, nj, nk = self.dims[b - 1]
        g = (nk + 4, nj + 4, ni + 4)
        vol = np.zeros(g)
        dl = np.zeros(g + (3,))
        self._check(self.lib.mose_gpu_download_metrics(self.h, b, _dp(vol), _dp(dl)))
        return vol, dl

    def download_faces(self, b: int, direction: int):
        ni, nj, nk = self.dims[b - 1]
        shape = {1: (nk, nj, ni + 1), 2: (nk, nj + 1, ni), 3: (nk + 1, nj, ni)}[direction]
        N = np.zeros(shape + (3,))
        A = np.zeros(shape)
        self._check(self.lib.mose_gpu_download_faces(self.h, b, direction, _dp(N), _dp(A)))
        return N, A

    # ---- reference-style driver ----------------------------------------------
    def run_phases(self):
        """One Explicit_Step through the separate phases (the drop-in path a
        Fortran driver with an External_Function hook takes)."""
        dt = self.compute_dt()
        if self.case.time_accurate:
            self.set_global_dt(dt)
        self.copy_state()
        for irk in range(1, self.case.n_rk + 1):
            self.fill_ghost_cell()
            self.fluxes_and_bc_fluxes()
            self.rk_newstate(irk)
        self.synchronize()
        return dt
