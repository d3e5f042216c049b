"""GPU parity of the inlet boundaries 401 (total temperature and pressure),
403 (total temperature and mass flux), 404 (static temperature and mass
flux) and the ambient far field 407 (Lib_BC_Fluxes_Inflow.f90,
Lib_BC_Fluxes_FarField.f90) against the CPU oracle, on the perturbed
curvilinear channels in 2-D and 3-D.  The formulas call pow, whose CUDA and
glibc results may differ in the last bit, so the bar is the normwise
relative L-infinity 1e-12 of the other pow-based boundary (406)."""
import numpy as np
import pytest

from mose_b200 import cases
from mose_b200.cases import GC

from tests.test_gpu_parity import compare_state, rel_linf, solver

pytestmark = pytest.mark.gpu

G = 1.4
M = 0.8
P_INF = 1.0 / G
T_INF = P_INF          # R = 1, rho = 1
T0 = T_INF * (1.0 + 0.5 * (G - 1.0) * M * M)
P0 = P_INF * (1.0 + 0.5 * (G - 1.0) * M * M) ** (G / (G - 1.0))
NORMAL = np.finfo(np.float64).max
OUT406 = (406, [P_INF, 1.0, 0.0, 0.0, 0.0, 0.0])


def _swap(case, inflow, outflow):
    rec, data = case.bc_rec, case.bc_data
    f1 = rec[:, 5] == 405
    f2 = rec[:, 5] == 406
    rec[f1, 5], data[f1] = inflow[0], inflow[1]
    rec[f2, 5], data[f2] = outflow[0], outflow[1]
    return case


def channel2d(inflow, outflow=OUT406):
    return _swap(cases.perturbed_channel(24, steps=1, amp=0.02, seed=3), inflow, outflow)


def channel3d(inflow, outflow=OUT406):
    case = cases.channel_3d(10, steps=1)
    rng = np.random.default_rng(7)
    p = case.prim[0]
    for v in (0, 1, 4):
        p[..., v] *= 1 + 0.02 * rng.standard_normal(p.shape[:-1])
    for v in (2, 3):
        p[..., v] = 0.02 * M * rng.standard_normal(p.shape[:-1])
    return _swap(case, inflow, outflow)


FAR = (407, [T0, P0, P_INF, 0.0, 0.0, 1.0])
CASES2D = {
    "401": lambda: channel2d((401, [T0, P0, 0.0, 0.0, 1.0, 0.0])),
    "401_normal_relaxed": lambda: channel2d((401, [T0, 1.3 * P0, NORMAL, NORMAL, 0.8, 0.0])),
    "401_angle": lambda: channel2d((401, [T0, P0, 0.15, 0.0, 1.0, 0.0])),
    "403": lambda: channel2d((403, [T0, 1.0 * M, 0.0, 0.0, 1.0, 0.0])),
    "404": lambda: channel2d((404, [T_INF, 1.0 * M, -0.1, NORMAL, 1.0, 0.0])),
    "407_both_ends": lambda: channel2d(FAR, FAR),
}
CASES3D = {
    "401": lambda: channel3d((401, [T0, P0, 0.05, -0.08, 1.0, 0.0])),
    "403": lambda: channel3d((403, [T0, 1.0 * M, NORMAL, NORMAL, 1.0, 0.0])),
    "404_407": lambda: channel3d((404, [T_INF, 1.0 * M, 0.0, 0.1, 1.0, 0.0]), (407, [T0, P0, P_INF, 0.0, 0.05, 1.0])),
}


def _residual_rel(s, o, nblk):
    worst = 0.0
    for b in range(1, nblk + 1):
        rg = s.download_residual(b)[GC:-GC, GC:-GC, GC:-GC]
        ro = o.get_residual(b)[GC:-GC, GC:-GC, GC:-GC]
        vars_ = [0, 1, 2, 4] if rg.shape[0] == 1 else [0, 1, 2, 3, 4]
        worst = max(worst, rel_linf(rg[..., vars_], ro[..., vars_]))
    return worst


@pytest.mark.parametrize("name", sorted(CASES2D))
def test_inlet2d_residual_and_steps(oracle_mod, name):
    case = CASES2D[name]()
    o = oracle_mod.Oracle(case)
    s = solver(case)
    o.fill_ghost_cell(); o.fluxes(); o.bc_fluxes()
    s.fill_ghost_cell(); s.fluxes_and_bc_fluxes()
    assert _residual_rel(s, o, 1) <= 1e-12
    s2 = solver(case)
    o = oracle_mod.Oracle(case)
    for _ in range(4):
        o.step()
        s2.explicit_step()
    compare_state(s2, o, 1, exact=False, tol=1e-12)
    for _ in range(6):
        o.step()
    s2.advance(6)
    compare_state(s2, o, 1, exact=False, tol=1e-12)


def _compare3d(s, o, tol=1e-12):
    g = s.download_prim(1)[GC:-GC, GC:-GC, GC:-GC]
    r = o.get_prim(1)[GC:-GC, GC:-GC, GC:-GC]
    assert rel_linf(g, r) <= tol, rel_linf(g, r)


@pytest.mark.parametrize("name", sorted(CASES3D))
def test_inlet3d_steps(oracle_mod, name):
    case = CASES3D[name]()
    o = oracle_mod.Oracle(case)
    s = solver(case)
    o.fill_ghost_cell(); o.fluxes(); o.bc_fluxes()
    s.fill_ghost_cell(); s.fluxes_and_bc_fluxes()
    assert _residual_rel(s, o, 1) <= 1e-12
    o = oracle_mod.Oracle(case)
    s = solver(case)
    for _ in range(3):
        o.step()
        s.explicit_step()
    _compare3d(s, o)
    for _ in range(3):
        o.step()
    s.advance(3)
    _compare3d(s, o)


@pytest.mark.parametrize("name", ["401_normal_relaxed", "403", "407_both_ends"])
def test_inlet2d_fast_precisions(oracle_mod, name):
    """The FP64 and mixed stage kernels reach the same boundary formulas: FP64
    within 1e-12 of the oracle after one step, mixed within a density L2 of
    1e-6 after five."""
    from mose_b200 import _lib
    case = CASES2D[name]()
    o = oracle_mod.Oracle(case)
    s = solver(case, precision=_lib.PRECISION_FP64)
    o.step()
    s.explicit_step()
    compare_state(s, o, 1, exact=False, tol=1e-12)
    o = oracle_mod.Oracle(case)
    s = solver(case, precision=_lib.PRECISION_MIXED)
    for _ in range(5):
        o.step()
        s.explicit_step()
    g = s.download_prim(1)[GC:-GC, GC:-GC, GC:-GC][..., 0]
    r = o.get_prim(1)[GC:-GC, GC:-GC, GC:-GC][..., 0]
    l2 = float(np.sqrt(((g - r) ** 2).sum() / (r ** 2).sum()))
    assert l2 < 1e-6, l2


def test_far_field_rejects_normal_token():
    """407 uses its angles as given, so the token 'normal' is refused at setup."""
    from mose_b200 import MoseError
    case = channel2d((407, [T0, P0, P_INF, NORMAL, 0.0, 1.0]))
    with pytest.raises(MoseError):
        solver(case)


RAMP = (np.array([0.0, 0.03, 0.07, 0.2]), np.array([0.97 * P0, 1.04 * P0, 1.01 * P0, 1.06 * P0]), False)
WAVE = (np.array([0.0, 0.02, 0.05]), np.array([P0, 1.08 * P0, P0]), True)


def channel402(table, rel_fac=1.0, alpha=0.0):
    case = channel2d((402, [T0, 0.0, alpha, 0.0, rel_fac, 0.0]))
    case.series = [table]
    return case


@pytest.mark.parametrize("name,table", [("ramp", RAMP), ("periodic", WAVE)])
def test_time_table_inlet_steps(oracle_mod, name, table):
    """402: p0 from its time table at the step's time (Mod_BC_Fluxes.f90:
    129-131, Series_Data_m.f90:55-86), through fused steps and
    graph-replayed steps; the periodic table wraps several times."""
    case = channel402(table, rel_fac=0.9 if name == "periodic" else 1.0, alpha=NORMAL if name == "ramp" else 0.0)
    o = oracle_mod.Oracle(case)
    s = solver(case)
    for _ in range(4):
        o.step()
        s.explicit_step()
    compare_state(s, o, 1, exact=False, tol=1e-12)
    for _ in range(8):
        o.step()
    s.advance(8)
    # the states differ by pow's last bits, so the CFL step may too
    assert abs(s.time - o.time) <= 1e-14 * o.time and o.time > 0.1
    compare_state(s, o, 1, exact=False, tol=1e-12)


def test_time_table_inlet_phase_path(oracle_mod):
    """The residual phase reads the table at the caller's domain time."""
    case = channel402(RAMP)
    o = oracle_mod.Oracle(case)
    s = solver(case)
    for t in (0.0, 0.05, 0.5):
        o.set_time(t)
        s.set_time(t)
        o.fill_ghost_cell(); o.fluxes(); o.bc_fluxes()
        s.fill_ghost_cell(); s.fluxes_and_bc_fluxes()
        assert _residual_rel(s, o, 1) <= 1e-12


def test_time_table_inlet_needs_its_table():
    from mose_b200 import MoseError
    case = channel402(RAMP)
    case.series = []
    with pytest.raises(MoseError):
        solver(case)
