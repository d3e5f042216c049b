"""GPU parity of implicit residual smoothing (irs-beta > 0: Lib_IRS.f90 and
the IRS branch of Newstate_Conservative, Lib_Newstate.f90:40-72) against
the CPU oracle, bit for bit in the exact precision: multi-block with
connections and extrapolation faces (local and global time stepping), a
periodic block (201, whose residual ghost takes the zero-gradient branch),
the 1-D tube (one direction), the phase-by-phase entry points, the
graph-replayed advance, and the reference's own Prandtl-Meyer inputs; 3-D
boxes (the k sweeps and k-face residual ghosts, walls, primitive
integration) bit for bit; the fp64 residual within 1e-12 in 2-D and 3-D."""
from pathlib import Path

import numpy as np
import pytest

from mose_b200 import cases
from mose_b200.cases import Case

from tests.test_gpu_parity import compare_state, solver

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"


def with_irs(case, beta=0.5, time_accurate=None):
    case.irs_beta = beta
    if time_accurate is not None:
        case.time_accurate = time_accurate
    return case


IRS_CASES = {
    "quadrant_steady": lambda: with_irs(cases.four_quadrant(seed=2, nbx=3, nby=2, nmin=20, nmax=60, steps=3,
                                                            riemann="HLLE", limiter="vanleer"), 0.5, False),
    "quadrant_unsteady": lambda: with_irs(cases.four_quadrant(seed=7, nbx=2, nby=2, nmin=17, nmax=40, steps=3), 0.8),
    "vortex_periodic": lambda: with_irs(cases.isentropic_vortex(40, steps=3), 0.5),
    "sod": lambda: with_irs(cases.sod(150), 0.5),
}


@pytest.mark.parametrize("name", sorted(IRS_CASES))
def test_irs_steps_bitwise(oracle_mod, name):
    case = IRS_CASES[name]()
    o = oracle_mod.Oracle(case)
    s = solver(case)
    for _ in range(2):
        dto, to = o.step()
        dtg, tg = s.explicit_step()
        assert dtg == dto and tg == to
    compare_state(s, o, len(case.nodes))
    for _ in range(3):
        o.step()
    s.advance(3)
    compare_state(s, o, len(case.nodes))


def test_irs_phase_path_bitwise(oracle_mod):
    case = IRS_CASES["quadrant_steady"]()
    o = oracle_mod.Oracle(case)
    s = solver(case)
    for _ in range(2):
        dto, _ = o.step()
        dtg = s.run_phases()
        assert dtg == dto
        compare_state(s, o, len(case.nodes))


def test_irs_changes_the_solution(oracle_mod):
    """The smoothing is active: the same step without it differs."""
    a = IRS_CASES["quadrant_steady"]()
    b = IRS_CASES["quadrant_steady"]()
    b.irs_beta = 0.0
    sa, sb = solver(a), solver(b)
    sa.explicit_step()
    sb.explicit_step()
    pa, pb = sa.download_prim(1), sb.download_prim(1)
    assert not np.array_equal(pa, pb)


def test_prandtl_meyer_reference_inputs_bitwise(oracle_mod):
    """The reference's Prandtl-Meyer case (its mesh, ic and bc files and
    input.ini numerics: HLLE, van Leer, CFL 1, local time stepping, IRS 0.5,
    inflow angles 'normal') for 60 iterations."""
    d = np.load(GOLDEN / "prandtl_meyer.npz")
    case = Case("prandtl_meyer", [d["nodes"]], d["bc_rec"], d["bc_data"], [d["prim"]], n_rk=int(d["n_rk"]),
                cfl=float(d["cfl"]), time_accurate=bool(d["time_accurate"]), limiter=str(d["limiter"]),
                riemann=str(d["riemann"]), gamma=float(d["gamma"]), rgas=float(d["rgas"]),
                irs_beta=float(d["irs_beta"]))
    o = oracle_mod.Oracle(case)
    s = solver(case)
    for _ in range(20):
        o.step()
        s.explicit_step()
    compare_state(s, o, 1)
    for _ in range(40):
        o.step()
    s.advance(40)
    compare_state(s, o, 1)
    assert np.isfinite(s.compute_residual()).all()


@pytest.mark.parametrize("name", ["quadrant_steady", "vortex_periodic"])
def test_irs_fp64_precision(oracle_mod, name):
    """IRS with the residual in the fp64 precision (the smoothing and the
    update keep the reference's arithmetic): the states stay within the
    normwise relative L-infinity bar of 1e-12 of the oracle over 3 steps."""
    from mose_b200 import _lib
    from tests.test_gpu_parity import _per_var_rel
    case = IRS_CASES[name]()
    o = oracle_mod.Oracle(case)
    s = solver(case, precision=_lib.PRECISION_FP64)
    for _ in range(3):
        o.step()
        s.explicit_step()
    assert _per_var_rel(s, o, len(case.nodes)) <= 1e-12


def _prim(case):
    case.integration = "prim"
    return case


V3 = (0, 1, 2, 3, 4)
IRS3D = {
    # the Jacobi sweeps along i, j and k (Residual_Smoothing_Blk :42-103), the
    # residual ghosts of the k faces, local time stepping
    "box3d_steady": lambda: with_irs(cases.periodic_box_3d(sizes=[[8, 6], [7, 9], [6, 5]], seed=2, steps=3), 0.5,
                                     False),
    # multi-tile blocks, slip walls on the y ends (their residual ghosts copy
    # the boundary cell), global dt
    "box3d_ywalls_unsteady": lambda: with_irs(cases.periodic_box_3d(sizes=[[40, 24], [20], [6, 5]], nb=(2, 1, 2),
                                                                    seed=4, steps=3, ywalls=True), 0.6),
    # Newstate_Primitive's IRS branch in 3-D
    "box3d_prim": lambda: with_irs(_prim(cases.periodic_box_3d(sizes=[[7], [6], [8]], nb=(1, 1, 1), seed=3,
                                                               steps=3)), 0.5),
}


@pytest.mark.parametrize("name", sorted(IRS3D))
def test_irs_3d_steps_bitwise(oracle_mod, name):
    case = IRS3D[name]()
    o = oracle_mod.Oracle(case)
    s = solver(case)
    for _ in range(2):
        dto, to = o.step()
        dtg, tg = s.explicit_step()
        assert dtg == dto and tg == to
    compare_state(s, o, len(case.nodes), vars_=V3)
    for _ in range(2):
        o.step()
    s.advance(2)
    compare_state(s, o, len(case.nodes), vars_=V3)


def test_irs_3d_changes_the_solution():
    a = IRS3D["box3d_steady"]()
    b = IRS3D["box3d_steady"]()
    b.irs_beta = 0.0
    sa, sb = solver(a), solver(b)
    sa.explicit_step()
    sb.explicit_step()
    assert not np.array_equal(sa.download_prim(1), sb.download_prim(1))


@pytest.mark.parametrize("name", ["box3d_steady", "box3d_ywalls_unsteady"])
def test_irs_3d_fp64_precision(oracle_mod, name):
    """3-D IRS with the residual in the fp64 precision: within the normwise
    bar of 1e-12 of the oracle over 3 steps."""
    from mose_b200 import _lib
    from tests.test_gpu_parity import _per_var_rel
    case = IRS3D[name]()
    o = oracle_mod.Oracle(case)
    s = solver(case, precision=_lib.PRECISION_FP64)
    for _ in range(3):
        o.step()
        s.explicit_step()
    assert _per_var_rel(s, o, len(case.nodes), vars_=V3) <= 1e-12
