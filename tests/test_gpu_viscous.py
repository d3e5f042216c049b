"""GPU parity of the Navier-Stokes path (model = 1, laminar) against the
oracle, through the C ABI: the diffusive fluxes of Lib_Diffusive.f90 between
the convective sweeps, the viscous boundary terms (BC_Connection_Visc,
BC_Symmetry_Visc, BC_Wall_Heat, BC_Wall_Temperature) after each record's
Euler flux, and the VNN time-step limit.  Reference-exact precision: bit
for bit."""
import numpy as np
import pytest

from mose_b200 import cases
from mose_b200.cases import GC

pytestmark = pytest.mark.gpu

CASES = {
    "one_block": lambda: cases.shear_layer(24, steps=3, seed=0),
    "blocks_2x2_warped": lambda: cases.shear_layer(12, nbx=2, nby=2, warp=0.06, steps=3, seed=1),
    "symmetry_top_hot_wall": lambda: cases.shear_layer(16, nbx=2, top="symmetry", tw=0.9, steps=3, seed=2),
    "minmod_ausm": lambda: cases.shear_layer(16, nby=2, limiter="minmod", riemann="AUSM+", warp=0.04, steps=3,
                                             seed=3),
}


def interior(P):
    return P[GC:-GC, GC:-GC, GC:-GC]


def solver(case, **kw):
    from mose_b200 import Solver
    return Solver(case, **kw)


def assert_state_equal(s, o, nb):
    for b in range(1, nb + 1):
        g = interior(s.download_prim(b))[..., [0, 1, 2, 4]]
        r = interior(o.get_prim(b))[..., [0, 1, 2, 4]]
        assert np.array_equal(g, r), f"block {b}: max |diff| {np.abs(g - r).max()}"


@pytest.mark.parametrize("name", sorted(CASES))
def test_viscous_residual_bitwise(oracle_mod, name):
    case = CASES[name]()
    o = oracle_mod.Oracle(case)
    s = solver(case)
    o.fill_ghost_cell()
    o.fluxes()
    o.bc_fluxes()
    s.fill_ghost_cell()
    s.fluxes_and_bc_fluxes()
    for b in range(1, len(case.nodes) + 1):
        rg = interior(s.download_residual(b))[..., [0, 1, 2, 4]]
        ro = interior(o.get_residual(b))[..., [0, 1, 2, 4]]
        assert np.array_equal(rg, ro), f"block {b}: max |diff| {np.abs(rg - ro).max()}"


@pytest.mark.parametrize("name", sorted(CASES))
def test_viscous_steps_bitwise(oracle_mod, name):
    """Fused steps (the VNN-limited dt pass, then per stage ghost fill,
    viscous residual and update), the graph-replayed advance and the phase
    path, each against the oracle."""
    case = CASES[name]()
    o = oracle_mod.Oracle(case)
    s = solver(case)
    for _ in range(2):
        dto, to = o.step()
        dtg, tg = s.explicit_step()
        assert dtg == dto and tg == to
    assert_state_equal(s, o, len(case.nodes))
    for _ in range(3):
        o.step()
    _, tg = s.advance(3)
    assert tg == o.time
    assert_state_equal(s, o, len(case.nodes))
    dto, _ = o.step()
    assert s.run_phases() == dto
    assert_state_equal(s, o, len(case.nodes))


def test_viscous_local_time_stepping(oracle_mod):
    case = cases.shear_layer(12, nbx=2, warp=0.05, steps=2, seed=4)
    case.time_accurate = False
    o = oracle_mod.Oracle(case)
    s = solver(case)
    for _ in range(2):
        o.step()
        s.explicit_step()
    assert_state_equal(s, o, 2)
    for b in (1, 2):
        assert np.array_equal(s.download_dt(b), o.get_dtlocal(b))


def test_viscous_setup_refuses_what_it_does_not_run():
    from mose_b200 import MoseError, _lib
    with pytest.raises(MoseError) as ei:
        solver(cases.shear_layer(8, steps=1), precision=_lib.PRECISION_FP64)
    assert ei.value.code == _lib.ERR_UNSUPPORTED
