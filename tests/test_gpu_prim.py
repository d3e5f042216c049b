"""GPU parity of integration-variables = prim (Newstate_Primitive,
Lib_Newstate.f90:168-317) against the CPU oracle: the reference-exact
precision bit for bit on multi-block 2-D, 1-D and 3-D cases, with implicit
residual smoothing, and through the phase entry points; the faster
precisions refuse it."""
import numpy as np
import pytest

from mose_b200 import cases

from tests.test_gpu_parity import compare_state, solver

pytestmark = pytest.mark.gpu


def _prim(case, **kw):
    case.integration = "prim"
    for k, v in kw.items():
        setattr(case, k, v)
    return case


CASES = {
    "quadrant": lambda: _prim(cases.four_quadrant(seed=3, nbx=3, nby=2, nmin=17, nmax=40, steps=3)),
    "sod": lambda: _prim(cases.sod(200)),
    "vortex_local_dt": lambda: _prim(cases.isentropic_vortex(40, steps=3), time_accurate=False),
    "quadrant_irs": lambda: _prim(cases.four_quadrant(seed=4, nbx=2, nby=2, nmin=17, nmax=30, steps=3,
                                                      riemann="HLLE"), irs_beta=0.5, time_accurate=False),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_primitive_steps_bitwise(oracle_mod, name):
    case = CASES[name]()
    o = oracle_mod.Oracle(case)
    s = solver(case)
    for _ in range(2):
        o.step()
        s.explicit_step()
    compare_state(s, o, len(case.nodes))
    for _ in range(3):
        o.step()
    s.advance(3)
    compare_state(s, o, len(case.nodes))


@pytest.mark.parametrize("name", ["quadrant", "quadrant_irs"])
def test_primitive_phase_path_bitwise(oracle_mod, name):
    case = CASES[name]()
    o = oracle_mod.Oracle(case)
    s = solver(case)
    for _ in range(2):
        dto, _ = o.step()
        dtg = s.run_phases()
        assert dtg == dto
        compare_state(s, o, len(case.nodes))


def test_primitive_3d_bitwise(oracle_mod):
    case = _prim(cases.periodic_box_3d(16, nb=(2, 1, 1), steps=2, seed=1))
    o = oracle_mod.Oracle(case)
    s = solver(case)
    for _ in range(2):
        o.step()
        s.explicit_step()
    for b in range(1, len(case.nodes) + 1):
        g = s.download_prim(b)[2:-2, 2:-2, 2:-2]
        r = o.get_prim(b)[2:-2, 2:-2, 2:-2]
        assert np.array_equal(g, r), np.abs(g - r).max()


def test_primitive_needs_the_exact_precision():
    from mose_b200 import MoseError, _lib
    with pytest.raises(MoseError):
        solver(CASES["sod"](), precision=_lib.PRECISION_FP64)
