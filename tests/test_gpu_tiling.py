"""The 2-D work-list tiling and its autotuner: every tiling gives the same
bits (each face flux and cell update is the same arithmetic whichever CTA
does it), the autotuner leaves the state as it found it and never keeps a
tiling slower than the default, and bad tilings are refused."""
import numpy as np
import pytest

from mose_b200 import cases

from tests.test_gpu_parity import compare_state, interior, solver

pytestmark = pytest.mark.gpu

TILINGS = [dict(), dict(rows_per_item=16, strip_width=30, order=1, ctas_per_sm=1),
           dict(rows_per_item=512, strip_width=46, order=0, ctas_per_sm=2), dict(rows_per_item=24, order=1)]


def quadrant():
    return cases.four_quadrant(seed=7, nbx=3, nby=2, nmin=20, nmax=90, steps=3)


@pytest.mark.parametrize("k", range(len(TILINGS)))
def test_tiling_keeps_parity(oracle_mod, k):
    case = quadrant()
    o = oracle_mod.Oracle(case)
    s = solver(case)
    s.set_tiling(**TILINGS[k])
    got = s.tiling()
    for key, v in TILINGS[k].items():
        assert got[key] == v
    for _ in range(2):
        o.step()
        s.explicit_step()
    compare_state(s, o, len(case.nodes))
    for _ in range(3):
        o.step()
    s.advance(3)
    compare_state(s, o, len(case.nodes))


def test_fp64_results_do_not_depend_on_tiling():
    from mose_b200 import _lib
    out = []
    for t in TILINGS:
        case = cases.isentropic_vortex(96, steps=3)
        s = solver(case, precision=_lib.PRECISION_FP64)
        s.set_tiling(**t)
        s.advance(4)
        out.append(interior(s.download_prim(1)).copy())
    for P in out[1:]:
        assert np.array_equal(P, out[0])


def test_autotune_restores_state_and_keeps_parity(oracle_mod):
    case = quadrant()
    o = oracle_mod.Oracle(case)
    s = solver(case)
    before = [interior(s.download_prim(b)).copy() for b in range(1, len(case.nodes) + 1)]
    res = s.autotune(steps=2)
    assert res["ms_per_step"] <= res["default_ms_per_step"]
    assert res["ms_per_step"] > 0.0 and s.tiling() == {k: res[k] for k in s.TILING_KEYS}
    for b, P in enumerate(before, start=1):
        assert np.array_equal(interior(s.download_prim(b)), P)
    assert s.time == 0.0
    for _ in range(3):
        o.step()
        s.explicit_step()
    compare_state(s, o, len(case.nodes))


def test_bad_tiling_is_refused():
    from mose_b200 import MoseError
    s = solver(quadrant())
    for bad in (dict(strip_width=70), dict(strip_width=4), dict(order=2), dict(rows_per_item=-1)):
        with pytest.raises(MoseError):
            s.set_tiling(**bad)
    s3 = solver(cases.periodic_box_3d(sizes=[[6], [6], [6]], nb=(1, 1, 1), steps=1))
    with pytest.raises(MoseError):
        s3.autotune()
