"""The restated FP64 reciprocal / reciprocal square root / square root used by
the "fp64" and "mixed" precisions: each result within one ulp (relative
error at most 2^-52) over 2^24 seeded inputs spread over 120 binades, measured
on the device through exact FMA residuals, and the restated square root at
most one ulp from the correctly rounded one."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_fast_reciprocals_within_one_ulp():
    from mose_b200 import _lib
    lib = _lib.load()
    out = np.zeros(4)
    rc = lib.mose_gpu_check_fast_math(1 << 24, 12345, out.ctypes.data_as(C.POINTER(C.c_double)))
    assert rc == 0
    rcp, rsq, sq, ulp_sqrt = out
    # units of 2^-53: 1.0 = half an ulp at the top of a binade, 2.0 = one ulp
    assert rcp <= 2.0, out
    assert rsq <= 2.0, out
    assert sq <= 2.0, out
    assert ulp_sqrt <= 1.0, out


def test_fp64_issue_ceilings():
    """The FP64 ceiling microbenchmark returns finite rates in a plausible
    range for one B200 (FMA tens of TFLOP/s; division and square root
    slower than FMA) and timed launches of a few milliseconds."""
    from mose_b200 import _lib
    lib = _lib.load_probe()
    out = np.zeros(6)
    assert lib.mose_probe_fp64_peak(0, out.ctypes.data_as(C.POINTER(C.c_double))) == 0
    fma_tf, div_g, sqrt_g = out[:3]
    assert np.all(np.isfinite(out)) and np.all(out > 0), out
    assert 5.0 < fma_tf < 200.0, out
    fma_g = fma_tf * 1e3 / 2.0           # FMAs per ns
    assert div_g < fma_g and sqrt_g < fma_g, out
    assert np.all(out[3:] < 1000.0), out
