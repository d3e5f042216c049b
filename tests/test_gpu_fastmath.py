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
