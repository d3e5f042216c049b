"""The allocation-free residual-norm entry point.

mose_gpu_residual_norms_noalloc serves callers that keep P and PO in their
own device arrays and cannot let the library allocate device memory (their
memory belongs to another allocator or to a budget fixed at start-up).  It is
checked here, through the C ABI, against the context's own
mose_gpu_residual_norms on the same state, on two calls in a row.  This file
sorts last so that a run stopping at its first failure has run everything
else first."""
import ctypes as C

import numpy as np
import pytest

from mose_b200 import cases

pytestmark = pytest.mark.gpu


def _run(case):
    import torch

    from mose_b200 import Solver, _lib
    lib = _lib.load()
    s = Solver(case)
    nb = len(case.nodes)
    before = [np.ascontiguousarray(s.download_prim(b)) for b in range(1, nb + 1)]
    s.explicit_step()
    after = [np.ascontiguousarray(s.download_prim(b)) for b in range(1, nb + 1)]
    expect = s.compute_residual()            # the existing entry point: sums over blocks
    assert np.all(expect[[0, 1, 2, 4]] > 0)
    if all(d[2] == 1 for d in s.dims):
        assert expect[3] == 0.0              # 2-D: w is identically zero
    else:
        assert expect[3] > 0.0               # 3-D: the w sums and the k-plane offsets are exercised
    dev = torch.device("cuda", 0)
    P = [torch.from_numpy(a).to(dev) for a in after]
    PO = [torch.from_numpy(a).to(dev) for a in before]
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    results = []
    for _ in range(2):                       # two calls in a row share the scratch array
        total = torch.zeros(5, dtype=torch.float64, device=dev)
        for b in range(nb):
            ni, nj, nk = s.dims[b]
            rc = lib.mose_gpu_residual_norms_noalloc(C.c_void_p(P[b].data_ptr()), C.c_void_p(PO[b].data_ptr()),
                                                     ni, nj, nk, C.c_void_p(total.data_ptr()), stream)
            assert rc == 0, lib.mose_gpu_noalloc_last_error().decode()
        torch.cuda.synchronize(dev)
        results.append(total.cpu().numpy())
    for got in results:
        # the sums run in a different order than the context's reduction
        np.testing.assert_allclose(got, expect, rtol=1e-12, atol=0)
    s.close()


def test_noalloc_norms_single_block():
    _run(cases.isentropic_vortex(64, steps=1))


def test_noalloc_norms_multi_block_accumulates():
    _run(cases.four_quadrant(seed=4, nbx=2, nby=2, nmin=20, nmax=60, steps=1))


def test_noalloc_norms_3d_blocks():
    # two 3-D blocks: the arrays carry k ghost planes (offsets over nk > 1)
    _run(cases.periodic_box_3d(12, nb=(2, 1, 1), sizes=[[12, 8], [10], [6]], steps=1, seed=1))


def test_noalloc_rejects_blocks_beyond_the_limit():
    import torch

    from mose_b200 import _lib
    lib = _lib.load()
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = C.c_void_p(buf.data_ptr())
    # the size check happens before any launch: the arrays are never touched
    rc = lib.mose_gpu_residual_norms_noalloc(p, p, 4096 * 65536 + 1, 1, 1, p, None)
    assert rc == _lib.ERR_INVALID
    assert b"exceeds the no-allocation limit" in lib.mose_gpu_noalloc_last_error()
