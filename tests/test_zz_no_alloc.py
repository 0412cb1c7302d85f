"""The allocation-free solve entry point (swc_solve_noalloc) against swc_solve.

Callers whose device memory belongs to a pool that forbids further CUDA allocations, or
whose host only lets them allocate at start-up, use swc_solve_noalloc: it runs the same
supernodal solve with its scratch in a fixed array of the library's device image.  This
test calls both entry points through the C ABI on the same factor and checks that the
allocation-free one gives the same solution, within the solve tests' tolerance (1e-12
relative), on two calls in a row (the second reuses the scratch the first left behind).
The file is collected last so that a run stopping at its first failure has run the rest."""
import ctypes

import numpy as np
import pytest

from conftest import load_sym
import swcholesky_b200 as swc
from swcholesky_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_solve_noalloc_matches_solve(cuda_ok):
    import torch
    gs = load_sym("grid3d_24")
    A, _, _ = W.build("grid3d_24")
    P = W.assemble(A, gs["perm"], gs["super"])
    L = swc.lib()
    nrhs = 2
    rng = np.random.default_rng(7)
    b = torch.from_numpy(rng.standard_normal((nrhs, P.n))).cuda()   # column-major (n, nrhs)
    # the allocation-free solve runs first on its handle (no swc_solve workspace exists)
    h = swc.Handle(0)
    h.analyze(P.n, P.A2p, P.A2i, P.lC, P.Ls, P.Li_ptr, P.super, P.prunePtr, P.pruneSet)
    assert h.factor(P.A2x) == 0
    xs = []
    free_after_first = None
    for call in range(2):
        x = torch.full_like(b, float("nan"))
        torch.cuda.synchronize()   # b and the NaN fill are on torch's stream, the solve on the handle's
        if call == 1:
            free_after_first = torch.cuda.mem_get_info()[0]
        rc = L.swc_solve_noalloc(h._h, ctypes.c_void_p(b.data_ptr()),
                                 ctypes.c_void_p(x.data_ptr()), nrhs)
        assert rc == swc.SWC_OK, L.swc_last_error().decode()
        torch.cuda.synchronize()
        if call == 1:
            # the second call allocated no device memory
            assert torch.cuda.mem_get_info()[0] == free_after_first
        xs.append(x.cpu().numpy())
    # the reference result: swc_solve on a second handle with the same factor
    h2 = swc.Handle(0)
    h2.analyze(P.n, P.A2p, P.A2i, P.lC, P.Ls, P.Li_ptr, P.super, P.prunePtr, P.pruneSet)
    assert h2.factor(P.A2x) == 0
    x_ref = torch.zeros_like(b)
    torch.cuda.synchronize()
    assert L.swc_solve(h2._h, ctypes.c_void_p(b.data_ptr()), ctypes.c_void_p(x_ref.data_ptr()),
                       nrhs, 1) == swc.SWC_OK
    torch.cuda.synchronize()
    ref = x_ref.cpu().numpy()
    for x in xs:
        assert np.isfinite(x).all()
        assert np.abs(x - ref).max() <= 1e-12 * np.abs(ref).max()


def test_solve_noalloc_rejects_oversized(cuda_ok):
    import torch
    gs = load_sym("grid3d_24")
    A, _, _ = W.build("grid3d_24")
    P = W.assemble(A, gs["perm"], gs["super"])
    h = swc.Handle(0)
    h.analyze(P.n, P.A2p, P.A2i, P.lC, P.Ls, P.Li_ptr, P.super, P.prunePtr, P.pruneSet)
    assert h.factor(P.A2x) == 0
    off_rows = int(P.Li_ptr[-1]) - P.n
    nrhs = 1048576 // off_rows + 1          # one right-hand side more than fits
    b = torch.zeros((nrhs, P.n), dtype=torch.float64, device="cuda")
    x = torch.zeros_like(b)
    L = swc.lib()
    rc = L.swc_solve_noalloc(h._h, ctypes.c_void_p(b.data_ptr()), ctypes.c_void_p(x.data_ptr()),
                             nrhs)
    assert rc == swc.SWC_INVALID_INPUT
    assert "scratch" in L.swc_last_error().decode()
