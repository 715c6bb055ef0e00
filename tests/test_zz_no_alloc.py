"""The allocation-free assembly entry point, ceos_cnh_assemble_noalloc.

It exists for callers that cannot call cudaMalloc while they assemble (their GPU memory is
owned by their own allocator or pool): they pass only their own device buffers and the library
takes its assembly scratch from a static 8 MiB device array.  This test drives it through the
C ABI and checks f_int and K against the regular entry point (ceos_evaluate on a CEOS_MIXED
compressible Neo-Hookean handle) on the same inputs, for two calls in a row so that whatever the
first call leaves in the shared static scratch cannot leak into the second.  Tolerance: the
mixed-precision bar of the other GPU tests, 2e-5 relative to the largest entry.

Kept in its own file, collected last, so that a run stopping at the first failure has already
run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 2e-5
MU, LAMBDA = 1.0, 100.0 - 2.0 / 3.0


def _entry():
    import ceos_b200 as G
    L = G.lib()
    f = L.ceos_cnh_assemble_noalloc
    P = C.c_void_p
    f.argtypes = [C.c_int, C.c_int, P, P, P, P, P, C.c_longlong, C.c_double, C.c_double, P, P, P]
    f.restype = C.c_int
    return f


def _relerr(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def test_noalloc_matches_regular_entry_point_twice():
    import torch
    import ceos_b200 as G
    from ceos_b200 import meshgen

    X, conn = meshgen.structured_box(10, 10, 10, jitter=0.05, seed=0)
    g = G.ElementLoop(X, conn, G.CNH, [MU, LAMBDA], precision=G.MIXED)
    rowmap, col = g.pattern()
    dev = torch.device("cuda:0")
    dX = torch.tensor(X.reshape(-1), dtype=torch.float64, device=dev)
    dconn = torch.tensor(conn.reshape(-1), dtype=torch.int32, device=dev)
    drow = torch.tensor(rowmap, dtype=torch.int32, device=dev)
    dcol = torch.tensor(col, dtype=torch.int32, device=dev)
    dfint = torch.empty(g.n_dof, dtype=torch.float64, device=dev)
    dK = torch.empty(g.nnz, dtype=torch.float64, device=dev)
    f = _entry()
    rng = np.random.default_rng(7)
    for call in range(2):
        # a smooth stretch-and-shear field plus small noise (element size 0.1: no element folds)
        A = np.array([[0.2, 0.05, 0.0], [-0.03, -0.08, 0.02], [0.01, 0.04, 0.06]]) * (call + 1)
        U = (X @ A.T).reshape(-1) + 0.002 * rng.standard_normal(X.size)
        f_ref, K_ref, rc_ref, _ = g.evaluate(0.0, U)
        assert rc_ref == 0
        dU = torch.tensor(U, dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        rc = f(g.n_nodes, g.n_elem, C.c_void_p(dX.data_ptr()), C.c_void_p(dU.data_ptr()),
               C.c_void_p(dconn.data_ptr()), C.c_void_p(drow.data_ptr()), C.c_void_p(dcol.data_ptr()), g.nnz,
               MU, LAMBDA, C.c_void_p(dfint.data_ptr()), C.c_void_p(dK.data_ptr()), None)
        assert rc == 0, rc
        assert _relerr(dfint.cpu().numpy(), f_ref) <= TOL, call
        assert _relerr(dK.cpu().numpy(), K_ref) <= TOL, call
    g.close()


def test_noalloc_rejects_meshes_beyond_the_static_scratch():
    """n_nodes + (nnz - 6 n_nodes)/9 node-pair blocks must fit 8 MiB / 48 B = 174,762."""
    import torch
    f = _entry()
    dummy = torch.zeros(16, dtype=torch.float64, device="cuda:0")
    p = C.c_void_p(dummy.data_ptr())
    n_nodes = 20000
    nnz = 6 * n_nodes + 9 * 13 * n_nodes  # 14 blocks per node: 280,000 > 174,762
    rc = f(n_nodes, 1, p, p, p, p, p, nnz, MU, LAMBDA, p, p, None)
    assert rc == -1
