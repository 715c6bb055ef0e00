"""The allocation-free assembly entry point, ceos_cnh_assemble_noalloc.

It exists for callers that cannot call cudaMalloc while they assemble (their GPU memory is
owned by their own allocator or pool): they pass only their own device buffers and the library
takes its assembly scratch from a static 8 MiB device array.  These tests drive it through the
C ABI and check:
- f_int and K against the regular entry point (ceos_evaluate on a CEOS_MIXED compressible
  Neo-Hookean handle) on the same inputs, for two calls in a row, so that whatever the first call
  leaves in the shared static scratch cannot leak into the second (bar 2e-5 relative to the
  largest entry, the mixed-precision bar of the other GPU tests);
- f_int and K against the FP64 oracle, on a general deformation (2e-5) and on the
  near-incompressible simple-shear patch whose interior forces cancel (5e-5 of the largest entry:
  the volumetric stress lambda ln J with lambda = 99 mu turns the FP32 rounding of F into about
  3e-5 of the small boundary forces; element-local differences formed in FP64 keep the rest of
  the element-scale precision);
- the status paths: a folded element returns 1 and the next clean call returns 0 (the flag word
  is cleared between calls); a node id outside the mesh, a CSR row that does not have the upper
  pattern's layout and a column array that lacks a neighbour each return CEOS_E_MESH without
  touching memory outside the buffers; sizes beyond the static scratch return CEOS_E_ARG.

Kept in its own file, collected last, so that a run stopping at the first failure has already
run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 2e-5
MU, LAMBDA = 1.0, 100.0 - 2.0 / 3.0
E_ARG, E_MESH = -1, -4


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


class _Device:
    """Caller-owned device copies of one mesh and its CSR pattern, and the output buffers."""

    def __init__(self, X, conn, rowmap, col):
        import torch
        dev = torch.device("cuda:0")
        self.n_nodes, self.n_elem, self.nnz = X.shape[0], conn.shape[0], col.size
        self.X = torch.tensor(X.reshape(-1), dtype=torch.float64, device=dev)
        self.conn = torch.tensor(np.asarray(conn).reshape(-1), dtype=torch.int32, device=dev)
        self.rowmap = torch.tensor(rowmap, dtype=torch.int32, device=dev)
        self.col = torch.tensor(col, dtype=torch.int32, device=dev)
        self.fint = torch.empty(3 * self.n_nodes, dtype=torch.float64, device=dev)
        self.K = torch.empty(self.nnz, dtype=torch.float64, device=dev)
        self.f = _entry()

    def call(self, U, conn=None, rowmap=None, col=None):
        import torch
        dU = torch.tensor(U, dtype=torch.float64, device="cuda:0")
        torch.cuda.synchronize()
        p = lambda t: C.c_void_p(t.data_ptr())
        rc = self.f(self.n_nodes, self.n_elem, p(self.X), p(dU), p(conn if conn is not None else self.conn),
                    p(rowmap if rowmap is not None else self.rowmap), p(col if col is not None else self.col),
                    self.nnz, MU, LAMBDA, p(self.fint), p(self.K), None)
        return rc, self.fint.cpu().numpy(), self.K.cpu().numpy()


def _setup(nx=10):
    import ceos_b200 as G
    from ceos_b200 import meshgen
    X, conn = meshgen.structured_box(nx, nx, nx, jitter=0.05, seed=0)
    g = G.ElementLoop(X, conn, G.CNH, [MU, LAMBDA], precision=G.MIXED)
    rowmap, col = g.pattern()
    return X, conn, g, _Device(X, conn, rowmap, col)


def test_noalloc_matches_regular_entry_point_twice():
    X, conn, g, d = _setup()
    rng = np.random.default_rng(7)
    for call in range(2):
        # a smooth stretch-and-shear field plus small noise (element size 0.1: no element folds)
        A = np.array([[0.2, 0.05, 0.0], [-0.03, -0.08, 0.02], [0.01, 0.04, 0.06]]) * (call + 1)
        U = (X @ A.T).reshape(-1) + 0.002 * rng.standard_normal(X.size)
        f_ref, K_ref, rc_ref, _ = g.evaluate(0.0, U)
        assert rc_ref == 0
        rc, f, K = d.call(U)
        assert rc == 0, rc
        assert _relerr(f, f_ref) <= TOL, call
        assert _relerr(K, K_ref) <= TOL, call
    g.close()


def test_noalloc_matches_fp64_oracle():
    import oracle as O
    X, conn, g, d = _setup()
    g.close()
    o = O.Model(X, conn, [O.CNH], [MU, LAMBDA])
    A = np.array([[0.15, 0.04, -0.02], [0.03, -0.06, 0.05], [-0.01, 0.02, 0.08]])
    U = (X @ A.T).reshape(-1) + 0.01 * np.sin(3 * X[:, [1, 2, 0]]).reshape(-1)
    f_o, K_o, rc_o, _ = o.evaluate(0.0, U)
    assert rc_o == 0
    rc, f, K = d.call(U)
    assert rc == 0
    assert _relerr(f, f_o) <= TOL
    assert _relerr(K, K_o) <= TOL


def test_noalloc_near_incompressible_shear_patch_vs_oracle():
    """K = 100 mu under simple shear 0.3 z on a jittered 16^3 mesh: the interior nodal forces cancel,
    so f_int is small against the element forces and its largest entries are the boundary forces."""
    import oracle as O
    X, conn, g, d = _setup(16)
    g.close()
    U = np.zeros_like(X)
    U[:, 0] = 0.3 * X[:, 2]
    U = U.reshape(-1)
    o = O.Model(X, conn, [O.CNH], [MU, LAMBDA])
    f_o, K_o, _, _ = o.evaluate(0.0, U)
    rc, f, K = d.call(U)
    assert rc == 0
    assert _relerr(f, f_o) <= 5e-5
    assert _relerr(K, K_o) <= 2e-6


def test_noalloc_status_paths_and_flag_reset():
    X, conn, g, d = _setup(6)
    U0 = np.zeros(X.size)
    interior = np.nonzero(np.all((X > 0.1) & (X < 0.9), axis=1))[0]
    U = U0.copy()
    U[3 * interior[0]] = 0.9                       # pushes one node through its elements
    rc, _, _ = d.call(U)
    assert rc == 1                                 # det J <= 1e-13 (ClassStatus error 1)
    rc, f, K = d.call(U0)
    assert rc == 0                                 # the flag word starts clear on every call
    f_ref, K_ref, _, _ = g.evaluate(0.0, U0)
    assert np.abs(f).max() <= 1e-12 and _relerr(K, K_ref) <= TOL

    import torch
    bad_conn = d.conn.clone()
    bad_conn[5] = d.n_nodes + 7                    # a node id outside the mesh
    assert d.call(U0, conn=bad_conn)[0] == E_MESH
    bad_row = d.rowmap.clone()
    bad_row[3 * 4] = 2 ** 30                       # row 12 (node 4) leaves [0, nnz)
    assert d.call(U0, rowmap=bad_row)[0] == E_MESH
    rowmap, col = g.pattern()
    col2 = col.copy()
    col2[rowmap[0] - 1 + 3] += 1                   # node 0 loses its first upper neighbour
    assert d.call(U0, col=torch.tensor(col2, dtype=torch.int32, device="cuda:0"))[0] == E_MESH
    rc, f, K = d.call(U0)
    assert rc == 0 and _relerr(K, K_ref) <= TOL    # and a clean call afterwards is unaffected
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
    assert rc == E_ARG
