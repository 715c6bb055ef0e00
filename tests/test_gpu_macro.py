"""Device pieces of the macro FE^2 path on the GPU: the external-material element loop against the
built-in compressible Neo-Hookean loop, the device Dirichlet PCG against a host residual, and a
macro element whose Gauss points are solved by batched RVEs against the FP64 RVE oracle."""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp
import torch

import fe2_oracle as F2
import oracle as O
from ceos_b200 import CNH, FP64, ElementLoop, meshgen
from ceos_b200 import macro as M

pytestmark = pytest.mark.gpu


def _cnh_setup(nx=3):
    X, conn = meshgen.structured_box(nx, nx, nx, jitter=0.05, seed=2)
    rng = np.random.default_rng(1)
    U = 0.02 * X @ rng.uniform(-1, 1, (3, 3)).T + 0.002 * rng.uniform(-1, 1, X.shape)
    return X, conn, U.reshape(-1)


def test_external_material_reproduces_builtin_cnh():
    X, conn, U = _cnh_setup()
    p = [1.0, 99.3]
    ref = ElementLoop(X, conn, CNH, p, precision=FP64)
    fr, kr, rc, _ = ref.evaluate(0.0, U)
    assert rc == 0
    ext = ElementLoop(X, conn, M.EXTERNAL, [[0.0]], precision=FP64)
    L = M._setup()
    dU = torch.as_tensor(U, device="cuda")
    ne = ext.n_elem
    dF = torch.zeros(9 * 8 * ne, dtype=torch.float64, device="cuda")
    assert L.ceos_gp_deformation_device(ext.handle, C.c_void_p(dU.data_ptr()), C.c_void_p(dF.data_ptr()), None) == 0
    torch.cuda.synchronize()
    F = dF.view(9, 8 * ne).T.cpu().numpy().reshape(-1, 3, 3)
    vals = np.zeros((8 * ne, 27))
    iu = np.triu_indices(6)
    for q in range(8 * ne):
        s, D, _, _ = O.material_point(O.CNH, p, F[q])
        vals[q, :6] = s
        vals[q, 6:] = D[iu]
    qi = np.arange(8 * ne, dtype=np.int32)
    assert L.ceos_state_scatter(ext.handle, len(qi), qi.ctypes.data_as(C.c_void_p),
                                np.ascontiguousarray(vals).ctypes.data_as(C.c_void_p), 27) == 0
    fe, ke, rc, _ = ext.evaluate(0.0, U)
    assert rc == 0
    assert np.abs(fe - fr).max() <= 1e-11 * np.abs(fr).max()
    assert np.abs(ke - kr).max() <= 1e-11 * np.abs(kr).max()


def test_device_pcg_solves_dirichlet_system():
    X, conn, U = _cnh_setup(4)
    loop = ElementLoop(X, conn, CNH, [1.0, 99.3], precision=FP64)
    _, kval, rc, _ = loop.evaluate(0.0, U)
    fixed, presc = M.uniaxial_bc(X)
    mask = np.zeros(loop.n_dof, np.uint8)
    mask[fixed] = 1
    mask[presc] = 1
    rng = np.random.default_rng(3)
    b = rng.normal(size=loop.n_dof) * (mask == 0)
    L = M._setup()
    pcg = C.c_void_p()
    assert L.ceos_pcg_create(loop.handle, C.byref(pcg)) == 0
    dK = torch.as_tensor(kval, device="cuda")
    dm = torch.as_tensor(mask, device="cuda")
    db = torch.as_tensor(b, device="cuda")
    dx = torch.zeros_like(db)
    it, rel = C.c_int(), C.c_double()
    rc = L.ceos_pcg_solve(pcg, C.c_void_p(dK.data_ptr()), C.c_void_p(dm.data_ptr()), C.c_void_p(db.data_ptr()),
                          C.c_void_p(dx.data_ptr()), 1e-10, 5000, C.byref(it), C.byref(rel))
    assert rc == 0 and rel.value <= 1e-10
    x = dx.cpu().numpy()
    rowmap, col = loop.pattern()
    r = np.repeat(np.arange(loop.n_dof), np.diff(rowmap))
    K = sp.csr_matrix((kval, (r, col - 1)), shape=(loop.n_dof, loop.n_dof))
    K = K + K.T - sp.diags(K.diagonal())
    free = mask == 0
    res = (K @ x - b)[free]
    assert np.all(x[~free] == 0.0)
    assert np.linalg.norm(res) <= 1e-9 * np.linalg.norm(b)
    L.ceos_pcg_destroy(pcg)


def test_macro_element_with_rve_points_matches_oracle():
    """One macro cell, 8 Gauss points each with a 3^3 RVE (vf 0.3), stretched 4 % in two steps by
    the direct method; every point's first Piola stress equals the FP64 RVE oracle at its F."""
    m = M.MacroFE2(1, np.array([0.3]), n_cells=3)
    out = m.run(stretch=1.04, n_steps=2, mode="direct", tol=1e-8)
    assert np.all(out["newton"] >= 1)
    P = m.gp_first_piola()
    F = m._gp_F_host()
    for q in (0, 3, 7):
        Po = F2.RVE(3, 0.3).solve(F[q])
        assert np.abs(P[q] - Po).max() <= 1e-6 * np.abs(Po).max(), q
    m.close()


def test_fallback_pool_reproduces_direct_rve_solves():
    """A surrogate whose training box is empty sends every point to RVE solves; through the warm RVE
    pool (the large-mesh path, forced here) and the sticky fallback the macro run must reproduce the
    direct run's Gauss-point stresses."""
    from ceos_b200 import surrogate as SG
    sur = SG.Surrogate(batch_max=256)
    sur.set_params(SG.init_params(0))
    sur.set_scaling(0.15, 1.0, 0.25, 0.15, lo=np.full(7, 1e3), hi=np.full(7, 1e3 + 1))
    vf = np.array([0.3])
    fields = {}
    for mode in ("direct", "surrogate"):
        m = M.MacroFE2(1, vf, n_cells=3, surrogate=sur)
        m.point_batch_limit = 0  # large-mesh path: slots in the warm pool
        m.pool_size = 16
        out = m.run(stretch=1.03, n_steps=2, mode=mode, tol=1e-8)
        if mode == "surrogate":
            assert out["fallback_points"].min() >= 8  # every point, every material evaluation
        fields[mode] = m.gp_first_piola()
        m.close()
    Pd, Ps = fields["direct"], fields["surrogate"]
    assert np.abs(Ps - Pd).max() <= 1e-6 * np.abs(Pd).max()
    sur.close()
