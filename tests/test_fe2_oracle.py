"""CPU checks of the FP64 RVE oracle that checks the batched FE^2 solver."""
import numpy as np

import fe2_oracle as F2


def test_homogenized_stress_equals_virtual_work_and_tangent_is_symmetric():
    r = F2.RVE(3, 0.3)
    Fb = np.eye(3) + np.array([[0.08, 0.03, 0.0], [0.01, -0.04, 0.02], [0.0, 0.02, 0.05]])
    P = r.solve(Fb)
    fint, _, _, _ = r.model.evaluate(0.0, r.U)
    Pvw = np.array([[(fint[i::3] * r.X[:, J]).sum() for J in range(3)] for i in range(3)])
    assert np.abs(P - Pvw).max() <= 1e-12 * np.abs(P).max()
    A = r.tangent_fd(Fb.reshape(-1))
    # hyperelastic homogenized response: major symmetry dP_iJ/dF_kL = dP_kL/dF_iJ
    assert np.abs(A - A.T).max() <= 1e-5 * np.abs(A).max()


def test_homogeneous_rve_is_affine():
    """vf = 0: no fibre, the periodic fluctuation vanishes and Pbar is the matrix stress."""
    r = F2.RVE(3, 0.0)
    Fb = np.eye(3) + np.array([[0.1, 0.02, 0], [0, -0.03, 0], [0.01, 0, 0.02]])
    P = r.solve(Fb)
    assert r.iters <= 1
    mu, lam = 1.0, 100.0 - 2.0 / 3.0
    J = np.linalg.det(Fb)
    sig = mu / J * (Fb @ Fb.T - np.eye(3)) + lam / J * np.log(J) * np.eye(3)
    assert np.allclose(P, J * sig @ np.linalg.inv(Fb).T, rtol=1e-10, atol=1e-12)


def test_partial_volume_fibre_fraction():
    """Cells carry the fibre's area fraction, so the realised volume fraction follows the nominal
    one smoothly at every resolution (the centroid rule jumps by whole cell columns)."""
    for n in (6, 8, 12):
        for vf in (0.1, 0.25, 0.4):
            X, conn, phi, ind = F2.rve_mesh(n, vf)
            assert phi.min() >= 0.0 and phi.max() <= 1.0
            assert abs(phi.mean() - vf) < 4e-3, (n, vf, phi.mean())
    # an interior cell of the fibre is pure fibre, a corner cell pure matrix
    phi = F2.fibre_fraction(8, 0.4 / np.pi)
    assert phi[4, 4] == 1.0 and phi[0, 0] == 0.0


def test_reference_periodic_map_structure():
    """The reference's BuildT on an n^3 RVE: n^3 independent nodes (minus faces, edges, vertex and
    interior), every plus node tied to its periodic image, the 8 vertices to one node."""
    for n in (2, 3, 4):
        X, conn, phi, ind = F2.rve_mesh(n, 0.2)
        T, vdofs = F2.reference_periodic_T(X)
        assert T.shape == (3 * X.shape[0], 3 * n ** 3)
        assert np.all(np.asarray(T.sum(axis=1)).ravel() == 1.0)
        assert len(vdofs) == 24
        cols = T.tocsr().indices.reshape(-1, 3)[:, 0]
        assert len(set(cols[vdofs[::3] // 3])) == 1          # all vertices share one column
        # the same grouping as the project's periodic map: equal T columns <=> equal index mod n
        same = (cols[:, None] == cols[None, :])
        same_ind = (ind[:, None] == ind[None, :])
        assert np.array_equal(same, same_ind)


def test_reference_periodic_formulation_equals_project_formulation():
    """An isochoric macro deformation (F33 = 1/(F11 F22), so the reference's F33 line is the identity)
    with in-plane shear: the reference's T^T K T formulation with fixed vertices and the project's
    periodic map with one fixed independent node give the same homogenized stress."""
    Fb = np.array([[1.08, 0.05, 0.0], [0.0, 0.96, 0.0], [0.0, 0.0, 1.0 / (1.08 * 0.96)]])
    for n, vf in ((3, 0.3), (4, 0.2)):
        Pp = F2.RVE(n, vf).solve(Fb)
        Pr = F2.RVEReference(n, vf).solve(Fb)
        assert np.abs(Pr - Pp).max() <= 1e-9 * np.abs(Pp).max(), (n, np.abs(Pr - Pp).max())
