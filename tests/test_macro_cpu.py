"""CPU checks of the macro FE^2 host logic: the conversion of RVE outputs (first Piola stress and
its tangent dP/dF) into the Cauchy stress and spatial tangent the element loop reads, against
the compressible Neo-Hookean oracle, and the uniaxial boundary conditions."""
import numpy as np

import oracle as O
from ceos_b200 import meshgen
from ceos_b200.macro import spatial_from_PA, uniaxial_bc


def _P(F, p):
    s, _, _, _ = O.material_point(O.CNH, p, F)
    S = np.array([[s[0], s[3], s[5]], [s[3], s[1], s[4]], [s[5], s[4], s[2]]])
    return np.linalg.det(F) * S @ np.linalg.inv(F).T


def test_spatial_tangent_from_first_piola_tangent():
    rng = np.random.default_rng(0)
    p = [1.0, 99.3]
    for _ in range(3):
        F = np.eye(3) + rng.uniform(-0.2, 0.2, (3, 3))
        h = 1e-6
        A = np.zeros((9, 9))
        for k in range(9):
            dF = np.zeros(9)
            dF[k] = h
            A[:, k] = ((_P(F + dF.reshape(3, 3), p) - _P(F - dF.reshape(3, 3), p)) / (2 * h)).reshape(-1)
        sig, D = spatial_from_PA(F[None], _P(F, p)[None], A[None])
        s, Dref, _, _ = O.material_point(O.CNH, p, F)
        assert np.abs(sig[0] - s).max() <= 1e-12 * np.abs(s).max()
        assert np.abs(D[0] - Dref[np.triu_indices(6)]).max() <= 1e-8 * np.abs(Dref).max()


def test_uniaxial_bc_removes_rigid_motion():
    X, _ = meshgen.structured_box(3, 3, 3, jitter=0.0)
    fixed, presc = uniaxial_bc(X)
    assert len(presc) == 16 and np.all(presc % 3 == 0)
    assert len(set(fixed) & set(presc)) == 0
    # symmetry planes: x-dofs of x=0, y-dofs of y=0, z-dofs of z=0 (16 nodes each)
    assert len(fixed) == 3 * 16
    assert sorted(set(int(d) % 3 for d in fixed)) == [0, 1, 2]


def test_stress_error_measures_and_sampling():
    from ceos_b200 import fe2_surrogate as FS
    rng = np.random.default_rng(0)
    P = rng.normal(size=(50, 3, 3))
    e = FS.stress_errors(P * 1.01, P)
    assert abs(e["aggregate"] - 0.01) < 1e-12 and abs(e["median"] - 0.01) < 1e-12
    P2 = P.copy()
    P2[3] = np.nan  # unsolved reference points are ignored
    assert FS.stress_errors(P, P2)["n"] == 49
    F, vf = FS.sample_points(400, seed=2, small_fraction=0.5)
    G = F - np.eye(3)
    assert np.all(np.abs(G) <= 0.15 + 1e-12) and np.all(np.linalg.det(F) > 0)
    assert np.all((vf >= 0.1) & (vf <= 0.4))
    # the scaled half has smaller strains on average
    assert np.abs(G[:200]).mean() < np.abs(G[200:]).mean()


def test_path_samples_follow_the_uniaxial_macro_load():
    """The surrogate's training data covers the macro load path: stretch along the fibre axis up to
    1.26, nearly isochoric lateral contraction, local perturbations of a few percent."""
    from ceos_b200 import fe2_surrogate as FS
    F, vf = FS.sample_points(1000, seed=5, path_fraction=0.5, axis=2)
    path = F[500:]
    lam = path[:, 2, 2]
    assert lam.max() > 1.2 and lam.min() > 0.9
    J = np.linalg.det(path)
    assert np.all(np.abs(J - 1.0) < 0.25) and np.all(J > 0)
    C33 = np.einsum("nk,nk->n", path[:, :, 2], path[:, :, 2])
    assert C33.max() > 1.44            # the training box reaches C33 of stretch 1.2
    cube = F[:500] - np.eye(3)
    assert np.all(np.abs(cube) <= 0.15 + 1e-12)


def test_uniaxial_bc_along_the_fibre_axis():
    X, _ = meshgen.structured_box(3, 3, 3, jitter=0.0)
    fixed, presc = uniaxial_bc(X, axis=2)
    assert len(presc) == 16 and np.all(presc % 3 == 2)
    assert np.all(X[presc // 3, 2] == 1.0)
    assert len(set(fixed) & set(presc)) == 0 and len(fixed) == 3 * 16
