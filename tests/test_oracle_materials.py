"""Known-answer and tangent-consistency checks of the oracle's constitutive models.

The reference ships no golden vectors for these models, so they are pinned by closed forms and by
the reference's own technique of finite-difference tangents (ModConstitutiveModel.f90:104-164):
the spatial tangent D must satisfy J D : d = L_v(tau)[d] = dtau[d] - d tau - tau d for every
symmetric rate d, with tau = J sigma and the perturbation F -> (I + h d) F.
"""
import numpy as np
import pytest

import oracle as O

CNH_P = [1.0, 100.0 - 2.0 / 3.0]
PRONY_P = [1.0, 100.0, 3, 0.3, 0.01, 0.2, 0.1, 0.1, 1.0, 0.0, 1.0]
J2_P = [200.0e3, 0.3, 250.0, 1000.0]
VI = [(0, 0), (1, 1), (2, 2), (0, 1), (1, 2), (0, 2)]


def sym(v):
    return np.array([[v[0], v[3], v[5]], [v[3], v[1], v[4]], [v[5], v[4], v[2]]])


def voigt(A):
    return np.array([A[0, 0], A[1, 1], A[2, 2], A[0, 1], A[1, 2], A[0, 2]])


def tau_of(model, params, F, dt, st_old, full=False):
    if full:
        sig, D, _ = O.j2_finite_full_tangent(params, F, st_old)
    else:
        sig, D, _, rc = O.material_point(model, params, F, dt, st_old)
        assert rc == 0
    return np.linalg.det(F) * sym(sig), D


def fd_tangent(model, params, F, dt=0.0, st_old=None, h=1e-7, full=False):
    J = np.linalg.det(F)
    tau0, D = tau_of(model, params, F, dt, st_old, full)
    Dfd = np.zeros((6, 6))
    for j, (a, b) in enumerate(VI):
        d = np.zeros((3, 3))
        d[a, b] += 0.5 if a != b else 1.0
        d[b, a] += 0.5 if a != b else 0.0  # engineering shear: unit Voigt strain = d_ab = d_ba = 1/2
        tp, _ = tau_of(model, params, (np.eye(3) + h * d) @ F, dt, st_old, full)
        tm, _ = tau_of(model, params, (np.eye(3) - h * d) @ F, dt, st_old, full)
        L = (tp - tm) / (2 * h) - d @ tau0 - tau0 @ d
        Dfd[:, j] = voigt(L) / J
    return D, Dfd


def rand_F(seed, amp=0.15):
    rng = np.random.default_rng(seed)
    F = np.eye(3) + rng.uniform(-amp, amp, (3, 3))
    assert np.linalg.det(F) > 0.3
    return F


def test_cnh_uniaxial_closed_form():
    lam = 1.3
    F = np.diag([lam, 1.0, 1.0])
    sig, D, _, rc = O.material_point(O.CNH, CNH_P, F)
    mu, la = CNH_P
    J = lam
    assert rc == 0
    assert np.isclose(sig[0], mu / J * (lam ** 2 - 1) + la / J * np.log(J), rtol=1e-14)
    assert np.isclose(sig[1], la / J * np.log(J), rtol=1e-14)
    assert np.allclose(sig[3:], 0.0)


@pytest.mark.parametrize("seed", [0, 1, 2])
@pytest.mark.parametrize("model,params", [(O.CNH, CNH_P), (O.SVK, [100.0, 0.3])])
def test_hyperelastic_tangent_consistency(model, params, seed):
    D, Dfd = fd_tangent(model, params, rand_F(seed))
    assert np.abs(D - Dfd).max() <= 1e-6 * np.abs(D).max()


@pytest.mark.parametrize("seed", [0, 1])
def test_visco_prony_tangent_consistency(seed):
    st = O.init_state(O.VISCO_PRONY, PRONY_P)
    # history: one increment, then the tangent of the next one at fixed committed state
    _, _, st1, _ = O.material_point(O.VISCO_PRONY, PRONY_P, rand_F(seed + 10, 0.05), 0.02, st)
    D, Dfd = fd_tangent(O.VISCO_PRONY, PRONY_P, rand_F(seed), dt=0.025, st_old=st1)
    assert np.abs(D - Dfd).max() <= 1e-6 * np.abs(D).max()


def test_visco_prony_instantaneous_and_relaxed_limits():
    """dt -> 0 from the virgin state: isochoric stress scaled by (1 + sum beta);
    dt >> tau: the ground state alone."""
    F = np.diag([1.1, 1 / np.sqrt(1.1), 1 / np.sqrt(1.1)])
    ground = list(PRONY_P)
    ground[2] = 0
    sg, _, _, _ = O.material_point(O.VISCO_PRONY, ground, F, 1.0, np.zeros(30))
    s0, _, _, _ = O.material_point(O.VISCO_PRONY, PRONY_P, F, 1e-12, np.zeros(30))
    sinf, _, _, _ = O.material_point(O.VISCO_PRONY, PRONY_P, F, 1e6, np.zeros(30))
    dev = lambda s: s - np.r_[np.full(3, s[:3].mean()), np.zeros(3)]
    assert np.allclose(dev(s0), 1.6 * dev(sg), rtol=1e-9)
    assert np.allclose(sinf, sg, rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_j2_finite_tangent_consistency_and_yield(seed):
    st = O.init_state(O.J2_FINITE, J2_P)
    F = rand_F(seed, 0.01)  # strains ~1e-2 >> yield strain 1.25e-3: plastic
    D, Dfd = fd_tangent(O.J2_FINITE, J2_P, F, st_old=st, full=True)
    assert np.abs(D - Dfd).max() <= 1e-5 * np.abs(D).max()
    sig, Dsym, st_new, _ = O.material_point(O.J2_FINITE, J2_P, F, 0.0, st)
    assert st_new[6] > 0.0
    J = np.linalg.det(F)
    s = J * sig - np.r_[np.full(3, (J * sig[:3]).mean()), np.zeros(3)]
    ns = np.sqrt((s[:3] ** 2).sum() + 2 * (s[3:] ** 2).sum())
    assert np.isclose(ns, np.sqrt(2 / 3) * (J2_P[2] + J2_P[3] * st_new[6]), rtol=1e-10)
    assert np.allclose(Dsym, 0.5 * (D + D.T), rtol=1e-12, atol=1e-9)


def test_j2_finite_elastic_is_neo_hookean_like():
    """Below yield there is no plastic flow and the tangent is consistent."""
    st = O.init_state(O.J2_FINITE, J2_P)
    F = rand_F(3, 1e-4)
    sig, D, st_new, _ = O.material_point(O.J2_FINITE, J2_P, F, 0.0, st)
    assert st_new[6] == 0.0
    D2, Dfd = fd_tangent(O.J2_FINITE, J2_P, F, st_old=st, full=True, h=1e-9)
    assert np.abs(D2 - Dfd).max() <= 1e-5 * np.abs(D2).max()


def test_j2_small_return_mapping_consistency():
    """Small-strain J2 as the reference writes it: after a plastic step q = sigma_y + H alpha."""
    st = O.init_state(O.J2_SMALL, J2_P)
    F = np.eye(3) + np.array([[0.01, 0.002, 0], [0.0, -0.003, 0], [0, 0, -0.003]])
    sig, D, st_new, _ = O.material_point(O.J2_SMALL, J2_P, F, 0.0, st)
    assert st_new[6] > 0
    p = sig[:3].mean()
    s = sig - np.r_[np.full(3, p), np.zeros(3)]
    q = np.sqrt(1.5 * ((s[:3] ** 2).sum() + 2 * (s[3:] ** 2).sum()))
    assert np.isclose(q, J2_P[2] + J2_P[3] * st_new[6], rtol=1e-12)


VV_P = [0.0, 1.0, 100.0 - 2.0 / 3.0, 0.0, 0.5, 0.2]  # K_inf, Mu_inf, Lambda_inf, K_e, Mu_e, Ni_v


@pytest.mark.parametrize("seed", [0, 1])
def test_visco_var_tangent_consistency_and_incompressible_flow(seed):
    """The reference's variational model (ModViscoelasticMatrix.f90): the consistent tangent of
    the local-Newton solution matches finite differences, and the converged viscous flow keeps
    det Fv = 1 to the local tolerance."""
    st0 = O.init_state(O.VISCO_VAR, VV_P)
    _, _, st1, rc = O.material_point(O.VISCO_VAR, VV_P, rand_F(seed + 5, 0.05), 0.1, st0)
    assert rc == 0
    assert abs(np.linalg.det(st1[:9].reshape(3, 3, order="F")) - 1.0) < 1e-5
    D, Dfd = fd_tangent(O.VISCO_VAR, VV_P, rand_F(seed, 0.05), dt=0.1, st_old=st1, h=1e-6)
    assert np.abs(D - Dfd).max() <= 1e-5 * np.abs(D).max()


def test_visco_var_relaxes_to_equilibrium_branch():
    """Held isochoric stretch: after a long time the Maxwell branch relaxes and the stress tends to
    the equilibrium Neo-Hookean branch alone (Mu_inf, Lambda_inf).  (The viscous flow is
    isochoric, J_v = 1, so a volumetric stretch would keep a residual branch stress.)"""
    F = np.diag([1.05, 1.05 ** -0.5, 1.05 ** -0.5])
    st = O.init_state(O.VISCO_VAR, VV_P)
    s_first = None
    for k in range(60):
        sig, _, st, rc = O.material_point(O.VISCO_VAR, VV_P, F, 0.5, st)
        assert rc == 0
        if s_first is None:
            s_first = sig.copy()
    eq = list(VV_P)
    eq[4] = 1e-12  # no Maxwell branch
    s_eq, _, _, _ = O.material_point(O.VISCO_VAR, eq, F, 0.5, O.init_state(O.VISCO_VAR, eq))
    assert abs(s_first[0] - s_eq[0]) > 1e-3 * abs(s_eq[0])   # the branch carries stress at first
    assert np.allclose(sig, s_eq, rtol=1e-4, atol=1e-8)     # and has relaxed at the end


def test_mean_dilatation_element_tangent_matches_finite_differences():
    """The Mean Dilatation K (full-integration B^T D B + G^T S G with the Jbar pressure, plus
    Bdiv^T Bdiv d2psi/dJbar2 / V0) is the derivative of its f_int: central differences of f_int
    over the displacements of a jittered 2x2x2 mesh reproduce the assembled K."""
    from ceos_b200 import meshgen
    X, conn = meshgen.structured_box(2, 2, 2, jitter=0.05, seed=4)
    m = O.Model(X, conn, [O.NH_Q1P0], [[1.0, 50.0]])
    rng = np.random.default_rng(1)
    U = 0.05 * (X @ rng.uniform(-1, 1, (3, 3)).T).reshape(-1) + 0.01 * rng.uniform(-1, 1, X.size)
    f0, kval, rc, _ = m.evaluate(0.0, U)
    assert rc == 0
    rowmap, col = m.pattern()
    n = X.size
    K = np.zeros((n, n))
    for r in range(n):
        for p in range(rowmap[r] - 1, rowmap[r + 1] - 1):
            K[r, col[p] - 1] = kval[p]
            K[col[p] - 1, r] = kval[p]
    h = 1e-7
    for j in range(0, n, 5):
        e = np.zeros(n)
        e[j] = h
        fp, _, _, _ = m.evaluate(0.0, U + e, tangent=False)
        fm, _, _, _ = m.evaluate(0.0, U - e, tangent=False)
        assert np.abs((fp - fm) / (2 * h) - K[:, j]).max() <= 1e-5 * np.abs(K).max(), j
