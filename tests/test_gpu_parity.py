"""GPU parity of the sm_100a element loop against the FP64 oracle, through the C ABI.

Bars (stated per test): the CSR pattern and slot map are bit-exact; in FP64 mode f_int and K
agree with the oracle to 1e-12 relative (max-norm relative to the largest entry); in mixed
mode to per-model bars of 2e-6 to 3e-5 (f_int) and 1e-6 (K); Newton histories match iteration counts exactly and norms to 1e-6 relative."""
import numpy as np
import pytest

import oracle as O
import ceos_b200 as G
from ceos_b200 import meshgen

pytestmark = pytest.mark.gpu

CNH_P = [1.0, 100.0 - 2.0 / 3.0]                       # mu = 1, K = 100 -> lambda = K - 2 mu / 3
SVK_P = [100.0e9, 0.3]
J2S_P = [200.0e3, 0.3, 250.0, 1000.0]
J2F_P = [200.0e3, 0.3, 250.0, 1000.0]
PRONY_P = [1.0, 100.0, 3, 0.3, 0.01, 0.2, 0.1, 0.1, 1.0, 0.0, 1.0]
VV_P = [0.0, 1.0, 100.0 - 2.0 / 3.0, 0.0, 0.5, 0.2]   # K_inf, Mu_inf, Lambda_inf, K_e, Mu_e, Ni_v
Q1P0_P = [0.5, 100.0]                                  # C10, BulkModulus (Mean Dilatation element)


def smooth_u(X, amp, seed=1):
    rng = np.random.default_rng(seed)
    A = rng.uniform(-1, 1, (3, 3)) * amp
    u = X @ A.T + amp * 0.3 * np.sin(3 * X[:, [1, 2, 0]])
    return u.reshape(-1)


def relerr(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def shuffled_mesh(nx, ny, nz, seed=3):
    X, conn = meshgen.structured_box(nx, ny, nz, jitter=0.05, seed=seed)
    rng = np.random.default_rng(seed)
    perm = rng.permutation(X.shape[0])          # new id of old node i is perm[i]
    Xn = np.empty_like(X)
    Xn[perm] = X
    conn_n = perm[conn - 1] + 1
    eperm = rng.permutation(conn.shape[0])
    return Xn, conn_n[eperm].astype(np.int32)


@pytest.mark.parametrize("mesh", ["c1", "small", "shuffled", "golden"])
def test_pattern_and_slot_map_bit_exact(mesh, golden):
    if mesh == "c1":
        X, conn = meshgen.structured_box(10, 10, 10, jitter=0.05, seed=0)
    elif mesh == "small":
        X, conn = meshgen.structured_box(3, 2, 2, jitter=0.05, seed=1)
    elif mesh == "shuffled":
        X, conn = shuffled_mesh(5, 4, 3)
    else:
        X, conn = np.array(golden["X"]).reshape(-1, 3), np.array(golden["conn"]).reshape(-1, 8)
    g = G.ElementLoop(X, conn, G.CNH, CNH_P)
    rowmap, col, row = g.pattern(with_row=True)
    orow, ocol, orr = O.pattern(X.shape[0], conn)
    np.testing.assert_array_equal(rowmap, orow)
    np.testing.assert_array_equal(col, ocol)
    np.testing.assert_array_equal(row, orr)
    np.testing.assert_array_equal(g.slot_map(), O.slot_map(X.shape[0], conn, orow, ocol))
    g.close()


def _pair(model, params, X, conn, precision=G.FP64, per_element=False):
    g = G.ElementLoop(X, conn, model, params, precision=precision, per_element=per_element)
    o = O.Model(X, conn, [model], params, per_element=per_element)
    return g, o


@pytest.mark.parametrize("model,params,amp", [
    (G.CNH, CNH_P, 0.08), (G.SVK, SVK_P, 0.05), (G.J2_SMALL, J2S_P, 0.01),
    (G.J2_FINITE, J2F_P, 0.01), (G.VISCO_PRONY, PRONY_P, 0.08), (G.VISCO_VAR, VV_P, 0.05),
    (G.NH_Q1P0, Q1P0_P, 0.08)])
def test_evaluate_fp64(model, params, amp):
    X, conn = meshgen.structured_box(6, 5, 4, jitter=0.05, seed=2)
    g, o = _pair(model, params, X, conn)
    t = 0.0
    for step in range(3):                      # three increments with commits: history matters
        t += 0.025
        U = smooth_u(X, amp * (step + 1), seed=step)
        fg, kg, rc, nf = g.evaluate(t, U)
        fo, ko, rco, nfo = o.evaluate(t, U)
        assert rc == rco == 0 and nf == nfo == 0
        assert relerr(fg, fo) <= 1e-12, ("fint", step)
        assert relerr(kg, ko) <= 1e-12, ("K", step)
        if g.nstate:
            np.testing.assert_allclose(g.state(1), o.state(1)[:, :, :g.nstate], rtol=1e-11, atol=1e-13)
        g.commit()
        o.commit()
        g.set_committed_time(t)
        o.set_time_old(t)
    g.close()


# Mixed-precision bars (f_int, K) about 3x the largest error measured on a B200 over both increments
# and all three assemblies: f_int 5.6e-7 / 5.8e-7 / 9.2e-6 / 1.3e-6 / 1.8e-6 (CNH, Prony, finite J2,
# variational visco, Q1P0), K at most 3.3e-7.  Finite J2 carries the largest f_int error: the return
# mapping of a plastic Gauss point amplifies the FP32 rounding of F.
@pytest.mark.parametrize("model,params,amp,ftol,ktol", [
    (G.CNH, CNH_P, 0.08, 2e-6, 1e-6), (G.VISCO_PRONY, PRONY_P, 0.08, 2e-6, 1e-6),
    (G.J2_FINITE, J2F_P, 0.01, 3e-5, 1e-6), (G.VISCO_VAR, VV_P, 0.05, 4e-6, 1e-6),
    (G.NH_Q1P0, Q1P0_P, 0.08, 6e-6, 1e-6)])
@pytest.mark.parametrize("assembly", ["two-pass", "fused", "banded"])
def test_evaluate_mixed(model, params, amp, ftol, ktol, assembly):
    X, conn = meshgen.structured_box(6, 5, 4, jitter=0.05, seed=2)
    g, o = _pair(model, params, X, conn, precision=G.MIXED)
    g.set_assembly(assembly)
    t = 0.0
    for step in range(2):
        t += 0.025
        U = smooth_u(X, amp * (step + 1), seed=step)
        fg, kg, rc, _ = g.evaluate(t, U)
        fo, ko, _, _ = o.evaluate(t, U)
        assert rc == 0
        assert relerr(fg, fo) <= ftol, ("fint", step)
        assert relerr(kg, ko) <= ktol, ("K", step)
        g.commit(); o.commit(); g.set_committed_time(t); o.set_time_old(t)
    g.close()


def test_block_slots_clean_across_evaluations_and_assemblies():
    """Every mixed-precision assembly leaves its FP32 block slots at zero for the next evaluation.  A
    sequence of evaluations on a mesh of two host-call slabs (32^3 elements) -- host-buffer and device
    calls, one without a tangent, and switches to the fused and banded assemblies (which resize the
    slots) and back -- gives the oracle's f_int and K at every evaluation with a tangent (bars of
    test_evaluate_mixed for this model)."""
    import torch
    X, conn = meshgen.structured_box(32, 32, 32, jitter=0.05, seed=4)
    g, o = _pair(G.CNH, CNH_P, X, conn, precision=G.MIXED)
    U = smooth_u(X, 0.08, seed=5)
    fo, ko, rco, _ = o.evaluate(0.0, U)
    assert rco == 0
    dU = torch.tensor(U, dtype=torch.float64, device="cuda")
    steps = ["host", "host", "device", "no-tangent", "host", "fused", "two-pass", "device", "banded",
             "two-pass", "host", "host"]
    for k, step in enumerate(steps):
        if step in ("fused", "banded", "two-pass"):
            g.set_assembly(step)
            step = "host"
        if step == "no-tangent":
            fg, kg, rc, _ = g.evaluate(0.0, U, tangent=False)
            assert rc == 0 and kg is None
            assert relerr(fg, fo) <= 2e-6, (k, "fint")
            continue
        if step == "device":
            df = torch.zeros(g.n_dof, dtype=torch.float64, device="cuda")
            dk = torch.zeros(g.nnz, dtype=torch.float64, device="cuda")
            g.evaluate_device(0.0, dU, df, dk)
            torch.cuda.synchronize()
            fg, kg = df.cpu().numpy(), dk.cpu().numpy()
        else:
            fg, kg, rc, _ = g.evaluate(0.0, U)
            assert rc == 0
        assert relerr(fg, fo) <= 2e-6, (k, g.assembly, "fint")
        assert relerr(kg, ko) <= 1e-6, (k, g.assembly, "K")
    g.close()


def test_mixed_near_incompressible_shear_patch():
    """Mixed precision on the benchmark's problem (visco-Prony, K = 100 mu, simple shear after two
    committed increments) on a 16^3 mesh: the interior nodal forces cancel, so f_int is small against
    the element forces and exposes any loss of element-scale precision.  The element-local
    coordinate and displacement differences keep f_int within 2e-6 and K within 2e-6 of the FP64
    oracle (relative to their largest entries); rounding absolute coordinates to FP32 gave 1.7e-4."""
    X, conn = meshgen.structured_box(16, 16, 16, jitter=0.05, seed=0)
    g, o = _pair(G.VISCO_PRONY, PRONY_P, X, conn, precision=G.MIXED)

    def shear(t):
        U = np.zeros_like(X)
        U[:, 0] = 0.3 * np.sin(2.0 * np.pi * t) * X[:, 2]
        return U.reshape(-1)

    for k in (1, 2):
        t = 0.025 * k
        g.evaluate(t, shear(t), tangent=False)
        o.evaluate(t, shear(t), tangent=False)
        g.commit(); o.commit(); g.set_committed_time(t); o.set_time_old(t)
    fg, kg, rc, _ = g.evaluate(0.075, shear(0.075))
    fo, ko, _, _ = o.evaluate(0.075, shear(0.075))
    assert rc == 0
    assert relerr(fg, fo) <= 2e-6
    assert relerr(kg, ko) <= 2e-6
    g.close()


def test_per_element_params():
    X, conn = meshgen.structured_box(4, 4, 3, jitter=0.05, seed=5)
    rng = np.random.default_rng(9)
    ne = conn.shape[0]
    f = np.exp(rng.uniform(np.log(0.9), np.log(1.1), ne))
    P = np.tile(np.array(J2F_P), (ne, 1))
    P[:, 0] *= f
    P[:, 2] *= np.exp(rng.uniform(np.log(0.9), np.log(1.1), ne))
    g, o = _pair(G.J2_FINITE, P, X, conn, per_element=True)
    U = smooth_u(X, 0.01)
    fg, kg, _, _ = g.evaluate(0.1, U)
    fo, ko, _, _ = o.evaluate(0.1, U)
    assert relerr(fg, fo) <= 1e-12 and relerr(kg, ko) <= 1e-12
    g.close()


def test_gp_stress_matches_oracle():
    X, conn = meshgen.structured_box(3, 3, 3, jitter=0.05, seed=4)
    g, o = _pair(G.CNH, CNH_P, X, conn)
    g.store_stress(True)
    U = smooth_u(X, 0.05)
    g.evaluate(0.0, U)
    o.evaluate(0.0, U)
    np.testing.assert_allclose(g.gp_stress(), o.gp_stress(), rtol=1e-12, atol=1e-12)
    g.close()


def test_inverted_element_reports_status_1():
    X, conn = meshgen.structured_box(3, 3, 3, jitter=0.0)
    g = G.ElementLoop(X, conn, G.CNH, CNH_P)
    U = np.zeros(X.size)
    node = 13  # an interior node (0-based id 21 in a 4x4x4 grid is interior): push it through
    interior = np.nonzero((X[:, 0] > 0.1) & (X[:, 0] < 0.9) & (X[:, 1] > 0.1) & (X[:, 1] < 0.9)
                          & (X[:, 2] > 0.1) & (X[:, 2] < 0.9))[0]
    node = interior[0]
    U[3 * node] = 0.9                       # folds its elements
    fint, kval, rc, nf = g.evaluate(0.0, U)
    assert rc == 1 and nf > 0
    ids, msg = g.failed_elements()
    o = O.Model(X, conn, [O.CNH], CNH_P)
    _, _, rco, nfo = o.evaluate(0.0, U)
    assert rco == 1 and nf == nfo
    assert "Jacobian" in msg
    # the context stays usable: a clean evaluation afterwards succeeds
    _, _, rc2, nf2 = g.evaluate(0.0, np.zeros(X.size))
    assert rc2 == 0 and nf2 == 0
    g.close()


def test_golden_case_through_gpu(golden):
    """The reference's golden Hexa8 SVK case driven through the C ABI (host driver + GPU loop)."""
    X = np.array(golden["X"]).reshape(-1, 3)
    conn = np.array(golden["conn"]).reshape(-1, 8)
    bc = meshgen.golden_hexa8_svk_bc(golden)
    g = G.ElementLoop(X, conn, G.SVK, SVK_P)
    node = golden["probe_node"]
    r = g.analysis(bc, tol=1e-3, itmax=10, norm_mode=1, probe_dofs=[3 * (node - 1) + d + 1 for d in range(3)])
    assert r["rc"] == 0
    for k, comp in enumerate("xyz"):
        marc = np.array(golden["marc"][comp])[1:, 1]
        assert np.abs(r["probe"][k] - marc).max() <= 1e-5
    ref = np.array([row[1] for row in golden["iterations_ref"][1:]])
    np.testing.assert_array_equal(r["iters"], ref)
    log = np.array([v for s in golden["log_norms"] for v in s])
    big = log > 1e-2
    np.testing.assert_allclose(r["norms"][big], log[big], rtol=1e-5)
    g.close()


def test_mean_dilatation_golden_case_through_gpu(golden_nh):
    """The reference's Mean Dilatation golden case (Neo_Hookean, model 4) through the C ABI."""
    X = np.array(golden_nh["X"]).reshape(-1, 3)
    conn = np.array(golden_nh["conn"]).reshape(-1, 8)
    bc = meshgen.golden_hexa8_svk_bc(golden_nh)
    mat = golden_nh["material"]
    g = G.ElementLoop(X, conn, G.NH_Q1P0, [mat["C10"], mat["BulkModulus"]])
    node = golden_nh["probe_node"]
    r = g.analysis(bc, tol=1e-3, itmax=10, norm_mode=1, probe_dofs=[3 * (node - 1) + d + 1 for d in range(3)])
    assert r["rc"] == 0
    for k, comp in enumerate("xyz"):
        marc = np.array(golden_nh["marc"][comp])[1:, 1]
        assert np.abs(r["probe"][k] - marc).max() <= 1e-4
    ref = np.array([row[1] for row in golden_nh["iterations_ref"][1:]])
    np.testing.assert_array_equal(r["iters"], ref)
    log = np.array([v for s in golden_nh["log_norms"] for v in s])
    big = log > 1.0
    np.testing.assert_allclose(r["norms"][big], log[big], rtol=1e-5)
    g.close()


def test_config1_newton_history_matches_oracle():
    """Config 1 (10x10x10 CNH, stretch 1.5 in 10 increments, relative 1e-8, max-abs norm)."""
    X, conn = meshgen.structured_box(10, 10, 10, jitter=0.05, seed=0)
    bc = meshgen.config1_bc(X)
    g = G.ElementLoop(X, conn, G.CNH, CNH_P)
    o = O.Model(X, conn, [O.CNH], CNH_P)
    rg = g.analysis(bc, tol=1e-8, itmax=20, norm_mode=0)
    ro = o.analysis(bc, tol=1e-8, itmax=20, norm_mode=0)
    assert rg["rc"] == 0 and ro["rc"] == 0
    np.testing.assert_array_equal(rg["iters"], ro["iters"])
    n = min(len(rg["norms"]), len(ro["norms"]))
    big = ro["norms"][:n] > 1e-9 * ro["norms"][0]
    np.testing.assert_allclose(rg["norms"][:n][big], ro["norms"][:n][big], rtol=1e-6)
    assert relerr(rg["U"], ro["U"]) < 1e-9
    g.close()


def test_fem_system_of_equations_plugin():
    """EvaluateR / EvaluateKt with the rearrangement BCs equal the oracle's system."""
    X, conn = meshgen.structured_box(4, 4, 4, jitter=0.05, seed=0)
    bc = meshgen.config1_bc(X, n_steps=4)
    g = G.ElementLoop(X, conn, G.CNH, CNH_P)
    soe = G.FEMSystemOfEquations(g, bc["fixed"], bc["presc"])
    soe.Ubar[bc["presc"] - 1] = bc["presc_final"][:, 0]
    Xs = np.zeros(g.n_dof)
    R = soe.EvaluateR(Xs)
    K, Rb = soe.EvaluateKt(Xs, R)
    assert np.allclose(Rb[bc["presc"] - 1], -bc["presc_final"][:, 0])
    assert np.all(Rb[bc["fixed"] - 1] == 0.0)
    g.close()


@pytest.mark.parametrize("shape", [(1, 1, 1), (2, 1, 1), (11, 3, 1)])
@pytest.mark.parametrize("assembly", ["two-pass", "fused", "banded"])
def test_tiny_meshes_all_assemblies(shape, assembly):
    """Edge cases of the tiling: a single element (one tile of 1, one conversion item), two elements,
    and 33 elements (a full tile of 32 plus a tile of 1), with FP64 and with each mixed-precision K
    assembly, against the FP64 oracle (mixed bars about 3x the errors measured on a B200: f_int
    1.4e-6, K 3.3e-7); the CSR pattern bit-exact."""
    X, conn = meshgen.structured_box(*shape, jitter=0.05, seed=7)
    U = smooth_u(X, 0.05, seed=3)
    o = O.Model(X, conn, [G.CNH], CNH_P)
    fo, ko, rco, _ = o.evaluate(0.0, U)
    assert rco == 0
    for precision, ftol, ktol in ((G.FP64, 1e-12, 1e-12), (G.MIXED, 4e-6, 1e-6)):
        g = G.ElementLoop(X, conn, G.CNH, CNH_P, precision=precision)
        if precision == G.MIXED:
            g.set_assembly(assembly)
        fg, kg, rc, _ = g.evaluate(0.0, U)
        rowmap, col = g.pattern()
        g.close()
        assert rc == 0
        assert relerr(fg, fo) <= ftol and relerr(kg, ko) <= ktol, (precision, relerr(fg, fo), relerr(kg, ko))
        orow, ocol, _ = O.pattern(X.shape[0], conn)
        assert (rowmap == orow).all() and (col == ocol).all()
