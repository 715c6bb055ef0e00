"""Newton histories through ceos_analysis against the FP64 oracle and the reference's golden cases.

The reference's Newton criterion (ModNewtonRaphsonFull.f90:44-168) must give the same iteration
count per increment.  Checked here:
- the device-resident Newton (ceos_analysis_set_device_solver: boundary conditions of
  ApplyBoundaryConditionsNEW as kernels, K kept on the device, PCG to 1e-12 in place of PARDISO)
  on both golden Hexa8 cases: every per-step iteration count of the reference's
  NumOfIterRef.dat, the MARC probe curves (1e-5 and 1e-4 as the host-path tests) and the logged
  norms (1e-5 relative);
- config 1 (10^3 CNH to stretch 1.5, relative 1e-8): device Newton = oracle counts, norms 1e-6;
- config 2 reduced (visco-Prony cube, cyclic simple shear 0.3 sin(2 pi t), 40 steps of 0.025 s) and
  config 3 reduced (finite-strain J2 plate with per-element E and sigma_y, uniaxial tension to 5 %
  in 50 increments): GPU counts = oracle counts per increment and final U within 1e-8 (1e-7 for J2);
  norms within 1e-6 relative above round-off over the whole visco history and over the J2 increments
  up to first yield (after it the first tangent of an increment is taken at points on their yield
  surface, where its elastic/plastic branch depends on round-off).  FP64 element loop with the
  device Newton at relative 1e-8.  The mixed-precision loop with the device Newton runs against the
  oracle under the reference's absolute criterion (norm_mode 1): its FP32 element forces put an
  absolute floor under the residual (about 1.2e-7 for the visco cube, 4.5e-4 for the J2 plate, where
  the bulk term lambda ln J with lambda = 99 mu amplifies the FP32 rounding of F).  A relative
  criterion puts that floor close to tol * R0 in the increments around the load reversals of the
  cyclic shear, where R0 is small, and the count there depends on round-off; an absolute tolerance
  10-20x above the floor (1e-5 visco, 1e-2 J2) does not.  Norms are compared within 1e-4 relative
  plus three times the floor; U within 1e-4 of max |U| (each run stops somewhere below the
  criterion).
"""
import numpy as np
import pytest

import oracle as O
import ceos_b200 as G
from ceos_b200 import meshgen

pytestmark = pytest.mark.gpu

CNH_P = [1.0, 100.0 - 2.0 / 3.0]
SVK_P = [100.0e9, 0.3]
PRONY_P = [1.0, 100.0, 3, 0.3, 0.01, 0.2, 0.1, 0.1, 1.0, 0.0, 1.0]


def _golden_run(fx, model, params, marc_tol, big):
    X = np.array(fx["X"]).reshape(-1, 3)
    conn = np.array(fx["conn"]).reshape(-1, 8)
    bc = meshgen.golden_hexa8_svk_bc(fx)
    g = G.ElementLoop(X, conn, model, params)
    node = fx["probe_node"]
    r = g.analysis(bc, tol=1e-3, itmax=10, norm_mode=1, probe_dofs=[3 * (node - 1) + d + 1 for d in range(3)],
                   device_solver=True)
    g.close()
    assert r["rc"] == 0
    for k, comp in enumerate("xyz"):
        marc = np.array(fx["marc"][comp])[1:, 1]
        assert np.abs(r["probe"][k] - marc).max() <= marc_tol
    ref = np.array([row[1] for row in fx["iterations_ref"][1:]])
    np.testing.assert_array_equal(r["iters"], ref)
    log = np.array([v for s in fx["log_norms"] for v in s])
    sel = log > big
    np.testing.assert_allclose(r["norms"][sel], log[sel], rtol=1e-5)


def test_device_newton_golden_svk(golden):
    _golden_run(golden, G.SVK, SVK_P, 1e-5, 1e-2)


def test_device_newton_golden_mean_dilatation(golden_nh):
    mat = golden_nh["material"]
    _golden_run(golden_nh, G.NH_Q1P0, [mat["C10"], mat["BulkModulus"]], 1e-4, 1.0)


def _compare(rg, ro, norm_rtol=1e-6, u_tol=1e-8, norm_steps=None, norm_atol=0.0):
    """Equal iteration counts and cut-backs per increment, final U within u_tol; the norm histories of
    the first norm_steps increments (all when None) within norm_rtol (plus norm_atol) above round-off."""
    assert rg["rc"] == 0 and ro["rc"] == 0, (rg["rc"], ro["rc"])
    np.testing.assert_array_equal(rg["iters"], ro["iters"])
    np.testing.assert_array_equal(rg["cutbacks"], ro["cutbacks"])
    assert len(rg["norms"]) == len(ro["norms"])
    n = len(ro["norms"]) if norm_steps is None else int(np.sum(ro["iters"][:norm_steps] + 1))
    big = ro["norms"][:n] > 1e-6 * ro["norms"].max()
    np.testing.assert_allclose(rg["norms"][:n][big], ro["norms"][:n][big], rtol=norm_rtol, atol=norm_atol)
    assert np.abs(rg["U"] - ro["U"]).max() <= u_tol * np.abs(ro["U"]).max()


def test_device_newton_config1_matches_oracle():
    X, conn = meshgen.structured_box(10, 10, 10, jitter=0.05, seed=0)
    bc = meshgen.config1_bc(X)
    g = G.ElementLoop(X, conn, G.CNH, CNH_P)
    o = O.Model(X, conn, [O.CNH], CNH_P)
    rg = g.analysis(bc, tol=1e-8, itmax=20, norm_mode=0, device_solver=True)
    ro = o.analysis(bc, tol=1e-8, itmax=20, norm_mode=0)
    g.close()
    _compare(rg, ro)


def _config2(nx):
    X, conn = meshgen.structured_box(nx, nx, nx, jitter=0.05, seed=0)
    return X, conn, meshgen.config2_bc(X), G.VISCO_PRONY, PRONY_P, False


def _config3(nx):
    X, conn = meshgen.structured_box(nx, nx, nx // 2, lx=2.0, ly=2.0, lz=1.0, jitter=0.05, seed=0)
    rng = np.random.default_rng(3)
    ne = conn.shape[0]
    fac = np.exp(rng.uniform(np.log(0.9), np.log(1.1), (ne, 2)))
    P = np.zeros((ne, 4))
    P[:, 0] = 200e3 * fac[:, 0]
    P[:, 1] = 0.3
    P[:, 2] = 250.0 * fac[:, 1]
    P[:, 3] = 1e3
    return X, conn, meshgen.config3_bc(X), G.J2_FINITE, P, True


@pytest.mark.parametrize("config,nx", [("c2", 8), ("c3", 12)])
def test_newton_history_fp64_matches_oracle(config, nx):
    X, conn, bc, model, params, pe = (_config2 if config == "c2" else _config3)(nx)
    g = G.ElementLoop(X, conn, model, params, per_element=pe)
    o = O.Model(X, conn, [model], params, per_element=pe)
    rg = g.analysis(bc, tol=1e-8, itmax=20, norm_mode=0, device_solver=True)
    ro = o.analysis(bc, tol=1e-8, itmax=20, norm_mode=0)
    g.close()
    # J2: once points have yielded, every plastic point starts an increment on its yield surface up to
    # round-off, so the elastic/plastic choice of the first tangent of the increment (and with it the
    # norm history) depends on the last bits; the iteration counts and the solution do not
    _compare(rg, ro, u_tol=1e-7 if config == "c3" else 1e-8, norm_steps=2 if config == "c3" else None)


@pytest.mark.parametrize("config,nx", [("c2", 8), ("c3", 12)])
def test_newton_history_mixed_matches_oracle(config, nx):
    X, conn, bc, model, params, pe = (_config2 if config == "c2" else _config3)(nx)
    g = G.ElementLoop(X, conn, model, params, per_element=pe, precision=G.MIXED)
    o = O.Model(X, conn, [model], params, per_element=pe)
    tol, floor = (1e-5, 1.2e-7) if config == "c2" else (1e-2, 4.5e-4)
    rg = g.analysis(bc, tol=tol, itmax=20, norm_mode=1, device_solver=True)
    ro = o.analysis(bc, tol=tol, itmax=20, norm_mode=1)
    g.close()
    # U: each run stops somewhere below the residual criterion, which fixes U only to about
    # tol / stiffness: 1e-4 of max |U| (measured difference 1.8e-5 on the visco cube)
    _compare(rg, ro, norm_rtol=1e-4, u_tol=1e-4, norm_steps=2 if config == "c3" else None, norm_atol=3 * floor)
