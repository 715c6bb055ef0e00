"""Pins the FP64 oracle against the reference's only golden Hexa8 case
(Checker/Cases/NonLinear_FEA_3D_Hexa8_StVenant): MARC displacement curves of node 11 with
the Checker's absolute tolerance 1e-5 (Run_Checker.bat), Newton iteration counts per step
(NumOfIterRef.dat, tolerance 1e-3) and the per-iteration residual norms of Log_CEOS.txt.
The golden logs follow an absolute max-norm criterion ||R||_inf < Tol (norm_mode=1)."""
import numpy as np

import oracle as O
from ceos_b200 import meshgen


def _run(golden, norm_mode=1):
    X = np.array(golden["X"]).reshape(-1, 3)
    conn = np.array(golden["conn"]).reshape(-1, 8)
    bc = meshgen.golden_hexa8_svk_bc(golden)
    m = O.Model(X, conn, [O.SVK], [[golden["material"]["YoungModulus"], golden["material"]["Poisson"]]])
    node = golden["probe_node"]
    dofs = [3 * (node - 1) + d + 1 for d in range(3)]
    return m.analysis(bc, tol=golden["newton"]["tol"], itmax=golden["newton"]["itmax"], norm_mode=norm_mode,
                      probe_dofs=dofs)


def test_golden_marc_curves_and_counts(golden):
    r = _run(golden)
    assert r["rc"] == 0
    for k, comp in enumerate("xyz"):
        marc = np.array(golden["marc"][comp])[1:, 1]
        assert np.abs(r["probe"][k] - marc).max() <= 1e-5, comp
    ref = np.array([row[1] for row in golden["iterations_ref"][1:]])
    assert np.abs(r["iters"] - ref).max() <= 1e-3
    assert int(r["iters"].sum()) == 162


def test_golden_iteration_norms(golden):
    r = _run(golden)
    log = np.array([v for s in golden["log_norms"] for v in s])
    ours = np.asarray(r["norms"])
    assert ours.size == log.size == 212
    big = log > 1e-2          # below that the printed norms are round-off
    np.testing.assert_allclose(ours[big], log[big], rtol=1e-5)
    # small norms: the same convergence decision against the absolute tolerance
    np.testing.assert_array_equal(ours[~big] < 1e-3, log[~big] < 1e-3)


def test_relative_criterion_runs(golden):
    """The current source's relative criterion converges in fewer iterations."""
    r = _run(golden, norm_mode=0)
    assert r["rc"] == 0
    assert int(r["iters"].sum()) < 162
