"""The reference's own case workflow on the GPU: Settings.dat + Mesh.dat -> analysis (FEMAnalysis.result)
-> post-processing (probe files, NumberOfIterationsToConverge.dat) -> Checker against the MARC curves
and iteration counts with the tolerances of each case's Run_Checker.bat; restart from a result file
of a path-dependent (J2) case; Gauss-point probes against the FP64 oracle."""
import os
import shutil

import numpy as np
import pytest

import oracle as O
from ceos_b200 import caseio as io

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = os.path.join(HERE, "golden", "cases")


@pytest.mark.parametrize("name,tol", [("hexa8_svk", 1e-5), ("hexa8_nh_q1p0", 1e-3)])
def test_checker_workflow(tmp_path, name, tol):
    case_dir = os.path.join(CASES, name)
    c = io.Case(case_dir)
    out = str(tmp_path)
    r = c.run(out)
    assert r["rc"] == 0
    n, recs = io.read_result(r["result_file"])
    assert n == c.n_dof and sum(rec["flag_end_step"] for rec in recs) == 51
    c.post_process(out)
    # Run_Checker.bat: three probe files against MARC, the iteration counts at 1e-3
    for comp in "xyz":
        ok, msg = io.check(io.find_file(out, f"ceos_disp_{comp}.probe"),
                           os.path.join(case_dir, f"marc_disp_{comp}.dat"), tol)
        assert ok, (comp, msg)
    ok, msg = io.check(os.path.join(out, "NumberOfIterationsToConverge.dat"),
                       os.path.join(case_dir, "NumOfIterRef.dat"), 1e-3)
    assert ok, msg


def _j2_case(tmp_path):
    d = tmp_path / "j2case"
    shutil.copytree(os.path.join(CASES, "hexa8_svk"), d)
    s = (d / "Settings.dat").read_text(encoding="latin-1")
    s = s.replace("\tSt_Venant_Kirchhoff\n\tYoung Modulus = 100.0E9 \n\tPoisson = 0.3\n",
                  "\tJ2_Plasticity\n\tYoung Modulus = 100.0E9\n\tPoisson = 0.3\n\tYield Stress = 250.0E6\n"
                  "\tHardening Modulus = 21.0E9\n")
    (d / "Settings.dat").write_text(s, encoding="latin-1")
    (d / "Table_Disp_Z.tab").write_text("Time\tValue\n0.0e0\t0.0e0\n1.0e0\t0.0150d0\n")
    (d / "Table_Load_Y.tab").write_text("Time\tValue\n0.0\t0.0\n1.0\t0.0\n")
    c = io.Case(str(d))
    assert c.model == io.J2_SMALL
    return c


def test_restart_of_a_path_dependent_case(tmp_path):
    """J2 plasticity (elastic-plastic from the first steps): 20 steps, restart from the result file
    for the remaining 30, against one uninterrupted run; a continuation without the replayed plastic
    state ends elsewhere, so the comparison sees the state."""
    c = _j2_case(tmp_path)
    full, part = tmp_path / "full", tmp_path / "part"
    full.mkdir()
    part.mkdir()
    r_full = c.run(str(full), norm_mode=0, tol=1e-8)
    assert r_full["rc"] == 0 and r_full["iters"].max() >= 4       # plastic steps need several iterations
    r_part = c.run(str(part), norm_mode=0, tol=1e-8, n_steps=20)
    assert r_part["rc"] == 0
    r_rest = c.restart(str(part), norm_mode=0, tol=1e-8)
    assert r_rest["rc"] == 0 and r_rest["first_step"] == 20
    assert np.abs(r_rest["iters"] - r_full["iters"][20:]).max() <= 1
    np.testing.assert_allclose(r_rest["U"], r_full["U"], rtol=1e-9, atol=1e-14)
    _, a = io.read_result(os.path.join(full, "FEMAnalysis.result"))
    _, b = io.read_result(os.path.join(part, "FEMAnalysis.result"))
    assert [x["step"] for x in a if x["flag_end_step"]] == [x["step"] for x in b if x["flag_end_step"]]
    # the same 30 steps continued from the step-20 U alone, on virgin Gauss-point states
    U20 = [x for x in b if x["step"] == 20 and x["flag_end_step"] == 1][0]["U"]
    loop = c.element_loop()
    try:
        r_fresh = loop.analysis(c._slice_bc(20), 1e-8, 10, 0, 2, 10, U0=U20)
    finally:
        loop.close()
    assert r_fresh["rc"] == 0
    assert np.abs(r_fresh["U"] - r_full["U"]).max() > 1e-3 * np.abs(r_full["U"]).max()


def test_gauss_point_probes_against_the_oracle(tmp_path):
    """Cauchy stress, F and logarithmic strain probes of one Gauss point of the St Venant case at
    every end step: sigma against the oracle's update at the same U, F through the SVK closed form
    sigma = F S F^T / J, the logarithmic strain through exp(2 E_log) = F F^T."""
    case_dir = os.path.join(CASES, "hexa8_svk")
    c = io.Case(case_dir)
    out = str(tmp_path)
    assert c.run(out)["rc"] == 0
    el, gp = 37, 5
    probes = [io.GaussPointProbe("s.probe", "Cauchy Stress", el, gp, "All"),
              io.GaussPointProbe("f.probe", "Deformation Gradient", el, gp, "All"),
              io.GaussPointProbe("e.probe", "Logarithmic Strain", el, gp, "1, 2, 3, 4, 5, 6"),
              io.GaussPointProbe("bad.probe", "Cauchy Stress", el, 9, "All")]
    c.post_process(out, probes=probes)
    S = np.loadtxt(os.path.join(out, "s.probe"), skiprows=1)
    F = np.loadtxt(os.path.join(out, "f.probe"), skiprows=1)
    E = np.loadtxt(os.path.join(out, "e.probe"), skiprows=1)
    assert S.shape == (51, 7) and F.shape == (51, 10) and E.shape == (51, 7)
    assert open(os.path.join(out, "bad.probe")).read().splitlines()[1].startswith("ERROR - Number of Gauss Point")
    _, recs = io.read_result(os.path.join(out, "FEMAnalysis.result"))
    ends = [r for r in recs if r["flag_end_step"] == 1]
    m = O.Model(c.mesh["X"], c.mesh["conn"], [O.SVK], c.params)
    Ey, nu = c.params[0]
    lam, mu = Ey * nu / ((1 + nu) * (1 - 2 * nu)), Ey / (2 * (1 + nu))
    for k in (10, 30, 50):
        rec = ends[k]
        assert S[k, 0] == pytest.approx(rec["time"], rel=1e-14)
        m.evaluate(rec["time"], rec["U"], tangent=False)
        sig_o = m.gp_stress()[el - 1, gp - 1]
        np.testing.assert_allclose(S[k, 1:], sig_o, rtol=1e-12, atol=1e-9 * np.abs(sig_o).max())
        Fk = F[k, 1:].reshape(3, 3).T                      # columns of Convert_to_Voigt_3D
        G = 0.5 * (Fk.T @ Fk - np.eye(3))
        Sk = lam * np.trace(G) * np.eye(3) + 2 * mu * G
        sig = Fk @ Sk @ Fk.T / np.linalg.det(Fk)
        v = np.array([sig[0, 0], sig[1, 1], sig[2, 2], sig[0, 1], sig[1, 2], sig[0, 2]])
        np.testing.assert_allclose(S[k, 1:], v, rtol=1e-9, atol=1e-9 * np.abs(v).max())
        El = np.array([[E[k, 1], E[k, 4], E[k, 6]], [E[k, 4], E[k, 2], E[k, 5]], [E[k, 6], E[k, 5], E[k, 3]]])
        w, V = np.linalg.eigh(El)
        np.testing.assert_allclose(V @ np.diag(np.exp(2 * w)) @ V.T, Fk @ Fk.T, rtol=0, atol=1e-12)
