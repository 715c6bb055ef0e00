"""Case files on the host (no GPU): the readers against the golden fixtures, the reference's reader
errors, FEMAnalysis.result round trips, the probe format, the Checker, and the record order of the
case driver (analysis, restart, post-processing) with a scripted stand-in for the GPU loop."""
import json
import os
import shutil

import numpy as np
import pytest

import oracle as O
from ceos_b200 import caseio as io
from ceos_b200 import meshgen

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = os.path.join(HERE, "golden", "cases")


@pytest.mark.parametrize("name", ["hexa8_svk", "hexa8_nh_q1p0"])
def test_case_reader_matches_golden_fixture(name):
    c = io.Case(os.path.join(CASES, name))
    with open(os.path.join(HERE, "golden", name + ".json")) as f:
        fx = json.load(f)
    np.testing.assert_array_equal(c.mesh["X"].reshape(-1), fx["X"])
    np.testing.assert_array_equal(c.mesh["conn"].reshape(-1), fx["conn"])
    np.testing.assert_array_equal(c.mesh["mat"], fx["mat_id"])
    bc = meshgen.golden_hexa8_svk_bc(fx)
    for k in bc:
        np.testing.assert_array_equal(np.asarray(c.bc[k]), np.asarray(bc[k]), err_msg=k)
    ns = c.settings["nonlinear_solver"]
    assert (ns["name"], ns["tol"], ns["maxiter"]) == ("newton_raphson_full", 1e-3, 10)
    assert c.settings["analysis"]["max_cutbacks"] == 10
    mat = fx["material"]
    if name == "hexa8_svk":
        assert c.model == io.SVK and c.params == [[mat["YoungModulus"], mat["Poisson"]]]
        assert c.settings["analysis"]["element_technology"] == "fullintegration"
    else:
        assert c.model == io.NH_Q1P0 and c.params == [[mat["C10"], mat["BulkModulus"]]]
        assert c.settings["analysis"]["element_technology"] == "meandilatation"
    assert c.labels[0] == (1, 1) and c.labels[-1] == (1, 50)
    probes = io.read_probes(os.path.join(CASES, name, "Post_Processing.post"))
    assert [(p.file_name, p.node, p.components) for p in probes] == [
        ("CEOS_Disp_X.probe", 11, [1]), ("CEOS_Disp_Y.probe", 11, [2]), ("CEOS_Disp_Z.probe", 11, [3])]


def _edit(tmp_path, name, old, new, case="hexa8_svk"):
    d = tmp_path / "case"
    if not d.exists():
        shutil.copytree(os.path.join(CASES, case), d)
    p = d / name
    s = p.read_text(encoding="latin-1")
    assert old in s
    p.write_text(s.replace(old, new, 1), encoding="latin-1")
    return str(d)


@pytest.mark.parametrize("name,old,new,message", [
    ("Mesh.dat", "END COORDINATES", "END COORDS", "Expected: End Coordinates"),
    ("Mesh.dat", "MATERIAL ID\n        96", "MATERIAL ID\n        95", "Elements without material were found"),
    ("Mesh.dat", "END CONNECTIVITY", "END CONN", "Expected: End connectivity"),
    ("Mesh.dat", "FIXED SUPPORTS", "LINE LOAD", "Line Load not implemented."),
    ("Mesh.dat", "FIXED SUPPORTS", "SURFACE LOAD", "Surface Load not implemented."),
    ("Mesh.dat", "FIXED SUPPORTS", "EDGE SUPPORTS", "ReadBoundaryConditions::Condition not detected."),
    ("Settings.dat", "Maximum Cut Backs = 10", "", "Analysis Settings :: Option not found [maximumcutbacks]"),
    ("Settings.dat", "Element Technology =  Full Integration", "Element Technology = Selective",
     "Element Technology not identified"),
    ("Settings.dat", "Poisson = 0.3\n", "Poison = 0.3\n", "Option not found [Poisson]"),
    ("Settings.dat", "\tSt_Venant_Kirchhoff", "\tHyperelastic_Tranverse_Isotropic", "Material model not identified"),
    ("Settings.dat", "Preprocessor = Gid 12", "Preprocessor = Gid 13", "Preprocessor not identified"),
    ("Time_Discretization.dat", "Number of Load Cases", "Number of Cases",
     "Expected (Number of Load Cases) in Time Discretization File"),
])
def test_reader_errors_follow_the_reference(tmp_path, name, old, new, message):
    d = _edit(tmp_path, name, old, new)
    with pytest.raises(io.CaseFormatError) as e:
        io.Case(d)
    assert message in str(e.value)


def test_parser_syntax_and_tables(tmp_path):
    assert io.fmt("  Young Modulus = 1 ! comment") == "youngmodulus=1"
    assert io.same("END MESH AND BOUNDARY CONDITIONS", "endmeshandboundaryconditions")
    p = tmp_path / "T.tab"
    p.write_text("! history\nTime\tValue\n0.0e0\t0.0e0\n\n1.0e0\t0.150d0\n2.0\t-1.5D-1 ! tail\n")
    tb = io.read_table(str(p))
    np.testing.assert_array_equal(tb, [[0.0, 0.0], [1.0, 0.15], [2.0, -0.15]])
    assert io.interpolate(tb, 0.5) == (0.075, 1)
    assert io.interpolate(tb, 1.5) == (0.0, 1)
    assert io.interpolate(tb, 2.5)[1] == 0 and io.interpolate(tb, -0.1)[1] == 0
    t = tmp_path / "Time.dat"
    t.write_text("Number of Load Cases\n2\nLoad Case\tInitial Time\tFinal Time\tSteps\n1 0.0 1.0 4\n2 1.0 3.0 2\n")
    assert io.read_time_discretization(str(t)) == [(0.0, 1.0, 4), (1.0, 3.0, 2)]


def test_several_load_cases_become_one_step_sequence(tmp_path):
    d = _edit(tmp_path, "Time_Discretization.dat", "1\t\t\t0.0E0\t\t\t1.0E0\t\t50",
              "1 0.0 0.5 10\n2 0.5 1.0 5")
    _edit(tmp_path, "Time_Discretization.dat", "Number of Load Cases\t\t\t\t\t\t\n1", "Number of Load Cases\n2")
    c = io.Case(d)
    assert len(c.t0) == 15 and c.labels[9] == (1, 10) and c.labels[10] == (2, 1) and c.labels[-1] == (2, 5)
    np.testing.assert_allclose(c.t0[:3], [0.0, 0.05, 0.1])
    np.testing.assert_allclose(c.t0[10:12], [0.5, 0.6])
    np.testing.assert_allclose(c.dt[[0, 14]], [0.05, 0.1])
    # the prescribed values follow the table at the step times of both load cases
    tb = io.read_table(os.path.join(d, "Table_Disp_Z.tab"))
    np.testing.assert_allclose(c.bc["presc_final"][0], np.interp(c.t0 + c.dt, tb[:, 0], tb[:, 1]))


def test_fortran_e_format():
    assert io.fortran_e(1.5) == "  0.150000000000000E+01"
    assert io.fortran_e(-2.5e-7) == " -0.250000000000000E-06"
    assert io.fortran_e(0.0) == "  0.000000000000000E+00"
    assert io.fortran_e(0.02) == "  0.200000000000000E-01"
    assert io.fortran_e(1e100) == "  0.100000000000000+101"
    assert io.fortran_e(9.9999999999999999e-1) == "  0.100000000000000E+01"
    for x in (1.5, -3.25e-12, 123456.789, 0.02):
        assert len(io.fortran_e(x)) == 23 and float(io.fortran_e(x)) == pytest.approx(x, rel=1e-14)


def test_result_file_round_trip(tmp_path):
    rng = np.random.default_rng(3)
    p = str(tmp_path / "FEMAnalysis.result")
    recs = []
    with io.ResultWriter(p, 12) as w:
        for k in range(4):
            U = rng.standard_normal(12) * 10.0 ** rng.integers(-300, 300, 12)
            U[0] = 0.0
            rec = (U, 0.1 * k, 1, k + 1, k % 2, k, k % 2, 3 + k)
            w.record(*rec)
            recs.append(rec)
    with io.ResultWriter(p, 12, append=True) as w:
        w.record(np.ones(12), 1.0, 2, 1, 0, 1, 1, 2)
    n, got = io.read_result(p)
    assert n == 12 and len(got) == 5
    for (U, t, lc, st, cut, sub, flag, nit), r in zip(recs, got):
        np.testing.assert_array_equal(r["U"], U)          # bit for bit
        assert (r["time"], r["load_case"], r["step"], r["cut_back"], r["substep"], r["flag_end_step"],
                r["n_iterations"]) == (t, lc, st, cut, sub, flag, nit)
    assert got[-1]["load_case"] == 2


def test_result_file_in_fortran_list_directed_form(tmp_path):
    """A result file as the reference's list-directed WRITE leaves it."""
    p = tmp_path / "FEMAnalysis.result"
    p.write_text(" Total Number of DOF =          3\n"
                 " TIME =  0.000000000000000E+000\n LOAD CASE =           1\n STEP =           1\n"
                 " CUT BACK =           0\n SUBSTEP =           0\n FLAG END STEP =           1\n"
                 " NUMBER OF ITERATIONS TO CONVERGE =           0\n  0.000000000000000E+000\n"
                 "  0.000000000000000E+000\n  0.000000000000000E+000\n"
                 " TIME =  2.000000000000000E-002\n LOAD CASE =           1\n STEP =           1\n"
                 " CUT BACK =           0\n SUBSTEP =           1\n FLAG END STEP =           1\n"
                 " NUMBER OF ITERATIONS TO CONVERGE =           3\n -1.234567890123457E-003\n"
                 "   1.50000000000000     \n  2.000000000000000E-003\n")
    n, recs = io.read_result(str(p))
    assert n == 3 and len(recs) == 2
    assert recs[1]["time"] == 0.02 and recs[1]["n_iterations"] == 3 and recs[1]["substep"] == 1
    np.testing.assert_array_equal(recs[1]["U"], [-1.234567890123457e-3, 1.5, 2e-3])


def test_checker(tmp_path):
    marc = os.path.join(CASES, "hexa8_svk", "marc_disp_x.dat")
    log = str(tmp_path / "Log_CHECKER.txt")
    assert io.check(marc, marc, 1e-5, log) == (True, "SUCCESS")
    rows = [ln for ln in open(marc, encoding="latin-1") if ln.strip()]
    t, v = rows[20].split()[:2]
    bad = tmp_path / "bad.probe"
    bad.write_text("".join(rows[:20]) + f" {t} {float(v) + 2e-5}\n" + "".join(rows[21:]))
    ok, msg = io.check(str(bad), marc, 1e-5, log)
    assert not ok and "second column" in msg
    assert io.check(str(bad), marc, 1e-4)[0]
    assert "SUCCESS" in open(log).read() and "greater than the tolerance" in open(log).read()


def _probe_rows(path):
    return [ln for ln in open(path) if ln.strip()]


class _View:
    def __init__(self, case, time, U):
        self.case, self.time, self.U = case, time, U


def test_oracle_curves_through_probes_pass_the_checker(tmp_path, golden):
    """The reference's Run_Checker.bat on probe files written by NodeProbe from the FP64 oracle's
    analysis of the St Venant case: the probe and Checker formats close the loop on real numbers."""
    c = io.Case(os.path.join(CASES, "hexa8_svk"))
    m = O.Model(c.mesh["X"], c.mesh["conn"], [O.SVK], c.params)
    dofs = [3 * 10 + d + 1 for d in range(3)]
    r = m.analysis(c.bc, tol=1e-3, itmax=10, norm_mode=1, probe_dofs=dofs)
    assert r["rc"] == 0
    probes = io.read_probes(os.path.join(CASES, "hexa8_svk", "Post_Processing.post"))
    for p in probes:
        p.initialize(str(tmp_path))
    times = [0.0] + list(c.t0 + c.dt)
    for k, t in enumerate(times):
        U = np.zeros(c.n_dof)
        if k:
            U[np.array(dofs) - 1] = r["probe"][:, k - 1]
        for p in probes:
            p.write(_View(c, t, U))
    for comp in "XYZ":
        f1 = str(tmp_path / f"CEOS_Disp_{comp}.probe")
        assert len(_probe_rows(f1)) == 52
        f2 = os.path.join(CASES, "hexa8_svk", f"marc_disp_{comp.lower()}.dat")
        assert io.check(f1, f2, 1e-5) == (True, "SUCCESS"), comp


class _ScriptedLoop:
    """Stands in for ElementLoop: analysis emits a scripted record sequence (one cut back in step
    2), evaluate/commit are logged."""

    def __init__(self, n_dof):
        self.n_dof, self.n_elem, self.log = n_dof, 1, []

    def analysis(self, bc, tol, itmax, norm_mode, norm_type, max_cutbacks, on_step=None, U0=None):
        self.log.append(("analysis", len(bc["t0"]), None if U0 is None else float(U0[0])))
        U = np.zeros(self.n_dof) if U0 is None else np.array(U0)
        for s in range(len(bc["t0"])):
            t0, dt = bc["t0"][s], bc["dt"][s]
            if s == 1:  # cut back, then substeps alpha = 0.382, 1
                a = 1 - 1 / ((1 + 5 ** 0.5) / 2)
                U = U + a
                on_step(t0 + a * dt, 1, s + 1, 1, 2, 0, 4, U)
            U = U + 1.0
            on_step(t0 + dt, 1, s + 1, 1 if s == 1 else 0, 3 if s == 1 else 1, 1, 2, U)
        return {"rc": 0}

    def evaluate(self, time, U, tangent=True, raise_on_error=False):
        self.log.append(("evaluate", time, float(U[0])))
        return None, None, 0, 0

    def commit(self):
        self.log.append(("commit",))

    def set_committed_time(self, t):
        self.log.append(("time", t))

    def store_stress(self, on=True):
        pass

    def close(self):
        pass


def test_case_driver_record_order(tmp_path):
    """Result records (initial record, substeps with Flag_EndStep 0, end steps), the post-processor's
    evaluate / probe / commit order, and the restart's replay of end-step records only."""
    c = io.Case(os.path.join(CASES, "hexa8_svk"))
    out = str(tmp_path)
    loop = _ScriptedLoop(c.n_dof)
    c.run(out, loop=loop, n_steps=3)
    n, recs = io.read_result(os.path.join(out, "FEMAnalysis.result"))
    assert n == c.n_dof
    assert [(r["step"], r["cut_back"], r["substep"], r["flag_end_step"]) for r in recs] == [
        (1, 0, 0, 1), (1, 0, 1, 1), (2, 1, 2, 0), (2, 1, 3, 1), (3, 0, 1, 1)]
    assert recs[0]["time"] == 0.0 and recs[1]["time"] == pytest.approx(0.02) and recs[3]["U"][0] == pytest.approx(
        2.0 + 1 - 1 / ((1 + 5 ** 0.5) / 2))
    # post-processing: every record evaluated and committed, probes written at end steps only
    loop.log.clear()
    files = c.post_process(out, loop=loop)
    ev = [e for e in loop.log if e[0] == "evaluate"]
    assert len(ev) == 5 and loop.log.count(("commit",)) == 5
    assert loop.log[:3] == [("evaluate", 0.0, 0.0), ("commit",), ("time", 0.0)]
    rows = _probe_rows(files[0])
    assert len(rows) == 1 + 4 and rows[0] == "  Time                    Value\n"
    assert rows[3].startswith(io.fortran_e(recs[3]["time"]))
    its = _probe_rows(files[-1])
    assert len(its) == 5 and its[3].split()[1] == "2"
    # restart: replays the four end-step records, continues from step 4 with the last U, appends
    loop.log.clear()
    r = c.restart(out, loop=loop)
    assert r["first_step"] == 3
    assert [e for e in loop.log if e[0] == "evaluate"] == [("evaluate", rec["time"], rec["U"][0])
                                                           for rec in recs if rec["flag_end_step"] == 1]
    an = [e for e in loop.log if e[0] == "analysis"][0]
    assert an == ("analysis", 47, recs[-1]["U"][0])
    n, recs2 = io.read_result(os.path.join(out, "FEMAnalysis.result"))
    assert len(recs2) == 5 + 47 + 1 and recs2[5]["step"] == 4 and recs2[-1]["step"] == 50
    # a second restart finds the analysis complete
    assert c.restart(out, loop=loop)["steps_run"] == 0


def test_restart_across_a_load_case_boundary(tmp_path):
    """Two load cases (10 + 5 steps): an analysis stopped after the last step of load case 1 restarts at
    (load case 2, step 1) with the U of that record, and its records carry the load-case labels."""
    d = _edit(tmp_path, "Time_Discretization.dat", "1\t\t\t0.0E0\t\t\t1.0E0\t\t50",
              "1 0.0 0.5 10\n2 0.5 1.0 5")
    _edit(tmp_path, "Time_Discretization.dat", "Number of Load Cases\t\t\t\t\t\t\n1", "Number of Load Cases\n2")
    c = io.Case(d)
    out = str(tmp_path)
    loop = _ScriptedLoop(c.n_dof)
    c.run(out, loop=loop, n_steps=10)
    _, recs = io.read_result(os.path.join(out, "FEMAnalysis.result"))
    assert (recs[-1]["load_case"], recs[-1]["step"]) == (1, 10)
    loop.log.clear()
    r = c.restart(out, loop=loop)
    assert r["first_step"] == 10
    an = [e for e in loop.log if e[0] == "analysis"][0]
    assert an == ("analysis", 5, recs[-1]["U"][0])
    _, recs2 = io.read_result(os.path.join(out, "FEMAnalysis.result"))
    new = recs2[len(recs):]
    ends = [(x["load_case"], x["step"]) for x in new if x["flag_end_step"] == 1]
    assert ends == [(2, s) for s in range(1, 6)]
    assert new[0]["time"] == pytest.approx(0.6)                       # end of (2, 1)
    # the scripted cut back in the call's second step: a substep record of (2, 2) with Flag_EndStep 0
    assert (new[1]["load_case"], new[1]["step"], new[1]["flag_end_step"]) == (2, 2, 0)
    assert new[1]["time"] == pytest.approx(0.6 + 0.1 * (1 - 1 / ((1 + 5 ** 0.5) / 2)))


def test_probe_error_lines_follow_the_reference(tmp_path):
    """ModProbe's error lines: a node beyond the mesh, a component beyond the node's dofs, a variable a
    node does not carry; the probe then stops writing (its Active flag)."""
    c = io.Case(os.path.join(CASES, "hexa8_svk"))
    probes = [io.NodeProbe("far.probe", "Displacements", 10 ** 6, "1"),
              io.NodeProbe("comp.probe", "Displacements", 11, "4"),
              io.NodeProbe("var.probe", "Cauchy Stress", 11, "1"),
              io.NodeProbe("all.probe", "Displacements", 11, "All")]
    for p in probes:
        p.initialize(str(tmp_path))
    U = np.arange(c.n_dof, dtype=float)
    for t in (0.1, 0.2):
        for p in probes:
            p.write(_View(c, t, U))
    lines = {p.file_name: open(tmp_path / p.file_name).read().splitlines() for p in probes}
    assert lines["far.probe"][1:] == ["ERROR - Node Number is greater than the Max Number of Nodes in the Mesh"]
    assert lines["comp.probe"][1:] == ["ERROR: Component is greater than the available"]
    assert lines["var.probe"][1:] == ["ERROR: Variable not available"]
    rows = [list(map(float, ln.split())) for ln in lines["all.probe"][1:]]
    assert rows == [[0.1, 30.0, 31.0, 32.0], [0.2, 30.0, 31.0, 32.0]]
