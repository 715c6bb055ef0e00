"""Case files of the reference's FEM program, read and written on the host around the GPU analysis.

The reference runs a case from a directory of text files and leaves its results in text files; this
module reads and writes the same files so that a case directory of the reference runs unchanged on
the GPU element loop (ElementLoop.analysis, the C ABI's ceos_analysis):

- Settings.dat: ReadInputFile and its block readers (FEM/Input/ModReadInputFile.f90:32-433,
  798-904), with the option syntax of Tools/ModParser.f90 (case-insensitive, blanks ignored, "!"
  starts a comment, "name = value", FormatString :229-236);
- the GiD mesh and its BOUNDARY CONDITIONS block: ReadMeshGiD and ReadBoundaryConditionsGiD
  (ModReadInputFile.f90:1396-1709);
- the time discretization and the load-history tables: ReadTimeDiscretization and
  ReadValueDiscretization (FEM/BoundaryConditions/ModLoadHistoryData.f90:43-225);
- FEMAnalysis.result: the header line and WriteFEMResults (FEM/ModFEMAnalysis.f90:1094-1129, 1188,
  1211, 1314-1337), read back as RestartAnalysis and the post-processor read it (:2827-2956);
- restart: RestartAnalysis's replay of the converged steps, then the remaining steps;
- post-processing: the replay of every record with probe output (FEM/PostProcessing/
  ModExportResultFile.f90:290-420) and the node and Gauss-point probes (ModProbe.f90:148-563);
- the Checker that compares two-column result files (Checker/Checker Code/Checker/Checker.f90).

Supported constitutive models are those of the GPU element loop (see MODELS); a case that names
another model, another element type or a load the reference does not implement raises
CaseFormatError with the reference's message.
"""
import math
import os

import numpy as np

from . import CNH, FP64, J2_SMALL, NH_Q1P0, SVK, VISCO_VAR, ElementLoop

# (reference model name, element technology) -> (model id, option names in the order of the
# model's ReadMaterialParameters); ModConstitutiveModelLibrary.f90:492-552 selects by both.
MODELS = {
    ("st_venant_kirchhoff", "fullintegration"): (SVK, ["YoungModulus", "Poisson"]),
    ("compressible_neo_hookean", "fullintegration"): (CNH, ["Mu", "Lambda"]),
    ("j2_plasticity", "fullintegration"): (J2_SMALL, ["YoungModulus", "Poisson", "YieldStress",
                                                      "HardeningModulus"]),
    ("neo_hookean", "meandilatation"): (NH_Q1P0, ["C10", "BulkModulus"]),
    ("matrix_viscoelastic", "fullintegration"): (VISCO_VAR, ["K_inf", "Mu_inf", "Lambda_inf", "K_e", "Mu_e",
                                                             "Ni_v"]),
}


class CaseFormatError(ValueError):
    """A case file the reference's reader would reject (its RaiseError / Error / stop message)."""


def fmt(s):
    """Parser FormatString (ModParser.f90:229-236): lower case, comment removed, blanks removed."""
    s = s.split("!", 1)[0]
    return "".join(s.lower().split())


def same(a, b):
    """Parser CompareStrings."""
    return fmt(a) == fmt(b)


def _number(s):
    """A Fortran real literal (list-directed read): d/D exponents accepted."""
    return float(s.strip().replace("d", "e").replace("D", "E"))


class _Lines:
    """The valid lines of a file in order, as GetNextString walks them: comments and blank lines are
    skipped; each item keeps the original text (GetOriginalLine) and its formatted form."""

    def __init__(self, path):
        self.path = path
        with open(path, "r", encoding="latin-1") as f:
            raw = [ln.rstrip("\r\n") for ln in f]
        self.items = [(ln.split("!", 1)[0].strip(), fmt(ln)) for ln in raw if fmt(ln)]
        self.i = 0

    def eof(self):
        return self.i >= len(self.items)

    def next(self, what="a line"):
        if self.eof():
            raise CaseFormatError(f"{os.path.basename(self.path)}: end of file while expecting {what}")
        self.i += 1
        return self.items[self.i - 1]

    def peek(self):
        return None if self.eof() else self.items[self.i]

    def option(self, what="an option"):
        """GetNextOption: 'name = value' (name formatted, value as written)."""
        orig, f = self.next(what)
        if "=" not in orig:
            raise CaseFormatError(f"{os.path.basename(self.path)}: expected {what}, found [{orig}]")
        name, value = orig.split("=", 1)
        return fmt(name), value.strip()

    def expect(self, text, message):
        orig, f = self.next(text)
        if f != fmt(text):
            raise CaseFormatError(message)


def find_file(case_dir, name):
    """A file of the case directory; names match case-insensitively, as on the file system the
    reference's cases were written for."""
    p = os.path.join(case_dir, name)
    if os.path.exists(p):
        return p
    want = name.lower()
    for f in os.listdir(case_dir):
        if f.lower() == want:
            return os.path.join(case_dir, f)
    raise CaseFormatError(f"file {name} not found in {case_dir}")


# ---------------------------------------------------------------------------------------------
# Settings.dat
# ---------------------------------------------------------------------------------------------

_ANALYSIS_REQUIRED = ["problemtype", "analysistype", "nonlinearanalysis", "hypothesisofanalysis",
                      "elementtechnology", "maximumcutbacks", "multiscaleanalysis"]


def read_settings(path):
    """Settings.dat (ReadInputFile, ModReadInputFile.f90:32-146).  Returns a dict with the blocks
    the element loop needs: analysis settings, nonlinear solver (tol, maxiter), materials (id,
    model name, options) and the mesh/time file names.  "Multiscale Model" and "Restart" of
    ReadAnalysisSettings (:170-313) default to Taylor and False when absent: the reference's own
    checker cases were written before those two options existed."""
    L = _Lines(path)
    out = {"analysis": None, "linear_solver": None, "nonlinear_solver": None, "materials": None,
           "mesh_and_bc": None}
    while not L.eof():
        orig, f = L.next()
        if f == "analysissettings":
            opts = {}
            while L.peek() is not None and L.peek()[1] != "endanalysissettings":
                name, value = L.option("an Analysis Settings option")
                opts[name] = value
            L.expect("end analysis settings", "End of block was expected. BlockName=Analysis Settings")
            for k in _ANALYSIS_REQUIRED:
                if k not in opts:
                    raise CaseFormatError(f"Analysis Settings :: Option not found [{k}]")
            a = {"problem_type": fmt(opts["problemtype"]), "analysis_type": fmt(opts["analysistype"]),
                 "nonlinear": fmt(opts["nonlinearanalysis"]) == "true",
                 "hypothesis": fmt(opts["hypothesisofanalysis"]),
                 "element_technology": fmt(opts["elementtechnology"]),
                 "max_cutbacks": int(_number(opts["maximumcutbacks"])),
                 "multiscale": fmt(opts["multiscaleanalysis"]) == "true",
                 "multiscale_model": fmt(opts.get("multiscalemodel", "taylor")),
                 "restart": fmt(opts.get("restart", "false")) == "true"}
            if a["problem_type"] not in ("mechanical", "thermal"):
                raise CaseFormatError("Problem Type not identified")
            if a["element_technology"] not in ("fullintegration", "reducedintegration", "meandilatation"):
                raise CaseFormatError("Element Technology not identified")
            out["analysis"] = a
        elif f == "linearsolver":
            out["linear_solver"] = L.next("a linear solver")[1]
            L.expect("end linear solver", "End of block was expected. BlockName=Linear Solver")
        elif f == "nonlinearsolver":
            if out["linear_solver"] is None:
                raise CaseFormatError("Linear Solver must be specified before the NonLinear solver")
            name = L.next("a nonlinear solver")[1]
            # NewtonRaphsonFull_ReadSolverParameters (ModNewtonRaphsonFull.f90:172-201): two options
            opts = dict(L.option("a solver option") for _ in range(2))
            for k in ("tol", "maxiter"):
                if k not in opts:
                    raise CaseFormatError(f"Nonlinear solver :: Option not found [{k}]")
            out["nonlinear_solver"] = {"name": name, "tol": _number(opts["tol"]),
                                       "maxiter": int(_number(opts["maxiter"]))}
            L.expect("end nonlinear solver", "End of block was expected. BlockName=NonLinear Solver")
        elif f == "material":
            if out["analysis"] is None:
                raise CaseFormatError("Analysis Settings must be specified before the material.")
            out["materials"] = _read_materials(L, out["analysis"]["element_technology"])
        elif f == "meshandboundaryconditions":
            if out["analysis"] is None or out["materials"] is None:
                raise CaseFormatError("Analysis Settings and Material must be specified before mesh.")
            opts = {}
            while L.peek() is not None and L.peek()[1] != "endmeshandboundaryconditions":
                name, value = L.option("a Mesh and Boundary Conditions option")
                opts[name] = value
            L.expect("end mesh and boundary conditions",
                     "End of block was expected. BlockName=Mesh and Boundary Conditions")
            if "meshfile" not in opts:
                raise CaseFormatError("MESH AND BOUNDARY CONDITIONS :: Mesh File was not found")
            if "timediscretizationfile" not in opts:
                raise CaseFormatError("MESH AND BOUNDARY CONDITIONS :: Time Discretization File was not found")
            if "preprocessor" not in opts:
                raise CaseFormatError("MESH AND BOUNDARY CONDITIONS :: Preprocessor was not found")
            pre = fmt(opts["preprocessor"])
            if pre not in ("gid7", "gid12", "hypermesh"):
                raise CaseFormatError("Preprocessor not identified")
            out["mesh_and_bc"] = {"mesh_file": opts["meshfile"], "time_file": opts["timediscretizationfile"],
                                  "preprocessor": pre}
        else:
            # blocks this path does not use (MULTISCALE SETTINGS, MACROSCOPIC DEFORMATION GRADIENT, ...)
            end = "end" + f
            while L.peek() is not None and L.peek()[1] != end:
                L.next()
            if L.peek() is None:
                raise CaseFormatError(f"End of block was expected. BlockName={orig}")
            L.next()
    for k, name in (("analysis", "Analysis Settings"), ("linear_solver", "Linear Solver"),
                    ("nonlinear_solver", "NonLinear Solver"), ("materials", "Material"),
                    ("mesh_and_bc", "Mesh and Boundary Conditions")):
        if out[k] is None:
            raise CaseFormatError(f"Block [{name}] was not detected!")
    return out


def _read_materials(L, element_technology):
    """ReadMaterialModel (ModReadInputFile.f90:827-904): Number of Materials, then per material its
    ID, the model name and the model's options (FillListOfOptions reads as many option lines as the
    model has options)."""
    name, value = L.option("Number of Materials")
    if name != "numberofmaterials":
        raise CaseFormatError("Expected Number of Materials")
    mats = []
    for _ in range(int(_number(value))):
        name, value = L.option("Material ID")
        if name != "materialid":
            raise CaseFormatError("Expected Material ID")
        mid = int(_number(value))
        model_name = L.next("a model name")[1]
        key = (model_name, element_technology)
        if key not in MODELS:
            raise CaseFormatError(f"Material model not identified or not available on this path: [{model_name}]"
                                  f" with element technology [{element_technology}]")
        model, names = MODELS[key]
        opts = dict(L.option("a material option") for _ in names)
        params = []
        for n in names:
            if fmt(n) not in opts:
                raise CaseFormatError(f"ReadMaterialParameters :: Option not found [{n}]")
            params.append(_number(opts[fmt(n)]))
        mats.append({"id": mid, "name": model_name, "model": model, "params": params})
    L.expect("end material", "End of block was expected. BlockName=Material")
    return mats


# ---------------------------------------------------------------------------------------------
# GiD mesh, boundary conditions, time discretization, tables
# ---------------------------------------------------------------------------------------------

def read_mesh_gid(path):
    """MESH block (ReadMeshGiD, ModReadInputFile.f90:1396-1561) and BOUNDARY CONDITIONS block
    (ReadBoundaryConditionsGiD, :1565-1709) of a GiD mesh file.  Returns X [n_nodes,3], conn
    [n_elem,8] (1-based, the file's node order), mat [n_elem] (material IDs), fixed [[node, fx, fy,
    fz]], loads and disps [[node, (flag, table), (flag, table), (flag, table)]]."""
    L = _Lines(path)
    L.next("MESH")
    dims = {}
    for _ in range(3):
        name, value = L.option("Nnodes, Nelem or Ndime")
        if name not in ("nnodes", "nelem", "ndime"):
            raise CaseFormatError("Expected Nnodes,Nelem or Ndime")
        dims[name] = int(_number(value))
        if dims[name] <= 0:
            raise CaseFormatError({"nnodes": "Nnodes", "nelem": "Nelem", "ndime": "Ndime"}[name] +
                                  " must be positive")
    nn, ne, nd = dims.get("nnodes"), dims.get("nelem"), dims.get("ndime")
    if nd != 3:
        raise CaseFormatError("only three-dimensional meshes (Ndime = 3) run on this path")
    L.expect("Coordinates", "Coordinates were not found")
    X = np.zeros((nn, 3))
    for _ in range(nn):
        t = L.next("a node")[0].split()
        X[int(t[0]) - 1] = [_number(v) for v in t[1:4]]
    L.expect("end coordinates", "Expected: End Coordinates")
    L.expect("MATERIAL ID", "MATERIAL ID was not found")
    if int(_number(L.next("the number of material IDs")[0])) != ne:
        raise CaseFormatError("Elements without material were found")
    mat = np.zeros(ne, np.int32)
    for _ in range(ne):
        t = L.next("a material ID")[0].split()
        mat[int(t[0]) - 1] = int(t[1])
    L.expect("end material id", "Expected: End Material ID")
    L.expect("CONNECTIVITY", "CONNECTIVITY was not found")
    conn = np.zeros((ne, 8), np.int32)
    for _ in range(ne):
        t = [int(v) for v in L.next("an element")[0].split()]
        eid, geo, enn = t[0], t[1], t[2]
        if enn != 8:  # ElementIdentifier: Hexa8 is the element of this path
            raise CaseFormatError(f"element {eid}: {enn} nodes; only Hexa8 elements run on this path")
        conn[eid - 1] = t[3:3 + enn]
    L.expect("end connectivity", "Expected: End connectivity")
    L.expect("end mesh", "End of block was expected. BlockName=MESH")
    # BOUNDARY CONDITIONS
    L.next("BOUNDARY CONDITIONS")
    fixed, loads, disps = [], [], []
    while True:
        orig, f = L.next("a boundary condition")
        if f == "fixedsupports":
            n = int(_number(L.next("the number of fixed supports")[0]))
            for _ in range(n):
                fixed.append([int(v) for v in L.next("a fixed support")[0].split()[:4]])
        elif f in ("nodalload", "nodaldisplacement"):
            n = int(_number(L.next("the number of nodal conditions")[0]))
            rows = []
            for _ in range(n):
                t = L.next("a nodal condition")[0].split()
                rows.append([int(t[0])] + [(int(t[1 + 2 * d]), t[2 + 2 * d]) for d in range(3)])
            (loads if f == "nodalload" else disps).extend(rows)
        elif f == "lineload":
            raise CaseFormatError("Line Load not implemented.")
        elif f == "surfaceload":
            raise CaseFormatError("Surface Load not implemented.")
        elif f == "loadcases":
            pass
        elif f == "endboundaryconditions":
            break
        else:
            raise CaseFormatError("ReadBoundaryConditions::Condition not detected.")
    return {"X": X, "conn": conn, "mat": mat, "fixed": fixed, "loads": loads, "disps": disps}


def read_time_discretization(path):
    """ReadTimeDiscretization (ModLoadHistoryData.f90:43-105): per load case (t0, t1, steps); the
    steps of a load case are equal, InitTime = t0 + (n-1) dt."""
    L = _Lines(path)
    if L.next()[1] != fmt("Number of Load Cases"):
        raise CaseFormatError("Expected (Number of Load Cases) in Time Discretization File")
    n_lc = int(_number(L.next()[0]))
    if L.next()[1] != fmt("Load Case Initial Time Final Time Steps"):
        raise CaseFormatError("Expected (Load Case\tInitial Time\tFinal Time\tSteps Time) in Time Discretization File")
    cases = []
    for _ in range(n_lc):
        t = L.next("a load case")[0].split()
        cases.append((_number(t[1]), _number(t[2]), int(_number(t[3]))))
    return cases


def read_table(path):
    """ReadValueDiscretization (ModLoadHistoryData.f90:122-225): (time, value) rows; the
    'Time Value' header line is skipped wherever it stands."""
    rows = []
    for orig, f in _Lines(path).items:
        if f == fmt("Time Value"):
            continue
        t = orig.split()
        rows.append((_number(t[0]), _number(t[1])))
    return np.array(rows, dtype=np.float64).reshape(-1, 2)


def interpolate(table, t):
    """LinearInterpolation of a load-history table; flag 0 outside the table's time range (the step
    is then inactive in the reference)."""
    tt, vv = table[:, 0], table[:, 1]
    if t < tt[0] - 1e-12 * max(1.0, abs(tt[0])) or t > tt[-1] + 1e-12 * max(1.0, abs(tt[-1])):
        return 0.0, 0
    return float(np.interp(t, tt, vv)), 1


def _table_file(name):
    """The reference appends .tab to a table name without an extension (:135-140)."""
    return name if "." in name else name + ".tab"


# ---------------------------------------------------------------------------------------------
# A case directory
# ---------------------------------------------------------------------------------------------

class Case:
    """A case directory of the reference (Settings.dat, the mesh file, the time discretization,
    the tables and Post_Processing.post) on the GPU element loop."""

    def __init__(self, case_dir, settings="Settings.dat"):
        self.dir = case_dir
        self.settings = read_settings(find_file(case_dir, settings))
        a = self.settings["analysis"]
        if a["problem_type"] != "mechanical" or a["analysis_type"] != "quasistatic":
            raise CaseFormatError("only mechanical quasi-static analyses run on this path")
        if a["hypothesis"] != "3d":
            raise CaseFormatError("only 3D analyses run on this path")
        if a["multiscale"]:
            raise CaseFormatError("multiscale cases run through ceos_b200.fe2, not the case driver")
        mb = self.settings["mesh_and_bc"]
        if mb["preprocessor"] == "hypermesh":
            raise CaseFormatError("HyperMesh meshes are not read on this path (GiD 7 and GiD 12 are)")
        self.mesh = read_mesh_gid(find_file(case_dir, mb["mesh_file"]))
        self.load_cases = read_time_discretization(find_file(case_dir, mb["time_file"]))
        mats = self.settings["materials"]
        models = {m["model"] for m in mats}
        if len(models) != 1:
            raise CaseFormatError("the GPU element loop runs one constitutive model per mesh")
        self.model = models.pop()
        index = {m["id"]: k for k, m in enumerate(mats)}
        missing = set(self.mesh["mat"].tolist()) - set(index)
        if missing:
            raise CaseFormatError("Element's Material was not found")
        self.mat_index = np.array([index[m] for m in self.mesh["mat"]], np.int32)
        self.params = [m["params"] for m in mats]
        self._steps()
        self._bc()

    @property
    def n_dof(self):
        return 3 * len(self.mesh["X"])

    def _steps(self):
        """Steps of all load cases in sequence: (load case, step) labels, InitTime and DeltaTime."""
        self.labels, t0, dt = [], [], []
        for lc, (ti, tf, n) in enumerate(self.load_cases, start=1):
            d = (tf - ti) / float(n)
            for s in range(1, n + 1):
                self.labels.append((lc, s))
                t0.append(ti + (s - 1) * d)
                dt.append(d)
        self.t0, self.dt = np.array(t0), np.array(dt)

    def _bc(self):
        """Per-dof prescribed values at the start and end of every step (GetBoundaryConditions,
        ModBoundaryConditions.f90:540-668, from the tables of CreateNodalBoundaryCondition)."""
        tables = {}

        def table(name):
            if name not in tables:
                tables[name] = read_table(find_file(self.dir, _table_file(name)))
            return tables[name]

        fixed = sorted({3 * (r[0] - 1) + d + 1 for r in self.mesh["fixed"] for d in range(3) if r[1 + d]})
        t1 = self.t0 + self.dt

        def expand(rows):
            dofs, vi, vf = [], [], []
            for r in rows:
                for d in range(3):
                    flag, name = r[1 + d]
                    if flag:
                        tb = table(name)
                        dofs.append(3 * (r[0] - 1) + d + 1)
                        vi.append([interpolate(tb, t)[0] for t in self.t0])
                        vf.append([interpolate(tb, t)[0] for t in t1])
            n = len(self.t0)
            return (np.asarray(dofs, np.int32), np.asarray(vi, np.float64).reshape(-1, n),
                    np.asarray(vf, np.float64).reshape(-1, n))

        presc, pi, pf = expand(self.mesh["disps"])
        force, fi, ff = expand(self.mesh["loads"])
        self.bc = {"t0": self.t0, "dt": self.dt, "fixed": np.asarray(fixed, np.int32), "presc": presc,
                   "presc_init": pi, "presc_final": pf, "force": force, "force_init": fi, "force_final": ff}

    def element_loop(self, precision=FP64, device=0):
        return ElementLoop(self.mesh["X"], self.mesh["conn"], self.model, self.params, mat_id=self.mat_index,
                           precision=precision, device=device)

    def _slice_bc(self, first, last=None):
        """The boundary conditions of steps [first, last)."""
        b = dict(self.bc)
        for k in ("t0", "dt"):
            b[k] = self.bc[k][first:last]
        for k in ("presc_init", "presc_final", "force_init", "force_final"):
            b[k] = self.bc[k][:, first:last]
        return b

    def run(self, out_dir, precision=FP64, norm_mode=1, norm_type=2, n_steps=None, loop=None, tol=None):
        """The quasi-static analysis of the case (QuasiStaticAnalysisFEM, ModFEMAnalysis.f90:1136-1374)
        on the GPU, writing out_dir/FEMAnalysis.result as the reference does.  norm_mode 1 is the
        absolute residual criterion of the version that produced the reference's checker logs
        (0: relative, the current source); tol overrides the case's Newton tolerance.  n_steps stops
        after that many steps (for a restart).  Returns the analysis result of ElementLoop.analysis plus the result file's path."""
        own = loop is None
        loop = loop if loop is not None else self.element_loop(precision)
        ns = self.settings["nonlinear_solver"]
        path = os.path.join(out_dir, "FEMAnalysis.result")
        bc = self._slice_bc(0, n_steps)
        try:
            with ResultWriter(path, self.n_dof) as w:
                w.record(np.zeros(self.n_dof), 0.0, 1, 1, 0, 0, 1, 0)
                r = loop.analysis(bc, ns["tol"] if tol is None else tol, ns["maxiter"], norm_mode, norm_type,
                                  self.settings["analysis"]["max_cutbacks"],
                                  on_step=self._writer_callback(w, 0))
        finally:
            if own:
                loop.close()
        r["result_file"] = path
        return r

    def _writer_callback(self, w, first):
        def on_step(time, lc, st, cutback, substep, flag_end, n_iter, U):
            lc_, st_ = self.labels[first + st - 1]
            w.record(U, time, lc_, st_, cutback, substep, flag_end, n_iter)
            return False
        return on_step

    def restart(self, out_dir, precision=FP64, norm_mode=1, norm_type=2, loop=None, tol=None):
        """Continue the analysis from out_dir/FEMAnalysis.result (RestartAnalysis, ModFEMAnalysis.f90:
        2827-2956, and the restart branch of :1436-1512): every record with Flag_EndStep = 1 is
        replayed in order (Gauss-point update at its U and time, then SwitchConvergedState), the
        analysis continues from the step after the last replayed one with that U, and its records
        are appended to the same file."""
        own = loop is None
        loop = loop if loop is not None else self.element_loop(precision)
        path = os.path.join(out_dir, "FEMAnalysis.result")
        try:
            n_dof, records = read_result(path)
            if n_dof != self.n_dof:
                raise CaseFormatError(f"FEMAnalysis.result holds {n_dof} dofs, the mesh {self.n_dof}")
            last, U = None, np.zeros(self.n_dof)
            for rec in records:
                if rec["flag_end_step"] != 1:
                    continue
                U = rec["U"]
                last = (rec["load_case"], rec["step"])
                loop.evaluate(rec["time"], U, tangent=False, raise_on_error=True)
                loop.commit()
                loop.set_committed_time(rec["time"])
            first = 0 if last is None or last == (1, 1) and not np.any(U) else self.labels.index(last) + 1
            if first >= len(self.t0):
                return {"rc": 0, "steps_run": 0, "result_file": path}
            ns = self.settings["nonlinear_solver"]
            with ResultWriter(path, self.n_dof, append=True) as w:
                r = loop.analysis(self._slice_bc(first), ns["tol"] if tol is None else tol, ns["maxiter"], norm_mode,
                                  norm_type,
                                  self.settings["analysis"]["max_cutbacks"],
                                  on_step=self._writer_callback(w, first), U0=U)
        finally:
            if own:
                loop.close()
        r["result_file"] = path
        r["first_step"] = first
        return r

    def post_process(self, out_dir, probes="Post_Processing.post", precision=FP64, loop=None):
        """Replay FEMAnalysis.result with the case's probes (ModExportResultFile.f90:290-420): the
        Gauss-point state is rebuilt from scratch, every record is evaluated at its U and time and
        then committed; records with Flag_EndStep = 1 write the probes and a line of
        NumberOfIterationsToConverge.dat.  Returns the written file paths."""
        plist = read_probes(find_file(self.dir, probes)) if isinstance(probes, str) else probes
        own = loop is None
        loop = loop if loop is not None else self.element_loop(precision)
        written = []
        try:
            for p in plist:
                p.initialize(out_dir)
                written.append(p.path)
            it_path = os.path.join(out_dir, "NumberOfIterationsToConverge.dat")
            written.append(it_path)
            need_gp = any(isinstance(p, GaussPointProbe) for p in plist)
            if need_gp:
                loop.store_stress(True)
            n_dof, records = read_result(os.path.join(out_dir, "FEMAnalysis.result"))
            with open(it_path, "w") as itf:
                itf.write("   Time                    Number Of Iterations To Converge\n")
                for rec in records:
                    U = rec["U"]
                    loop.evaluate(rec["time"], U, tangent=False)
                    if rec["flag_end_step"] == 1:
                        view = _StepView(self, loop, rec, need_gp)
                        for p in plist:
                            p.write(view)
                        itf.write(f" {fortran_e(rec['time'], 23, 15)} {rec['n_iterations']:11d}\n")
                    loop.commit()
                    loop.set_committed_time(rec["time"])
        finally:
            if own:
                loop.close()
        return written


# ---------------------------------------------------------------------------------------------
# FEMAnalysis.result
# ---------------------------------------------------------------------------------------------

class ResultWriter:
    """FEMAnalysis.result: 'Total Number of DOF = n', then per converged substep the seven option
    lines of WriteFEMResults and U one value per line.  Values are written with 17 significant
    digits, so a read-back restart sees the same U bit for bit."""

    def __init__(self, path, n_dof, append=False):
        self.f = open(path, "a" if append else "w")
        if not append:
            self.f.write(f" Total Number of DOF =  {n_dof:11d}\n")

    def record(self, U, time, lc, st, cutback, substep, flag_end, n_iter):
        w = self.f.write
        w(f" TIME = {time:25.17E}\n LOAD CASE = {lc:11d}\n STEP = {st:11d}\n CUT BACK = {cutback:11d}\n"
          f" SUBSTEP = {substep:11d}\n FLAG END STEP = {flag_end:11d}\n"
          f" NUMBER OF ITERATIONS TO CONVERGE = {n_iter:11d}\n")
        w("".join(f" {u:25.17E}\n" for u in np.asarray(U, np.float64)))

    def close(self):
        self.f.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


_RECORD_KEYS = [("time", float), ("load_case", int), ("step", int), ("cut_back", int), ("substep", int),
                ("flag_end_step", int), ("n_iterations", int)]


def read_result(path):
    """(n_dof, records) of a FEMAnalysis.result written by the reference or by ResultWriter; records
    is a list of dicts with time, load_case, step, cut_back, substep, flag_end_step, n_iterations and
    U (the reader of RestartAnalysis and of the post-processor, ModFEMAnalysis.f90:2866-2950)."""
    L = _Lines(path)
    name, value = L.option("Total Number of DOF")
    n_dof = int(_number(value))
    records = []
    while not L.eof():
        rec = {}
        for key, cast in _RECORD_KEYS:
            name, value = L.option(key)
            rec[key] = cast(_number(value)) if cast is float else int(round(_number(value)))
        U = np.empty(n_dof)
        for i in range(n_dof):
            U[i] = _number(L.next("a displacement")[0])
        rec["U"] = U
        records.append(rec)
    return n_dof, records


# ---------------------------------------------------------------------------------------------
# Probes
# ---------------------------------------------------------------------------------------------

def fortran_e(x, w=23, d=15):
    """Fortran Ew.d edit descriptor: 0.ddd...E+ee, right-justified in w columns (the probe files'
    E23.15, ModProbe.f90:196-208)."""
    x = float(x)
    if x == 0.0 or not math.isfinite(x):
        body = f"0.{'0' * d}E+00" if x == 0.0 else ("NaN" if math.isnan(x) else ("-" if x < 0 else "+") + "Infinity")
        if x == 0.0 and math.copysign(1.0, x) < 0:
            body = "-" + body
        return body.rjust(w)
    s = f"{abs(x):.{d - 1}e}"          # d.ddd e+XX with d significant digits
    mant, exp = s.split("e")
    digits = mant.replace(".", "")
    e = int(exp) + 1
    es = f"E{'+' if e >= 0 else '-'}{abs(e):02d}" if abs(e) <= 99 else f"{'+' if e >= 0 else '-'}{abs(e):03d}"
    return (("-" if x < 0 else "") + "0." + digits + es).rjust(w)


class _StepView:
    """What a probe reads of one post-processed record: time, U, Gauss-point stress and F."""

    def __init__(self, case, loop, rec, need_gp):
        self.case, self.loop, self.time, self.U = case, loop, rec["time"], rec["U"]
        self._sig = self._F = None
        self.need_gp = need_gp

    def stress(self):
        if self._sig is None:
            self._sig = self.loop.gp_stress()  # [n_elem, 8, 6] of the last evaluation
        return self._sig

    def F(self):
        if self._F is None:
            self._F = gp_deformation(self.loop, self.U)
        return self._F


def gp_deformation(loop, U):
    """F at every Gauss point [n_elem, 8, 3, 3] from the GPU (ceos_gp_deformation_device, the
    DeformationGradient of ModElement.f90:1210-1300 on the reference coordinates)."""
    import ctypes as C

    import torch

    from . import lib
    dev = torch.device("cuda", torch.cuda.current_device())
    dU = torch.as_tensor(np.ascontiguousarray(U, np.float64), device=dev)
    n_gp = 8 * loop.n_elem
    dF = torch.empty(9 * n_gp, dtype=torch.float64, device=dev)
    rc = lib().ceos_gp_deformation_device(loop.handle, C.c_void_p(dU.data_ptr()), C.c_void_p(dF.data_ptr()),
                                          C.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    if rc < 0:
        from . import CeosError
        raise CeosError(rc, "ceos_gp_deformation_device")
    torch.cuda.synchronize(dev)
    F = dF.view(3, 3, 8, loop.n_elem).cpu().numpy()   # [i][j][gp][e], q = gp * n_elem + e
    return np.transpose(F, (3, 2, 0, 1)).copy()


def log_strain(F):
    """StrainMeasure(F, Logarithmic) (Tools/ModContinuumMechanics.f90:76-92): sum of ln(sqrt(lambda_k))
    N_k over the eigenpairs of b = F F^T."""
    lam, vec = np.linalg.eigh(F @ F.T)
    return sum(math.log(math.sqrt(lam[k])) * np.outer(vec[:, k], vec[:, k]) for k in range(3))


VARIABLES = {"displacements": 1, "temperature": 2, "cauchystress": 3, "logarithmicstrain": 4,
             "deformationgradient": 5, "firstpiolastress": 6}


class _Probe:
    def __init__(self, file_name, variable, components):
        self.file_name, self.variable = file_name, fmt(variable)
        self.all = fmt(components) == "all"
        self.components = [] if self.all else [int(c) for c in components.replace(",", " ").split()]
        self.active = True
        self.path = None

    def initialize(self, out_dir):
        """InitializeFile (ModProbe.f90:148-180): the file starts again with its header."""
        self.path = os.path.join(out_dir, self.file_name)
        with open(self.path, "w") as f:
            f.write("  Time                    Value\n")

    def _line(self, text):
        with open(self.path, "a") as f:
            f.write(text + "\n")

    def _values(self, time, values):
        """WriteOnFile_Value: '(n(E23.15,1x))' with the time first."""
        self._line("".join(fortran_e(v) + " " for v in [time] + list(values)))

    def _error(self, text):
        self._line(text)
        self.active = False


class NodeProbe(_Probe):
    """WriteProbeResult_Node (ModProbe.f90:263-335): displacements of one node."""

    def __init__(self, file_name, variable, node, components):
        super().__init__(file_name, variable, components)
        self.node = node

    def write(self, v):
        if not self.active:
            return
        if self.node > len(v.case.mesh["X"]):
            return self._error("ERROR - Node Number is greater than the Max Number of Nodes in the Mesh")
        if self.variable != "displacements":
            return self._error("ERROR: Variable not available")
        base = 3 * (self.node - 1)
        if self.all:
            return self._values(v.time, v.U[base:base + 3])
        if any(c > 3 for c in self.components):
            return self._error("ERROR: Component is greater than the available")
        self._values(v.time, [v.U[base + c - 1] for c in self.components])


class GaussPointProbe(_Probe):
    """WriteProbeResult_GaussPoint (ModProbe.f90:387-563): Cauchy stress (Voigt 11,22,33,12,23,13),
    logarithmic strain (same order) or F (column-major, Convert_to_Voigt_3D) of one Gauss point."""

    def __init__(self, file_name, variable, element, gauss_point, components):
        super().__init__(file_name, variable, components)
        self.element, self.gauss_point = element, gauss_point

    def write(self, v):
        if not self.active:
            return
        if self.element > len(v.case.mesh["conn"]):
            return self._error("ERROR - Number of Element is greater than Max Number of Elements in Mesh")
        if self.gauss_point > 8:
            return self._error("ERROR - Number of Gauss Point is greater than Max Number of Gauss Points in the "
                               "Element")
        e, g = self.element - 1, self.gauss_point - 1
        if self.variable in ("cauchystress", "logarithmicstrain"):
            if any(c > 6 for c in self.components):
                what = "Stress" if self.variable == "cauchystress" else "Strain"
                return self._error(f"ERROR - {what} component is greater than Max {what} Size")
            if self.variable == "cauchystress":
                vals = v.stress()[e, g]
            else:
                E = log_strain(v.F()[e, g])
                vals = np.array([E[0, 0], E[1, 1], E[2, 2], E[0, 1], E[1, 2], E[0, 2]])
        elif self.variable == "deformationgradient":
            if any(c > 9 for c in self.components):
                return self._error("ERROR - Deformation Gradient component is greater than Max Size")
            vals = v.F()[e, g].T.reshape(-1)
        else:
            raise CaseFormatError("Error in ModProbe - WriteProbeResult_GaussPoint - VariableNameID - not identified")
        self._values(v.time, vals if self.all else [vals[c - 1] for c in self.components])


def read_probes(path):
    """The PROBE blocks of Post_Processing.post (ReadPostProcessingInputFile and the probe
    constructors of ModProbe.f90:212-383): Location Node or Gauss Point, File Name, Variable Name,
    Node or Element + Gauss Point, Components."""
    L = _Lines(path)
    probes = []
    while not L.eof():
        orig, f = L.next()
        if f != "probe":
            continue
        opts = {}
        while L.peek() is not None and L.peek()[1] != "endprobe":
            o, _ = L.next()
            if "=" in o:
                k, val = o.split("=", 1)
                opts[fmt(k)] = val.strip()
        L.next("END PROBE")
        loc = fmt(opts.get("location", ""))
        fname = opts.get("filename", "")
        var = opts.get("variablename", "")
        comps = opts.get("components", "All")
        if fmt(var) not in VARIABLES:
            raise CaseFormatError(f"Probe variable not identified: [{var}]")
        if loc == "node":
            probes.append(NodeProbe(fname, var, int(_number(opts["node"])), comps))
        elif loc == "gausspoint":
            probes.append(GaussPointProbe(fname, var, int(_number(opts["element"])),
                                          int(_number(opts["gausspoint"])), comps))
        else:
            raise CaseFormatError(f"Probe location not available on this path: [{opts.get('location', '')}]")
    return probes


# ---------------------------------------------------------------------------------------------
# Checker
# ---------------------------------------------------------------------------------------------

def check(file1, file2, tol=1.0e-8, log=None):
    """The reference's Checker (Checker/Checker Code/Checker/Checker.f90): skip one header line of
    each file, then compare the two columns of every row of file1 with the same row of file2 in
    absolute value against tol.  Returns (True, "SUCCESS") or (False, message); log (a path) gets
    the reference's Log_CHECKER.txt lines appended."""
    def rows(path):
        with open(path, "r", encoding="latin-1") as f:
            lines = [ln for ln in f if ln.strip()]
        return [[_number(t) for t in ln.split()[:2]] for ln in lines[1:]]

    out = [" " + "-" * 70, f"    Comparing File: {file1} with File: {file2}"]
    a, b = rows(file1), rows(file2)
    ok, msg = True, "SUCCESS"
    for k, (r1) in enumerate(a):
        if k >= len(b):
            ok, msg = False, f"File 2 ends before File 1 (row {k + 1})"
            break
        r2 = b[k]
        for col, name in ((0, "first"), (1, "second")):
            if abs(r1[col] - r2[col]) > tol:
                ok = False
                msg = (f"Absolute difference in {name} column greater than the tolerance. Tolerance = {tol}; "
                       f"File 1 :: point = {r1[col]}; File 2 :: point = {r2[col]}")
                break
        if not ok:
            break
    out += ["", "    " + msg, " " + "-" * 70]
    if log:
        with open(log, "a") as f:
            f.write("\n".join(out) + "\n")
    return ok, msg
