"""Generate the golden fixtures tests/golden/hexa8_svk.json and tests/golden/hexa8_nh_q1p0.json from
the reference's golden Checker cases.

Two reference cases pin the Hexa8 element loop, the upper-CSR assembly, the rearrangement boundary
conditions and the Newton driver (96 Hexa8 elements, 195 nodes, 50 load steps, the same mesh):
- Checker/Cases/NonLinear_FEA_3D_Hexa8_StVenant: St Venant-Kirchhoff, full integration;
- Checker/Cases/NonLinear_FEA_3D_Hexa8_NeoHookean_Incompressible: Neo_Hookean (C10, Bulk
  Modulus) with the Mean Dilatation element technology.
This script reads their input files (GiD-12 Mesh.dat, tables, time discretization) and expected
outputs (MARC displacement curves of node 11, NumOfIterRef.dat, the per-iteration NORM lines of
Log_CEOS.txt) and writes them as JSON fixtures, so that the tests never read the reference tree
at run time.  It also copies each case's text files unchanged (line ends normalised) into
tests/golden/cases/<case>/, the inputs of the case-file reader and of the Checker workflow.

Usage:  python tests/golden/make_golden.py /path/to/reference
"""
import json
import os
import re
import sys

CASE_FILES = ["Settings.dat", "Mesh.dat", "Time_Discretization.dat", "Table_Disp_Z.tab", "Table_Load_Y.tab",
              "Post_Processing.post", "marc_disp_x.dat", "marc_disp_y.dat", "marc_disp_z.dat", "NumOfIterRef.dat"]

CASES = [
    ("Checker/Cases/NonLinear_FEA_3D_Hexa8_StVenant", "hexa8_svk.json",
     {"model": "St_Venant_Kirchhoff", "YoungModulus": 100.0e9, "Poisson": 0.3}),
    ("Checker/Cases/NonLinear_FEA_3D_Hexa8_NeoHookean_Incompressible", "hexa8_nh_q1p0.json",
     {"model": "Neo_Hookean", "C10": 5.0e10, "BulkModulus": 5.0e13, "element_technology": "Mean Dilatation"}),
]


def _lines(path):
    with open(path, "r", encoding="latin-1") as f:
        return [ln.rstrip("\n") for ln in f]


def read_mesh(path):
    """Minimal GiD-12 reader (ModReadInputFile.f90:1396-1561, 1565-1709)."""
    L = [ln.strip() for ln in _lines(path)]
    i = 0
    coords, conn, mat = {}, {}, {}
    fixed, loads, disps = [], [], []
    while i < len(L):
        s = L[i].upper()
        if s == "COORDINATES":
            i += 1
            while L[i].upper() != "END COORDINATES":
                t = L[i].split()
                coords[int(t[0])] = [float(v) for v in t[1:4]]
                i += 1
        elif s == "MATERIAL ID":
            i += 2
            while L[i].upper() != "END MATERIAL ID":
                t = L[i].split()
                mat[int(t[0])] = int(t[1])
                i += 1
        elif s == "CONNECTIVITY":
            i += 1
            while L[i].upper() != "END CONNECTIVITY":
                t = [int(v) for v in L[i].split()]
                conn[t[0]] = t[3:3 + t[2]]
                i += 1
        elif s == "FIXED SUPPORTS":
            n = int(L[i + 1])
            for k in range(n):
                t = [int(v) for v in L[i + 2 + k].split()]
                fixed.append(t)
            i += 1 + n
        elif s == "NODAL LOAD":
            n = int(L[i + 1])
            for k in range(n):
                t = L[i + 2 + k].split()
                loads.append([int(t[0])] + [[int(t[1 + 2 * d]), t[2 + 2 * d]] for d in range(3)])
            i += 1 + n
        elif s == "NODAL DISPLACEMENT":
            n = int(L[i + 1])
            for k in range(n):
                t = L[i + 2 + k].split()
                disps.append([int(t[0])] + [[int(t[1 + 2 * d]), t[2 + 2 * d]] for d in range(3)])
            i += 1 + n
        i += 1
    nn, ne = len(coords), len(conn)
    return {
        "X": [c for k in range(1, nn + 1) for c in coords[k]],
        "conn": [n for e in range(1, ne + 1) for n in conn[e]],
        "mat_id": [mat[e] for e in range(1, ne + 1)],
        "fixed": fixed,
        "loads": loads,
        "disps": disps,
    }


def read_table(path):
    rows = []
    for ln in _lines(path):
        t = ln.split()
        if len(t) >= 2:
            try:
                rows.append([float(t[0].replace("d", "e").replace("D", "e")),
                             float(t[1].replace("d", "e").replace("D", "e"))])
            except ValueError:
                pass
    return rows


def read_two_cols(path):
    out = []
    for ln in _lines(path):
        t = ln.split()
        if len(t) >= 2:
            try:
                out.append([float(t[0]), float(t[1])])
            except ValueError:
                pass
    return out


def read_log_norms(path):
    steps, cur = [], None
    for ln in _lines(path):
        m = re.match(r"\s*Step:\s+(\d+)", ln)
        if m and "End" not in ln:
            cur = []
            steps.append(cur)
        m = re.search(r"IT:\s+(\d+)\s+NORM:\s+([0-9.Ee+-]+)", ln)
        if m and cur is not None:
            cur.append(float(m.group(2)))
    return steps


def main(ref):
    for case_rel, out_name, material in CASES:
        case = os.path.join(ref, case_rel)
        mesh = read_mesh(os.path.join(case, "Mesh.dat"))
        fx = {
            "source": case_rel,
            "material": material,
            "newton": {"tol": 1e-3, "itmax": 10, "max_cutbacks": 10},
            "time": {"t0": 0.0, "t1": 1.0, "steps": 50},
            "probe_node": 11,
            "tables": {
                "Table_Disp_Z": read_table(os.path.join(case, "Table_Disp_Z.tab")),
                "Table_Load_Y": read_table(os.path.join(case, "Table_Load_Y.tab")),
            },
            "marc": {
                "x": read_two_cols(os.path.join(case, "marc_disp_x.dat")),
                "y": read_two_cols(os.path.join(case, "marc_disp_y.dat")),
                "z": read_two_cols(os.path.join(case, "marc_disp_z.dat")),
            },
            "iterations_ref": read_two_cols(os.path.join(case, "NumOfIterRef.dat")),
            "log_norms": read_log_norms(os.path.join(case, "Log_CEOS.txt")),
        }
        fx.update(mesh)
        here = os.path.dirname(os.path.abspath(__file__))
        cdir = os.path.join(here, "cases", out_name[:-5])
        os.makedirs(cdir, exist_ok=True)
        for name in CASE_FILES:
            with open(os.path.join(case, name), "r", encoding="latin-1") as f:
                text = f.read().replace("\r\n", "\n")
            with open(os.path.join(cdir, name), "w", encoding="latin-1") as f:
                f.write(text)
        out = os.path.join(here, out_name)
        with open(out, "w") as f:
            json.dump(fx, f, separators=(",", ":"))
        print("wrote", out, "nodes", len(mesh["X"]) // 3, "elements", len(mesh["conn"]) // 8)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the reference checkout>")
    main(sys.argv[1])
