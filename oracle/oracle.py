"""ctypes binding of the FP64 CPU oracle (oracle/_build/libceos_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg as the checker.  The product (ceos-eems_b200) never imports it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libceos_oracle.so")

CNH, SVK, J2_SMALL, VISCO_VAR, VISCO_PRONY, J2_FINITE, NH_Q1P0 = 7, 5, 2, 12, 101, 102, 4

_lib = None


def build():
    subprocess.check_call(["make", "-s", "-C", HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        P = C.c_void_p
        dp, ip, lp = (np.ctypeslib.ndpointer(np.float64, flags="C"),
                      np.ctypeslib.ndpointer(np.int32, flags="C"),
                      np.ctypeslib.ndpointer(np.int64, flags="C"))
        L.or_model_nparams.restype = C.c_int
        L.or_model_nstate.restype = C.c_int
        L.or_material_point.restype = C.c_int
        L.or_material_point.argtypes = [C.c_int, dp, dp, C.c_double, dp, dp, dp, dp]
        L.or_j2_finite_full_tangent.argtypes = [dp, dp, dp, dp, dp, dp]
        L.or_model_init_state.argtypes = [C.c_int, dp, dp]
        L.or_pattern_nnz.restype = C.c_longlong
        L.or_pattern_nnz.argtypes = [C.c_int, C.c_int, ip]
        L.or_pattern_fill.argtypes = [C.c_int, C.c_int, ip, ip, ip, P]
        L.or_slot_map.argtypes = [C.c_int, C.c_int, ip, ip, ip, lp]
        L.or_create.restype = P
        L.or_create.argtypes = [C.c_int, C.c_int, dp, ip, ip, C.c_int, ip, C.c_int, C.c_int, dp]
        L.or_destroy.argtypes = [P]
        L.or_nnz.restype = C.c_longlong
        L.or_nnz.argtypes = [P]
        L.or_get_pattern.argtypes = [P, ip, ip]
        L.or_evaluate.restype = C.c_int
        L.or_evaluate.argtypes = [P, C.c_double, dp, dp, P, C.POINTER(C.c_int), P]
        L.or_evaluate_sample.restype = C.c_int
        L.or_evaluate_sample.argtypes = [P, C.c_double, dp, dp, P, C.c_int, C.c_int]
        L.or_commit.argtypes = [P]
        L.or_homogenize.argtypes = [P, dp, dp]
        L.or_set_time_old.argtypes = [P, C.c_double]
        L.or_get_gp_stress.argtypes = [P, dp]
        L.or_get_state.restype = C.c_int
        L.or_get_state.argtypes = [P, dp, C.c_int]
        L.or_set_state.restype = C.c_int
        L.or_set_state.argtypes = [P, dp, C.c_int]
        L.or_analysis.restype = C.c_int
        L.or_analysis.argtypes = [P, C.c_int, dp, dp, C.c_int, ip, C.c_int, ip, dp, dp, C.c_int, ip, dp, dp,
                                  C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, ip, ip, C.c_int, ip, dp,
                                  C.c_int, dp, C.POINTER(C.c_int), dp]
        _lib = L
    return _lib


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def nstate(model):
    return lib().or_model_nstate(model)


def init_state(model, params):
    st = np.zeros(max(nstate(model), 1))
    lib().or_model_init_state(model, _f64(params), st)
    return st[:nstate(model)]


def material_point(model, params, F, dt=0.0, st_old=None):
    """Return (sigma[6], D[6,6], st_new, status) for one Gauss point."""
    ns = max(nstate(model), 1)
    if st_old is None:
        st_old = np.zeros(ns)
        if nstate(model):
            st_old[:nstate(model)] = init_state(model, params)
    st_old = _f64(np.resize(st_old, ns) if len(st_old) < ns else st_old)
    st_new = np.zeros(ns)
    sig = np.zeros(6)
    D = np.zeros(36)
    p = np.zeros(16)
    p[:len(params)] = params
    rc = lib().or_material_point(model, p, _f64(np.asarray(F).reshape(9)), dt, st_old, st_new, sig, D)
    return sig, D.reshape(6, 6), st_new[:nstate(model)], rc


def j2_finite_full_tangent(params, F, st_old):
    st_new = np.zeros(7)
    sig = np.zeros(6)
    D = np.zeros(36)
    lib().or_j2_finite_full_tangent(_f64(params), _f64(np.asarray(F).reshape(9)), _f64(st_old), st_new, sig, D)
    return sig, D.reshape(6, 6), st_new


def pattern(n_nodes, conn):
    conn = _i32(conn).reshape(-1)
    ne = conn.size // 8
    nnz = lib().or_pattern_nnz(n_nodes, ne, conn)
    rowmap = np.zeros(3 * n_nodes + 1, np.int32)
    col = np.zeros(nnz, np.int32)
    row = np.zeros(nnz, np.int32)
    lib().or_pattern_fill(n_nodes, ne, conn, rowmap, col, row.ctypes.data_as(C.c_void_p))
    return rowmap, col, row


def slot_map(n_nodes, conn, rowmap, col):
    conn = _i32(conn).reshape(-1)
    ne = conn.size // 8
    out = np.zeros(ne * 576, np.int64)
    lib().or_slot_map(n_nodes, ne, conn, _i32(rowmap), _i32(col), out)
    return out.reshape(ne, 24, 24)


class Model:
    """Mesh + materials + Gauss-point state, evaluated with the reference's three passes."""

    def __init__(self, X, conn, models, params, mat_id=None, per_element=False):
        X = _f64(X).reshape(-1)
        conn = _i32(conn).reshape(-1)
        self.n_nodes = X.size // 3
        self.n_elem = conn.size // 8
        self.n_dof = 3 * self.n_nodes
        models = _i32(np.atleast_1d(models))
        if mat_id is None:
            mat_id = np.zeros(self.n_elem, np.int32)
        params = np.atleast_2d(np.asarray(params, np.float64))
        npm = 16
        P = np.zeros((params.shape[0], npm))
        P[:, :params.shape[1]] = params
        self._h = lib().or_create(self.n_nodes, self.n_elem, X, conn, _i32(mat_id), len(models), models,
                                  1 if per_element else 0, npm, _f64(P))
        self.nnz = lib().or_nnz(self._h)
        self.nstate = max(nstate(int(m)) for m in models)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().or_destroy(self._h)
            self._h = None

    def pattern(self):
        rowmap = np.zeros(self.n_dof + 1, np.int32)
        col = np.zeros(self.nnz, np.int32)
        lib().or_get_pattern(self._h, rowmap, col)
        return rowmap, col

    def evaluate(self, time, U, tangent=True):
        fint = np.zeros(self.n_dof)
        kval = np.zeros(self.nnz) if tangent else None
        nf = C.c_int(0)
        rc = lib().or_evaluate(self._h, time, _f64(U), fint,
                               kval.ctypes.data_as(C.c_void_p) if tangent else None, C.byref(nf), None)
        return fint, kval, rc, nf.value

    def evaluate_sample(self, time, U, n_eval, threads=1, tangent=True):
        fint = np.zeros(self.n_dof)
        kval = np.zeros(self.nnz) if tangent else None
        rc = lib().or_evaluate_sample(self._h, time, _f64(U), fint,
                                      kval.ctypes.data_as(C.c_void_p) if tangent else None, n_eval, threads)
        return fint, kval, rc

    def commit(self):
        lib().or_commit(self._h)

    def homogenize(self, U):
        P = np.zeros(9)
        lib().or_homogenize(self._h, _f64(U), P)
        return P.reshape(3, 3)

    def set_time_old(self, t):
        lib().or_set_time_old(self._h, t)

    def gp_stress(self):
        s = np.zeros(self.n_elem * 8 * 6)
        lib().or_get_gp_stress(self._h, s)
        return s.reshape(self.n_elem, 8, 6)

    def state(self, which=0):
        st = np.zeros(max(self.n_elem * 8 * self.nstate, 1))
        lib().or_get_state(self._h, st, which)
        return st[:self.n_elem * 8 * self.nstate].reshape(self.n_elem, 8, self.nstate)

    def set_state(self, st, which=0):
        lib().or_set_state(self._h, _f64(st).reshape(-1), which)

    def analysis(self, bc, tol, itmax, norm_mode, norm_type=2, max_cutbacks=10, probe_dofs=(), max_log=100000):
        """Run the quasi-static Newton analysis; bc is a BoundaryConditions-like dict
        (see ceos_b200.bc.step_tables)."""
        n_steps = len(bc["t0"])
        iters = np.zeros(n_steps, np.int32)
        cuts = np.zeros(n_steps, np.int32)
        probe_dofs = _i32(probe_dofs if len(probe_dofs) else [1])
        probe = np.zeros(len(probe_dofs) * n_steps)
        log = np.zeros(max_log)
        nlog = C.c_int(0)
        Uf = np.zeros(self.n_dof)
        rc = lib().or_analysis(
            self._h, n_steps, _f64(bc["t0"]), _f64(bc["dt"]),
            len(bc["fixed"]), _i32(bc["fixed"]) if len(bc["fixed"]) else np.zeros(1, np.int32),
            len(bc["presc"]), _i32(bc["presc"]) if len(bc["presc"]) else np.zeros(1, np.int32),
            _f64(bc["presc_init"]).reshape(-1) if len(bc["presc"]) else np.zeros(1),
            _f64(bc["presc_final"]).reshape(-1) if len(bc["presc"]) else np.zeros(1),
            len(bc["force"]), _i32(bc["force"]) if len(bc["force"]) else np.zeros(1, np.int32),
            _f64(bc["force_init"]).reshape(-1) if len(bc["force"]) else np.zeros(1),
            _f64(bc["force_final"]).reshape(-1) if len(bc["force"]) else np.zeros(1),
            tol, itmax, norm_mode, norm_type, max_cutbacks, iters, cuts, len(probe_dofs), probe_dofs, probe,
            max_log, log, C.byref(nlog), Uf)
        return {"rc": rc, "iters": iters, "cutbacks": cuts, "probe": probe.reshape(len(probe_dofs), n_steps),
                "norms": log[:min(nlog.value, max_log)], "U": Uf}
