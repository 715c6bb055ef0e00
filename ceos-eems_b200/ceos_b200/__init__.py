"""ceos_b200 -- Python binding of the B200 element loop (ceos_b200/lib/libceos_b200.so).

Mirrors the plugin interface the reference's Newton solver calls
(Tools/MathTools/ModNonLinearSystemOfEquations.f90:9-20, implemented by
FEM/Modules/ModFEMSystemOfEquations.f90): ``EvaluateR``, ``EvaluateKt`` and ``PostUpdate``,
on top of the C ABI of include/ceos_gpu.h.  There is no CPU fallback: every call goes
through the sm_100a library, and loading fails loudly when it is missing.
"""
import ctypes as C
import os

import numpy as np

from . import meshgen  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "lib", "libceos_b200.so")

J2_SMALL, NH_Q1P0, SVK, CNH, VISCO_VAR, VISCO_PRONY, J2_FINITE = 2, 4, 5, 7, 12, 101, 102
FP64, MIXED = 0, 1
OPT_STORE_STRESS = 1
OPT_TIME_KERNELS = 2
ASSEMBLY_TWO_PASS, ASSEMBLY_FUSED, ASSEMBLY_BANDED = 0, 1, 2
_ASSEMBLY = {"two-pass": ASSEMBLY_TWO_PASS, "fused": ASSEMBLY_FUSED, "banded": ASSEMBLY_BANDED}

_lib = None

# int (*)(void* user, double time, int load_case, int step, int cutback, int substep, int flag_end_step,
#         int n_iterations, int n_dof, const double* U)
STEP_CALLBACK = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                            C.c_int, C.POINTER(C.c_double))


class CeosError(RuntimeError):
    """Non-zero status of a C-ABI call (ClassStatus error convention)."""

    def __init__(self, code, msg=""):
        super().__init__(f"ceos status {code}: {msg}")
        self.code = code


class _Mesh(C.Structure):
    _fields_ = [("n_nodes", C.c_int), ("n_elem", C.c_int), ("X", C.c_void_p), ("conn", C.c_void_p),
                ("mat_id", C.c_void_p)]


class _Material(C.Structure):
    _fields_ = [("model", C.c_int), ("per_element", C.c_int), ("n_params", C.c_int), ("params", C.c_void_p)]


def build():
    """Compile the sm_100a library in-tree (make -C ceos-eems_b200)."""
    import subprocess
    subprocess.check_call(["make", "-s", "-C", os.path.dirname(HERE)])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            raise RuntimeError(f"CUDA library {LIBPATH} is not built; run ceos_b200.build()")
        L = C.CDLL(LIBPATH)
        P, I, LL, D = C.c_void_p, C.c_int, C.c_longlong, C.c_double
        ip = C.POINTER(C.c_int)
        L.ceos_create.argtypes = [C.POINTER(_Mesh), C.POINTER(_Material), I, I, I, C.POINTER(P)]
        L.ceos_pattern.argtypes = [P, ip, C.POINTER(LL), P, P, P]
        L.ceos_slot_map.argtypes = [P, P]
        L.ceos_evaluate.argtypes = [P, D, P, P, P, ip]
        L.ceos_evaluate_device.argtypes = [P, D, P, P, P, P]
        L.ceos_status.argtypes = [P, ip]
        L.ceos_commit_state.argtypes = [P]
        L.ceos_last_error.argtypes = [P, P, I, C.c_char_p, I]
        L.ceos_state_size.argtypes = [P, ip]
        L.ceos_get_state.argtypes = [P, I, P]
        L.ceos_set_state.argtypes = [P, I, P]
        L.ceos_gp_stress.argtypes = [P, P]
        L.ceos_set_options.argtypes = [P, I]
        L.ceos_set_assembly.argtypes = [P, I]
        L.ceos_launch_count.argtypes = [P, I, ip]
        L.ceos_test_stall_conversion.argtypes = [P, I, I]
        L.ceos_set_committed_time.argtypes = [P, D]
        L.ceos_kernel_time.argtypes = [P, C.POINTER(C.c_float)]
        L.ceos_destroy.argtypes = [P]
        L.ceos_destroy.restype = None
        L.ceos_analysis.argtypes = [P, I, P, P, I, P, I, P, P, P, I, P, P, P, D, I, I, I, I, P, P, I, P, P, I, P,
                                    ip, P]
        L.ceos_analysis_set_callback.argtypes = [P, STEP_CALLBACK, P]
        L.ceos_analysis_set_initial.argtypes = [P, P]
        L.ceos_analysis_set_device_solver.argtypes = [P, I, D, I]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _check(rc, h=None):
    if rc != 0:
        msg = ""
        if h is not None and rc > 0:
            buf = C.create_string_buffer(256)
            lib().ceos_last_error(h, None, 0, buf, 256)
            msg = buf.value.decode()
        raise CeosError(rc, msg)


class ElementLoop:
    """One handle of the C ABI: mesh + materials + Gauss-point state on one GPU."""

    def __init__(self, X, conn, model, params, mat_id=None, per_element=False, precision=FP64, device=0):
        X = _f64(X).reshape(-1)
        conn = _i32(conn).reshape(-1)
        self.n_nodes = X.size // 3
        self.n_elem = conn.size // 8
        self.n_dof = 3 * self.n_nodes
        self.model = model
        self.precision = precision
        self.assembly = "two-pass"
        params = np.asarray(params, dtype=np.float64)
        if per_element:
            params = np.atleast_2d(params)
            mats = [(_f64(params.reshape(-1)), params.shape[1], 1)]
        else:
            params = np.atleast_2d(params)
            mats = [(_f64(p), p.size, 0) for p in params]
        self._keep = [X, conn] + [m[0] for m in mats]
        mesh = _Mesh(self.n_nodes, self.n_elem, _ptr(X), _ptr(conn), None)
        if mat_id is not None:
            mid = _i32(mat_id)
            self._keep.append(mid)
            mesh.mat_id = _ptr(mid)
        arr = (_Material * len(mats))(*[_Material(model, pe, npar, _ptr(p)) for (p, npar, pe) in mats])
        h = C.c_void_p()
        rc = lib().ceos_create(C.byref(mesh), arr, len(mats), precision, device, C.byref(h))
        _check(rc)
        self._h = h
        nd = C.c_int()
        nnz = C.c_longlong()
        _check(lib().ceos_pattern(h, C.byref(nd), C.byref(nnz), None, None, None))
        self.nnz = nnz.value
        nv = C.c_int()
        lib().ceos_state_size(h, C.byref(nv))
        self.nstate = nv.value

    def close(self):
        if getattr(self, "_h", None):
            lib().ceos_destroy(self._h)
            self._h = None

    def __del__(self):
        try:  # at interpreter exit the library binding may already be gone
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def pattern(self, with_row=False):
        rowmap = np.zeros(self.n_dof + 1, np.int32)
        col = np.zeros(self.nnz, np.int32)
        row = np.zeros(self.nnz, np.int32) if with_row else None
        _check(lib().ceos_pattern(self._h, None, None, _ptr(rowmap), _ptr(col), _ptr(row)))
        return (rowmap, col, row) if with_row else (rowmap, col)

    def slot_map(self):
        out = np.zeros(self.n_elem * 576, np.int64)
        _check(lib().ceos_slot_map(self._h, _ptr(out)))
        return out.reshape(self.n_elem, 24, 24)

    def evaluate(self, time, U, tangent=True, raise_on_error=False):
        """Returns (fint, kval or None, status, n_failed_elements)."""
        U = _f64(U)
        fint = np.zeros(self.n_dof)
        kval = np.zeros(self.nnz) if tangent else None
        nf = C.c_int(0)
        rc = lib().ceos_evaluate(self._h, time, _ptr(U), _ptr(fint), _ptr(kval), C.byref(nf))
        if rc < 0 or (raise_on_error and rc):
            _check(rc, self._h)
        return fint, kval, rc, nf.value

    def evaluate_device(self, time, dU, dfint, dkval=None, stream=None):
        """Device-resident evaluation on torch CUDA tensors (asynchronous on `stream`)."""
        rc = lib().ceos_evaluate_device(self._h, time, C.c_void_p(dU.data_ptr()), C.c_void_p(dfint.data_ptr()),
                                        C.c_void_p(dkval.data_ptr()) if dkval is not None else None,
                                        C.c_void_p(stream) if stream else None)
        _check(rc)

    def status(self):
        nf = C.c_int(0)
        rc = lib().ceos_status(self._h, C.byref(nf))
        return rc, nf.value

    def failed_elements(self):
        ids = np.zeros(self.n_elem, np.int32)
        buf = C.create_string_buffer(256)
        n = lib().ceos_last_error(self._h, _ptr(ids), self.n_elem, buf, 256)
        return ids[:max(n, 0)], buf.value.decode()

    def commit(self):
        _check(lib().ceos_commit_state(self._h))

    def set_committed_time(self, t):
        _check(lib().ceos_set_committed_time(self._h, t))

    def state(self, which=0):
        if not self.nstate:
            return np.zeros((self.n_elem, 8, 0))
        out = np.zeros(self.n_elem * 8 * self.nstate)
        _check(lib().ceos_get_state(self._h, which, _ptr(out)))
        return out.reshape(self.n_elem, 8, self.nstate)

    def set_state(self, st, which=0):
        st = _f64(st).reshape(-1)
        _check(lib().ceos_set_state(self._h, which, _ptr(st)))

    def set_options(self, options):
        _check(lib().ceos_set_options(self._h, options))

    def store_stress(self, on=True):
        self.set_options(OPT_STORE_STRESS if on else 0)

    def set_assembly(self, mode):
        """Mixed-precision K assembly: "two-pass" (default; element loop into FP32 node-pair blocks,
        then a conversion launch writes the FP64 CSR rows), "fused" (one launch from a host-planned
        queue, blocks in an L2-sized ring) or "banded" (the two passes band by band on three streams,
        blocks in a ring of a few bands)."""
        _check(lib().ceos_set_assembly(self._h, _ASSEMBLY[mode]))
        self.assembly = mode

    def test_stall_conversion(self, item, on=True):
        """Failure-path test of the fused assembly: conversion item `item` waits for a flag that nothing
        sets (its bounded wait runs out and the launch reports an error), or is restored (on=False)."""
        _check(lib().ceos_test_stall_conversion(self._h, item, int(bool(on))))

    def launches_per_evaluation(self, tangent=True):
        """Kernels that one device-resident evaluation launches under the current assembly."""
        n = C.c_int(0)
        _check(lib().ceos_launch_count(self._h, int(bool(tangent)), C.byref(n)))
        return n.value

    def kernel_names(self):
        """Names of the kernels of one device-resident evaluation with a tangent."""
        if self.precision != MIXED:
            return ["element_loop_kernel"]
        return ["element_assemble_kernel"] if self.assembly == "fused" else ["element_loop_kernel", "csr_convert_kernel"]

    def kernel_time_ms(self):
        """(element loop ms, conversion ms) of the last evaluation; the conversion entry is 0 when one
        launch does both (fused assembly) or there is no conversion (FP64)."""
        ms = (C.c_float * 2)()
        _check(lib().ceos_kernel_time(self._h, ms))
        return ms[0], ms[1]

    def gp_stress(self):
        out = np.zeros(self.n_elem * 8 * 6)
        _check(lib().ceos_gp_stress(self._h, _ptr(out)))
        return out.reshape(self.n_elem, 8, 6)

    def analysis(self, bc, tol, itmax, norm_mode, norm_type=2, max_cutbacks=10, probe_dofs=(), max_log=100000,
                 on_step=None, U0=None, device_solver=False, lin_tol=1e-12, lin_max_iter=20000):
        """Quasi-static analysis of one load case through ceos_analysis.  on_step(time, load_case, step,
        cutback, substep, flag_end_step, n_iterations, U) is called for every converged substep (the
        WriteFEMResults call sites); a True return stops the analysis.  U0 starts from given
        displacements (a restart) instead of zero.  device_solver: the Newton iteration stays on the
        device (boundary conditions as kernels, PCG to lin_tol) instead of the host factorization."""
        _check(lib().ceos_analysis_set_device_solver(self._h, 1 if device_solver else 0, lin_tol, lin_max_iter))
        n_steps = len(bc["t0"])
        iters = np.zeros(n_steps, np.int32)
        cuts = np.zeros(n_steps, np.int32)
        probe_dofs = _i32(probe_dofs if len(probe_dofs) else [1])
        probe = np.zeros(len(probe_dofs) * n_steps)
        log = np.zeros(max_log)
        nlog = C.c_int(0)
        Uf = np.zeros(self.n_dof)
        keep = []

        def arr(a, dt):
            x = np.ascontiguousarray(a, dtype=dt).reshape(-1)
            if x.size == 0:
                x = np.zeros(1, dt)
            keep.append(x)
            return _ptr(x)

        cb = None
        if on_step is not None:
            def _cb(user, t, lc, st, cut, sub, flag, nit, ndof, U):
                try:
                    return 1 if on_step(t, lc, st, cut, sub, flag, nit, np.ctypeslib.as_array(U, (ndof,)).copy()) \
                        else 0
                except Exception:  # an exception cannot cross the C frame: stop the analysis instead
                    import traceback
                    traceback.print_exc()
                    return 1
            cb = STEP_CALLBACK(_cb)
        _check(lib().ceos_analysis_set_callback(self._h, cb if cb is not None else STEP_CALLBACK(), None))
        U0 = _f64(U0).reshape(-1) if U0 is not None else None
        if U0 is not None and U0.size != self.n_dof:
            raise ValueError(f"U0 has {U0.size} entries, the mesh {self.n_dof} dofs")
        _check(lib().ceos_analysis_set_initial(self._h, _ptr(U0)))
        rc = lib().ceos_analysis(
            self._h, n_steps, arr(bc["t0"], np.float64), arr(bc["dt"], np.float64),
            len(bc["fixed"]), arr(bc["fixed"], np.int32),
            len(bc["presc"]), arr(bc["presc"], np.int32), arr(bc["presc_init"], np.float64),
            arr(bc["presc_final"], np.float64),
            len(bc["force"]), arr(bc["force"], np.int32), arr(bc["force_init"], np.float64),
            arr(bc["force_final"], np.float64),
            tol, itmax, norm_mode, norm_type, max_cutbacks, _ptr(iters), _ptr(cuts), len(probe_dofs),
            _ptr(probe_dofs), _ptr(probe), max_log, _ptr(log), C.byref(nlog), _ptr(Uf))
        lib().ceos_analysis_set_callback(self._h, STEP_CALLBACK(), None)
        return {"rc": rc, "iters": iters, "cutbacks": cuts, "probe": probe.reshape(len(probe_dofs), n_steps),
                "norms": log[:min(nlog.value, max_log)], "U": Uf}


class FEMSystemOfEquations:
    """The reference's ClassFEMSystemOfEquations plugin (ModFEMSystemOfEquations.f90:40-106)
    over the GPU element loop: EvaluateR, EvaluateKt (with ApplyBoundaryConditionsNEW on the
    host) and PostUpdate."""

    def __init__(self, loop, fixed_dofs=(), presc_dofs=()):
        self.loop = loop
        self.Time = 0.0
        self.Fext = np.zeros(loop.n_dof)
        self.Ubar = np.zeros(loop.n_dof)
        self.it = 0
        self.fixed = np.asarray(fixed_dofs, np.int64) - 1
        self.presc = np.asarray(presc_dofs, np.int64) - 1
        self.rowmap, self.col = loop.pattern()
        r = np.repeat(np.arange(loop.n_dof), np.diff(self.rowmap))
        c = self.col - 1
        self._row, self._c = r, c
        isp = np.zeros(loop.n_dof, bool)
        isp[self.presc] = True
        isf = np.zeros(loop.n_dof, bool)
        isf[self.fixed] = True
        self.zp = np.nonzero(isp[r] | isp[c])[0]
        self.op = np.nonzero(isp[r] & (r == c))[0]
        self.zf = np.nonzero(isf[r] | isf[c])[0]
        self.of = np.nonzero(isf[r] & (r == c))[0]
        self.Status = 0
        self._kval = None

    def EvaluateR(self, X):
        fint, kval, rc, _ = self.loop.evaluate(self.Time, X, tangent=True)
        self.Status = rc
        self._kval = kval
        return fint - self.Fext

    def _symv(self, kval, x):
        y = np.bincount(self._row, weights=kval * x[self._c], minlength=self.loop.n_dof)
        off = self._row != self._c
        y += np.bincount(self._c[off], weights=kval[off] * x[self._row[off]], minlength=self.loop.n_dof)
        return y

    def EvaluateKt(self, X, R):
        """Returns (kval with BCs, R with BCs); R is the residual of EvaluateR."""
        kval = self._kval.copy()
        R = -R.copy()
        Ud = np.zeros(self.loop.n_dof)
        if self.presc.size:
            if self.it == 0:
                Ud[self.presc] = self.Ubar[self.presc] - X[self.presc]
                R -= self._symv(kval, Ud)
            kval[self.zp] = 0.0
            kval[self.op] = 1.0
            R[self.presc] = Ud[self.presc]
        if self.fixed.size:
            kval[self.zf] = 0.0
            kval[self.of] = 1.0
            R[self.fixed] = 0.0
        return kval, -R

    def PostUpdate(self, X):
        # UpdateMeshCoordinates: the kernel forms Coord = CoordX + U from U itself
        return None
