"""Batched FE^2 micro problems (C ABI ceos_fe2_*): many periodic fibre RVEs solved in one batch
on the GPU, returning the homogenized first Piola stress and its 9x9 tangent."""
import ctypes as C

import numpy as np

from . import CeosError, lib, _check, _ptr


def _setup():
    L = lib()
    P, I, D = C.c_void_p, C.c_int, C.c_double
    L.ceos_fe2_create.argtypes = [I, P, P, D, D, D, I, C.POINTER(P)]
    L.ceos_fe2_info.argtypes = [P, P, P, P, P]
    L.ceos_fe2_solve.argtypes = [P, P, D, I, P, P, P, P]
    L.ceos_fe2_message.argtypes = [P, C.c_char_p, I]
    L.ceos_fe2_set_increments.argtypes = [P, I]
    L.ceos_fe2_set_allow_failures.argtypes = [P, I]
    L.ceos_fe2_set_device_rounds.argtypes = [P, I]
    L.ceos_fe2_set_fractions.argtypes = [P, P]
    L.ceos_fe2_set_warm_start.argtypes = [P, I]
    L.ceos_fe2_set_solver_ctas.argtypes = [P, I]
    L.ceos_fe2_set_solve_mask.argtypes = [P, P]
    L.ceos_fe2_autotune.argtypes = [P, P, P, P, P, I]
    L.ceos_fe2_destroy.argtypes = [P]
    L.ceos_fe2_destroy.restype = None
    return L


def sample_rve_family(n_rve, seed=0, n_range=(6, 12), vf_range=(0.1, 0.4)):
    """RVE sizes n ~ U{n_range} and fibre volume fractions vf ~ U[vf_range] (seeded)."""
    rng = np.random.default_rng(seed)
    n = rng.integers(n_range[0], n_range[1] + 1, size=n_rve).astype(np.int32)
    vf = rng.uniform(vf_range[0], vf_range[1], size=n_rve)
    return n, vf


def sample_macro_F(n_rve, seed=1, amp=0.15):
    """F = I + G, G_ij ~ U[-amp, amp], redrawn until det F > 0."""
    rng = np.random.default_rng(seed)
    F = np.empty((n_rve, 3, 3))
    for r in range(n_rve):
        while True:
            Fr = np.eye(3) + rng.uniform(-amp, amp, (3, 3))
            if np.linalg.det(Fr) > 0:
                break
        F[r] = Fr
    return F


class BatchedRVE:
    def __init__(self, n_cells, vf, mu_matrix=1.0, stiff_ratio=50.0, k_over_mu=100.0, device=0):
        L = _setup()
        self.n_cells = np.ascontiguousarray(n_cells, dtype=np.int32)
        self.vf = np.ascontiguousarray(vf, dtype=np.float64)
        self.n_rve = self.n_cells.size
        h = C.c_void_p()
        _check(L.ceos_fe2_create(self.n_rve, _ptr(self.n_cells), _ptr(self.vf), mu_matrix, stiff_ratio, k_over_mu,
                                 device, C.byref(h)))
        self._h = h
        nn, ne, nr = C.c_int(), C.c_int(), C.c_int()
        self.vf_actual = np.zeros(self.n_rve)
        _check(L.ceos_fe2_info(h, C.byref(nn), C.byref(ne), C.byref(nr), _ptr(self.vf_actual)))
        self.n_nodes, self.n_elem, self.n_red = nn.value, ne.value, nr.value

    def set_increments(self, n_sub):
        _check(lib().ceos_fe2_set_increments(self._h, n_sub))

    def set_allow_failures(self, allow=True):
        """RVEs that cannot converge come back as NaN (and newton_iters -1) instead of raising."""
        _check(lib().ceos_fe2_set_allow_failures(self._h, 1 if allow else 0))
        self._allow = allow

    def set_device_rounds(self, on=True):
        """Run every Newton round of a solve on the device (the default: one CUDA graph with a WHILE node,
        launched once per solve), or (on=False) take the per-RVE decisions on the host between rounds."""
        _check(lib().ceos_fe2_set_device_rounds(self._h, 1 if on else 0))

    def set_solver_ctas(self, n=0):
        """RVEs the MINRES kernel keeps in flight (0: as many as occupancy allows)."""
        _check(lib().ceos_fe2_set_solver_ctas(self._h, n))

    def autotune(self, Fbar):
        """Time the MINRES launch shapes (threads per RVE x RVEs in flight) on the first Newton system of
        every RVE at Fbar and keep the fastest for the following solves.  Returns {"threads", "ctas"
        (0: occupancy limit), "ms": {(threads, in_flight): ms}}."""
        Fbar = np.ascontiguousarray(np.asarray(Fbar, dtype=np.float64).reshape(self.n_rve, 9))
        t, c = C.c_int(0), C.c_int(0)
        ms = np.full(6, -1.0)
        rc = lib().ceos_fe2_autotune(self._h, _ptr(Fbar), C.byref(t), C.byref(c), _ptr(ms), 6)
        if rc:
            buf = C.create_string_buffer(256)
            lib().ceos_fe2_message(self._h, buf, 256)
            raise CeosError(rc, buf.value.decode())
        shapes = [(bs, w) for bs in (256, 512) for w in ("occupancy", "2/SM", "1/SM")]
        return {"threads": t.value, "ctas": c.value,
                "ms": {k: float(v) for k, v in zip(shapes, ms) if v >= 0}}

    def set_warm_start(self, on=True):
        """Continue every RVE from its last converged state (macro load path) on the next solves."""
        _check(lib().ceos_fe2_set_warm_start(self._h, 1 if on else 0))

    def set_solve_mask(self, mask=None):
        """Solve only the RVEs where mask != 0 on the next solves (None: all)."""
        self._mask = None if mask is None else np.ascontiguousarray(mask, dtype=np.int32)
        _check(lib().ceos_fe2_set_solve_mask(self._h, _ptr(self._mask) if self._mask is not None else None))

    def set_fractions(self, vf):
        """New fibre volume fractions for the same RVE sizes (mesh and pattern kept)."""
        self.vf = np.ascontiguousarray(vf, dtype=np.float64)
        assert self.vf.size == self.n_rve
        _check(lib().ceos_fe2_set_fractions(self._h, _ptr(self.vf)))
        _check(lib().ceos_fe2_info(self._h, None, None, None, _ptr(self.vf_actual)))

    def solve(self, Fbar, tangent=False, tol=1e-8, max_newton=20):
        Fbar = np.ascontiguousarray(np.asarray(Fbar, dtype=np.float64).reshape(self.n_rve, 9))
        P = np.zeros((self.n_rve, 9))
        A = np.zeros((self.n_rve, 81)) if tangent else None
        nit = np.zeros(self.n_rve, np.int32)
        cgi = np.zeros(self.n_rve, np.int32)
        rc = lib().ceos_fe2_solve(self._h, _ptr(Fbar), tol, max_newton, _ptr(P), _ptr(A), _ptr(nit), _ptr(cgi))
        if rc and not (rc == 2 and getattr(self, "_allow", False)):
            buf = C.create_string_buffer(256)
            lib().ceos_fe2_message(self._h, buf, 256)
            raise CeosError(rc, buf.value.decode())
        out = {"P": P.reshape(self.n_rve, 3, 3), "newton_iters": nit, "cg_iters": cgi, "failed": nit < 0}
        if tangent:
            out["A"] = A.reshape(self.n_rve, 9, 9)
        return out

    def close(self):
        if getattr(self, "_h", None):
            lib().ceos_fe2_destroy(self._h)
            self._h = None

    def __del__(self):
        try:  # at interpreter exit the library binding may already be gone
            self.close()
        except Exception:
            pass
