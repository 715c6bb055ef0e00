"""Macro FE^2 on one GPU: a Hexa8 macro mesh whose Gauss points take their constitutive response
from the learned surrogate (points outside its training box fall back to RVE solves) or from
batched RVE solves everywhere (the direct method), with the macro Newton iteration, boundary
conditions, element loop and linear solves on the device.

The reference runs the macro problem with its FE^2 analysis (MultiScale/ModMultiscaleAnalysis.f90)
and one RVE solve per macro Gauss point; the element loop here reads each point's Cauchy stress
and spatial tangent from the external-material state (model 200) the material step writes.
"""
import ctypes as C
import time

import numpy as np
import torch

from . import FP64, CeosError, ElementLoop, _check, _ptr, lib, meshgen
from . import fe2 as FE2

EXTERNAL = 200
_VI = [0, 1, 2, 0, 1, 0]
_VJ = [0, 1, 2, 1, 2, 2]


def _setup():
    L = lib()
    P, I, D = C.c_void_p, C.c_int, C.c_double
    L.ceos_gp_deformation_device.argtypes = [P, P, P, P]
    L.ceos_state_device.argtypes = [P, C.POINTER(P), C.POINTER(C.c_longlong), C.POINTER(I)]
    L.ceos_pcg_create.argtypes = [P, C.POINTER(P)]
    L.ceos_pcg_solve.argtypes = [P, P, P, P, P, D, I, C.POINTER(I), C.POINTER(D)]
    L.ceos_pcg_destroy.argtypes = [P]
    L.ceos_pcg_destroy.restype = None
    L.ceos_state_scatter.argtypes = [P, I, P, P, I]
    return L


def spatial_from_PA(F, P, A):
    """Cauchy stress [N,6] and spatial tangent [N,21] (upper Voigt entries, tensor components) from
    the first Piola stress P [N,3,3] and its tangent A = dP/dF [N,9,9] (row (iJ), column (kL)):
    sigma = P F^T / J and c_ijkl = F_jJ F_lL A_iJkL / J - delta_ik sigma_jl, minor-symmetrised."""
    J = np.linalg.det(F)
    sig = np.einsum("niJ,njJ->nij", P, F) / J[:, None, None]
    A4 = A.reshape(-1, 3, 3, 3, 3)
    c = np.einsum("njJ,nlL,niJkL->nijkl", F, F, A4) / J[:, None, None, None, None]
    c -= np.einsum("ik,njl->nijkl", np.eye(3), sig)
    c = 0.25 * (c + c.transpose(0, 2, 1, 3, 4) + c.transpose(0, 1, 2, 4, 3) + c.transpose(0, 2, 1, 4, 3))
    s6 = np.stack([0.5 * (sig[:, i, j] + sig[:, j, i]) for i, j in zip(_VI, _VJ)], axis=1)
    D = []
    for p in range(6):
        for q in range(p, 6):
            D.append(c[:, _VI[p], _VJ[p], _VI[q], _VJ[q]])
    return s6, np.stack(D, axis=1)


def uniaxial_bc(X, axis=0):
    """Uniaxial stretch along `axis` with symmetry planes: u_x = 0 on x = 0, u_y = 0 on y = 0, u_z = 0
    on z = 0, the far face normal to `axis` prescribed along it.  The planes remove the rigid modes
    without a point constraint (a pinned corner concentrates strain in its elements).  Returns
    (fixed 0-based dofs, prescribed dofs)."""
    f = meshgen.node_grid_index(X)
    fixed = set(3 * n for n in np.nonzero(f["x0"])[0])
    fixed.update(3 * n + 1 for n in np.nonzero(f["y0"])[0])
    fixed.update(3 * n + 2 for n in np.nonzero(f["z0"])[0])
    far = np.nonzero(f["xyz"[axis] + "1"])[0]
    presc = np.array([3 * n + axis for n in far], np.int64)
    return np.array(sorted(fixed), np.int64), presc


class FallbackLimit(RuntimeError):
    """More Gauss points left the surrogate's training box than the caller allows to solve."""


class MacroFE2:
    """Macro unit cube of nx^3 Hexa8 cells; element e carries fibre fraction vf_elem[e] and every
    one of its Gauss points owns an n_cells^3 periodic RVE of that fraction."""

    def __init__(self, nx, vf_elem, n_cells=6, surrogate=None, mu_matrix=1.0, stiff_ratio=50.0, k_over_mu=100.0,
                 device=0, axis=0):
        self._L = _setup()
        X, conn = meshgen.structured_box(nx, nx, nx, jitter=0.0)
        self.X = X
        self.loop = ElementLoop(X, conn, EXTERNAL, [[0.0]], precision=FP64, device=device)
        self.n_elem = self.loop.n_elem
        self.n_gp = 8 * self.n_elem
        self.n_dof = self.loop.n_dof
        self.vf_elem = np.ascontiguousarray(vf_elem, np.float64)
        self.n_cells = n_cells
        self.rve_args = dict(mu_matrix=mu_matrix, stiff_ratio=stiff_ratio, k_over_mu=k_over_mu, device=device)
        self.sur = surrogate
        dev = torch.device("cuda", device)
        self.dev = dev
        self.U = torch.zeros(self.n_dof, dtype=torch.float64, device=dev)
        self.dU = torch.zeros_like(self.U)
        self.fint = torch.zeros_like(self.U)
        self.rhs = torch.zeros_like(self.U)
        self.kval = torch.zeros(self.loop.nnz, dtype=torch.float64, device=dev)
        self.F = torch.zeros(9 * self.n_gp, dtype=torch.float64, device=dev)
        self.vf_dev = torch.as_tensor(self.vf_elem, device=dev)
        self.flags = torch.zeros(self.n_gp, dtype=torch.int32, device=dev)
        self.axis = axis  # direction of the uniaxial stretch (the RVE fibres run along z = axis 2)
        fixed, self.presc = uniaxial_bc(X, axis)
        mask = np.zeros(self.n_dof, np.uint8)
        mask[fixed] = 1
        mask[self.presc] = 1
        self.fixed = fixed
        self.mask = torch.as_tensor(mask, device=dev)
        self.free = torch.as_tensor(mask == 0, device=dev)
        st = C.c_void_p()
        ld = C.c_longlong()
        f32 = C.c_int()
        _check(self._L.ceos_state_device(self.loop.handle, C.byref(st), C.byref(ld), C.byref(f32)))
        self.state_ptr, self.ld, self.state_f32 = st.value, ld.value, f32.value
        pcg = C.c_void_p()
        _check(self._L.ceos_pcg_create(self.loop.handle, C.byref(pcg)))
        self._pcg = pcg
        self._direct = None
        self.stats = {"material_s": 0.0, "fallback_s": 0.0, "loop_s": 0.0, "solve_s": 0.0, "fallback_points": 0,
                      "pcg_iters": 0}

    # ---- material step ------------------------------------------------------------------------
    def _gp_F_host(self, idx=None):
        F = self.F.view(9, self.n_gp).T
        F = F if idx is None else F[torch.as_tensor(idx, device=self.dev)]
        return F.cpu().numpy().reshape(-1, 3, 3)

    def _point_batch(self):
        """One RVE per macro Gauss point (point q = gp * n_elem + e), warm-started: every RVE follows
        its point's macro load path from solve to solve."""
        if self._direct is None:
            vf = np.tile(self.vf_elem, 8)
            self._direct = FE2.BatchedRVE(np.full(self.n_gp, self.n_cells, np.int32), vf, **self.rve_args)
            self._direct.set_warm_start(True)
        return self._direct

    def _pool_response(self, idx):
        """Large meshes: fallback points get RVE slots from a warm pool of pool_size RVEs (a point keeps
        its slot, and so its RVE state, for the whole run); the solve is masked to their slots."""
        if self._pool is None:
            self._pool = FE2.BatchedRVE(np.full(self.pool_size, self.n_cells, np.int32),
                                        np.full(self.pool_size, 0.25), **self.rve_args)
            self._pool.set_warm_start(True)
            self._slot = {}
            self._pool_vf = np.full(self.pool_size, 0.25)
        new = [q for q in idx if q not in self._slot]
        if len(self._slot) + len(new) > self.pool_size:
            raise FallbackLimit(f"{len(self._slot) + len(new)} fallback points exceed the RVE pool of {self.pool_size}")
        for q in new:
            sl = len(self._slot)
            self._slot[q] = sl
            self._pool_vf[sl] = self.vf_elem[q % self.n_elem]
        if new:
            self._pool.set_fractions(self._pool_vf)
        slots = np.array([self._slot[q] for q in idx])
        mask = np.zeros(self.pool_size, np.int32)
        mask[slots] = 1
        self._pool.set_solve_mask(mask)
        Fh = self._gp_F_host(idx)
        Fall = np.tile(np.eye(3), (self.pool_size, 1, 1))
        Fall[slots] = Fh
        out = self._pool.solve(Fall, tangent=True)
        sig, D = spatial_from_PA(Fh, out["P"][slots], out["A"][slots])
        vals = np.ascontiguousarray(np.concatenate([sig, D], axis=1))
        q = np.ascontiguousarray(idx, np.int32)
        _check(self._L.ceos_state_scatter(self.loop.handle, len(q), _ptr(q), _ptr(vals), 27))

    _pool = None
    pool_size = 512

    def _rve_response(self, idx, batch, all_points=False):
        """Solve the RVEs of points idx (Fbar from the current F) and write sigma, D into the state;
        with all_points the batch holds every point and idx selects the rows written."""
        Fh = self._gp_F_host(None if all_points else idx)
        out = batch.solve(Fh, tangent=True)
        if all_points:
            Fh, out = Fh[idx], {"P": out["P"][idx], "A": out["A"][idx]}
        sig, D = spatial_from_PA(Fh, out["P"], out["A"])
        vals = np.ascontiguousarray(np.concatenate([sig, D], axis=1))
        q = np.ascontiguousarray(idx, np.int32)
        _check(self._L.ceos_state_scatter(self.loop.handle, len(q), _ptr(q), _ptr(vals), 27))
        return out

    max_fallback = None  # cap on points sent back to RVE solves in one material step
    point_batch_limit = 16384  # meshes up to this many points keep one warm RVE per point
    stall_level = 1e-4         # relative residual below which a stalled Newton iteration counts as converged

    def material(self, mode):
        t0 = time.perf_counter()
        _check(self._L.ceos_gp_deformation_device(self.loop.handle, C.c_void_p(self.U.data_ptr()),
                                                  C.c_void_p(self.F.data_ptr()), None))
        torch.cuda.synchronize(self.dev)
        n_fb = 0
        if mode == "surrogate":
            self.sur.material_device(self.n_elem, C.c_void_p(self.F.data_ptr()), self.n_gp,
                                     C.c_void_p(self.vf_dev.data_ptr()), C.c_void_p(self.state_ptr), self.state_f32,
                                     self.ld, C.c_void_p(self.flags.data_ptr()))
            torch.cuda.synchronize(self.dev)
            idx = torch.nonzero(self.flags).flatten().cpu().numpy()
            # a point sent to RVE solves stays there for the rest of the load step, so that no point
            # switches between the two responses from one Newton iteration to the next
            if self._sticky is not None:
                idx = np.union1d(idx, self._sticky)
            self._sticky = idx
            if self.max_fallback is not None and idx.size > self.max_fallback:
                raise FallbackLimit(f"{idx.size} of {self.n_gp} points outside the training box")
            if idx.size:
                n_fb = idx.size
                t_fb = time.perf_counter()
                if self.n_gp <= self.point_batch_limit:
                    b = self._point_batch()
                    mask = np.zeros(self.n_gp, np.int32)
                    mask[idx] = 1
                    b.set_solve_mask(mask)
                    self._rve_response(idx, b, all_points=True)
                else:
                    self._pool_response(idx)
                self.stats["fallback_s"] += time.perf_counter() - t_fb
        else:
            b = self._point_batch()
            b.set_solve_mask(None)
            self._rve_response(np.arange(self.n_gp), b, all_points=True)
            n_fb = self.n_gp
        torch.cuda.synchronize(self.dev)
        self.stats["material_s"] += time.perf_counter() - t0
        self.stats["fallback_points"] += n_fb if mode == "surrogate" else 0
        return n_fb

    # ---- Newton -------------------------------------------------------------------------------
    def predict(self, ux_target):
        """Initial guess of a load step: the homogeneous uniaxial field (e along the load axis, -e/2 across
        it) for the first step, then secant extrapolation of the last two converged fields (prescribing
        the loaded face alone would put the whole increment into one element layer)."""
        Xd = torch.as_tensor(self.X, device=self.dev)
        ax = self.axis
        L = float(self.X[:, ax].max() - self.X[:, ax].min())
        if self._hist is None:
            e = ux_target / L
            U = torch.stack([(e if d == ax else -0.5 * e) * Xd[:, d] for d in range(3)], dim=1).reshape(-1)
        else:
            (u1, U1), (u0, U0) = self._hist
            U = U1 + (U1 - U0) * ((ux_target - u1) / (u1 - u0)) if u1 != u0 else U1.clone()
        U[self.mask.bool()] = 0.0
        self.U.copy_(U)

    _hist = None  # (ux, U) of the last two converged steps
    _sticky = None  # points on RVE solves in the current load step

    def newton_step(self, ux_target, mode, tol=1e-6, max_newton=15, pcg_tol=1e-8):
        """One load step: displacement ux_target of the loaded face along the load axis; returns Newton
        iterations."""
        self.predict(ux_target)
        self._sticky = None
        self.U[torch.as_tensor(self.presc, device=self.dev)] = ux_target
        it = self._newton(mode, tol, max_newton, pcg_tol)
        prev = self._hist[0] if self._hist is not None else (0.0, torch.zeros_like(self.U))
        self._hist = ((ux_target, self.U.clone()), prev)
        return it

    def _newton(self, mode, tol, max_newton, pcg_tol):
        r0 = None
        rprev = float("inf")
        for it in range(max_newton + 1):
            self.material(mode)
            t0 = time.perf_counter()
            self.loop.evaluate_device(0.0, self.U, self.fint, self.kval)
            torch.cuda.synchronize(self.dev)
            rc, nf = self.loop.status()
            if rc:
                raise CeosError(rc, f"{nf} macro elements folded")
            self.stats["loop_s"] += time.perf_counter() - t0
            torch.neg(self.fint, out=self.rhs)
            self.rhs[self.mask.bool()] = 0.0
            rn = float(torch.linalg.vector_norm(self.rhs))
            r0 = rn if r0 is None else r0
            # The stresses of a surrogate point carry FP32 round-off (about 1e-7 relative), which puts a
            # floor under the residual: below stall_level * r0, an iteration that no longer halves the
            # residual has reached it and ends the step.
            stalled = it >= 2 and rn <= self.stall_level * r0 and rn > 0.5 * rprev
            rprev = rn
            if rn <= tol * max(r0, 1e-300) or rn <= 1e-12 or stalled:
                return it
            if it == max_newton:
                break
            t0 = time.perf_counter()
            iters, rel = C.c_int(), C.c_double()
            # inexact Newton: the linear solve only needs to beat the Newton contraction
            lin_tol = max(pcg_tol, min(1e-3, 0.1 * rn / r0))
            rc = self._L.ceos_pcg_solve(self._pcg, C.c_void_p(self.kval.data_ptr()), C.c_void_p(self.mask.data_ptr()),
                                        C.c_void_p(self.rhs.data_ptr()), C.c_void_p(self.dU.data_ptr()), lin_tol,
                                        20000, C.byref(iters), C.byref(rel))
            if rc and rel.value > max(1e-4, 10 * lin_tol):
                raise CeosError(rc, f"macro PCG stalled at relative residual {rel.value:.2e}")
            self.stats["pcg_iters"] += iters.value
            self.U += self.dU
            torch.cuda.synchronize(self.dev)
            self.stats["solve_s"] += time.perf_counter() - t0
        raise CeosError(1, f"macro Newton did not converge (residual {rn:.3e}, first {r0:.3e})")

    def run(self, stretch=1.2, n_steps=10, mode="surrogate", tol=1e-6, max_newton=15):
        """Uniaxial stretch of the loaded face to `stretch` in n_steps increments.  Returns per-step wall
        times (s), Newton iterations and fallback points."""
        L = self.X[:, self.axis].max() - self.X[:, self.axis].min()
        times, its, fbs = [], [], []
        for k in range(1, n_steps + 1):
            fb0 = self.stats["fallback_points"]
            torch.cuda.synchronize(self.dev)
            t0 = time.perf_counter()
            its.append(self.newton_step((stretch - 1.0) * L * k / n_steps, mode, tol, max_newton))
            torch.cuda.synchronize(self.dev)
            times.append(time.perf_counter() - t0)
            fbs.append(self.stats["fallback_points"] - fb0)
        return {"step_s": np.array(times), "newton": np.array(its), "fallback_points": np.array(fbs)}

    def gp_first_piola(self):
        """First Piola stress at every Gauss point [n_gp,3,3] from the state (sigma) and F."""
        st = self.loop.state(0)  # [n_elem, 8, 27]
        sig6 = np.transpose(st[:, :, :6], (1, 0, 2)).reshape(self.n_gp, 6)
        sig = np.zeros((self.n_gp, 3, 3))
        for p, (i, j) in enumerate(zip(_VI, _VJ)):
            sig[:, i, j] = sig6[:, p]
            sig[:, j, i] = sig6[:, p]
        F = self._gp_F_host()
        J = np.linalg.det(F)
        return J[:, None, None] * np.einsum("nij,nKj->niK", sig, np.linalg.inv(F))

    def close(self):
        if getattr(self, "_pcg", None):
            self._L.ceos_pcg_destroy(self._pcg)
            self._pcg = None
        if self._direct is not None:
            self._direct.close()
            self._direct = None
        if self._pool is not None:
            self._pool.close()
            self._pool = None
        self.loop.close()
