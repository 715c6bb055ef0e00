"""FP64 CPU oracle of one periodic RVE (TEST INFRASTRUCTURE ONLY).

Restates the periodic micro problem the batched GPU solver handles (fibre cells with
partial-volume moduli, mu_e = phi mu_f + (1 - phi) mu_m and likewise the bulk modulus): the reference's periodic
multiscale model eliminates the slave DOFs with a matrix T and solves T^T K T du = -T^T R
(FEM/Modules/ModMultiscalePeriodicFEMSoE.f90:77-182), then homogenizes the first Piola stress
(HomogenizeStress, MultiScale/ModMultiscaleAnalysis.f90:140-329).  Here u = (Fbar - I) X + T w
with w the periodic fluctuation of the independent nodes, one independent node held fixed, the
element loop and HomogenizeStress taken from the C++ oracle and the reduced systems solved with
scipy's sparse LU.  The tangent is checked by central finite differences of Pbar(Fbar).
"""
import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import oracle as O


def fibre_fraction(n, rad2):
    """[n][n] fibre area fraction of cell column (i, j): share of 16 x 16 sub-points of its
    cross-section strictly inside x^2 + y^2 < rad2 about the RVE centre."""
    sub = (np.arange(16) + 0.5) / 16.0
    phi = np.zeros((n, n))
    for j in range(n):
        for i in range(n):
            x = (i + sub[None, :]) / n - 0.5
            y = (j + sub[:, None]) / n - 0.5
            phi[j, i] = np.count_nonzero(x * x + y * y < rad2) / 256.0
    return phi


def rve_mesh(n, vf):
    """Unit cube, n^3 cells, fibre along z through the centre; per-cell fibre fraction phi
    (partial-volume cells)."""
    m = n + 1
    k, j, i = np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij")
    X = np.stack([i.ravel() / n, j.ravel() / n, k.ravel() / n], axis=1)
    ke, je, ie = [a.ravel() for a in np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")]

    def nid(a, b, c):
        return (c * m + b) * m + a + 1

    conn = np.stack([nid(ie, je, ke), nid(ie + 1, je, ke), nid(ie + 1, je + 1, ke), nid(ie, je + 1, ke),
                     nid(ie, je, ke + 1), nid(ie + 1, je, ke + 1), nid(ie + 1, je + 1, ke + 1),
                     nid(ie, je + 1, ke + 1)], axis=1).astype(np.int32)
    phi = fibre_fraction(n, vf / np.pi)[je, ie]
    ind = ((k % n) * n * n + (j % n) * n + (i % n)).ravel()
    return X, conn, phi, ind


class RVE:
    def __init__(self, n, vf, mu_m=1.0, ratio=50.0, k_over_mu=100.0):
        self.X, self.conn, self.phi, ind = rve_mesh(n, vf)
        mu_f = ratio * mu_m
        # cell moduli mixed by fibre fraction (same operation order as the GPU set-up)
        mu_e = self.phi * mu_f + (1.0 - self.phi) * mu_m
        k_e = self.phi * (k_over_mu * mu_f) + (1.0 - self.phi) * (k_over_mu * mu_m)
        params = np.stack([mu_e, k_e - 2.0 * mu_e / 3.0], axis=1)
        self.model = O.Model(self.X, self.conn, [O.CNH], params, per_element=True)
        self.rowmap, self.col = self.model.pattern()
        nn = self.X.shape[0]
        # T: full dof (3a+d) <- reduced dof 3(ind-1)+d, independent node 0 fixed
        rows, cols = [], []
        for a in range(nn):
            if ind[a] == 0:
                continue
            for d in range(3):
                rows.append(3 * a + d)
                cols.append(3 * (ind[a] - 1) + d)
        self.n_red = 3 * (n ** 3 - 1)
        self.T = sp.csr_matrix((np.ones(len(rows)), (rows, cols)), shape=(3 * nn, self.n_red))
        self.vf_actual = self.phi.mean()

    def _K(self, kval):
        n = 3 * self.X.shape[0]
        r = np.repeat(np.arange(n), np.diff(self.rowmap))
        c = self.col - 1
        K = sp.csr_matrix((kval, (r, c)), shape=(n, n))
        return (K + K.T - sp.diags(K.diagonal())).tocsr()

    def solve(self, Fbar, tol=1e-10, itmax=25):
        Fbar = np.asarray(Fbar, dtype=np.float64).reshape(3, 3)
        w = np.zeros(self.n_red)
        aff = (self.X @ (Fbar - np.eye(3)).T).reshape(-1)
        r0 = None
        for it in range(itmax):
            U = aff + self.T @ w
            fint, kval, rc, _ = self.model.evaluate(0.0, U)
            assert rc == 0
            R = self.T.T @ fint
            nr = np.linalg.norm(R)
            r0 = nr if r0 is None else r0
            # relative to the first residual, with a floor at round-off of the internal forces
            if nr <= tol * max(r0, 1e-300) or nr <= 1e-11 * np.linalg.norm(fint):
                break
            Kred = (self.T.T @ self._K(kval) @ self.T).tocsc()
            w -= spla.spsolve(Kred, R)
        self.U = U
        self.iters = it
        return self.model.homogenize(U)

    def tangent_fd(self, Fbar, h=1e-6):
        A = np.zeros((9, 9))
        for kL in range(9):
            dF = np.zeros(9)
            dF[kL] = h
            Pp = self.solve(np.asarray(Fbar).reshape(-1) + dF).reshape(-1)
            Pm = self.solve(np.asarray(Fbar).reshape(-1) - dF).reshape(-1)
            A[:, kL] = (Pp - Pm) / (2 * h)
        return A


def reference_periodic_T(X, tol=1e-6):
    """The periodic map T of the reference's BuildT (FEM/Modules/ModMultiscalePeriodicFEMSoE.f90:226-895),
    restated: boundary nodes are classified by coordinates (tolerance 1e-6) into the minus/plus faces,
    edges and the 8 vertices; every plus node is tied to the minus node with the same remaining
    coordinates (T row of the plus dof = the minus node's column, its own column nulled), the 7 other
    vertices to XmYmZm, and the nulled columns are removed (the NulCols compaction, :854-871).  Returns
    (T [3 n_nodes x n_red] sparse, the 24 full vertex dofs that the analysis fixes, :874-897 with
    ModFEMAnalysis.f90:1526-1535).

    One branch of the reference is restated by its evident intent: for the YpZm edge (:775-783) the
    reference zeroes only two of the node's diagonal entries and records Xp(n) instead of YpZm(n) in
    NulCols; here the YpZm node is tied like the YmZp and YpZp edges."""
    n = X.shape[0]
    lo, hi = X.min(axis=0), X.max(axis=0)
    at_lo = np.abs(X - lo) < tol
    at_hi = np.abs(X - hi) < tol
    on_b = at_lo | at_hi
    minus_of = np.arange(n)                       # independent partner of every node
    key = {}
    for a in range(n):                            # minus-side representatives by reduced coordinates
        if not on_b[a].any():
            continue
        if at_hi[a].any():
            continue
        key[tuple(np.round(np.where(at_lo[a], -1.0, X[a]) / tol).astype(np.int64))] = a
    for a in range(n):
        if not at_hi[a].any():
            continue
        # the partner lies on the minus side of every axis on which a lies on the plus side
        q = np.where(at_hi[a] | at_lo[a], -1.0, X[a])
        minus_of[a] = key[tuple(np.round(q / tol).astype(np.int64))]
    rows, cols = [], []
    keep = np.ones(3 * n, bool)
    for a in range(n):
        if minus_of[a] != a:
            keep[3 * a:3 * a + 3] = False
    newcol = np.cumsum(keep) - 1
    for a in range(n):
        m = minus_of[a]
        for d in range(3):
            rows.append(3 * a + d)
            cols.append(newcol[3 * m + d])
    T = sp.csr_matrix((np.ones(len(rows)), (rows, cols)), shape=(3 * n, int(keep.sum())))
    vert = np.nonzero(on_b.all(axis=1))[0]
    vdofs = np.array([3 * a + d for a in vert for d in range(3)])
    return T, vdofs


class RVEReference(RVE):
    """One periodic RVE solved in the reference's periodic formulation: u = (Fbar - I) Y + T w with the
    reference's T (reference_periodic_T), the vertex dofs fixed by the rows and columns of
    ApplyBoundaryConditionsNEW (zero, unit diagonal, zero residual), the reduced system T^T K T and
    residual T^T R of EvaluateKt (ModMultiscalePeriodicFEMSoE.f90:77-182), Taylor displacement as the
    first iterate (ExpandFluctuation, :190-222), and HomogenizeStress.

    The reference also sets FMacroFinal(3,3) = 1/(F11 F22) (MultiScale/ModMultiscaleBoundaryConditions.f90:260),
    but no later statement reads FMacroFinal: the prescribed displacements use FMacroInitial and
    DeltaFMacro only.  The override therefore has no effect and is not restated."""

    def __init__(self, n, vf, **kw):
        super().__init__(n, vf, **kw)
        self.T, self.vdofs = reference_periodic_T(self.X)
        self.n_red = self.T.shape[1]

    def solve(self, Fbar, tol=1e-10, itmax=25):
        Fbar = np.asarray(Fbar, dtype=np.float64).reshape(3, 3)
        w = np.zeros(self.n_red)
        aff = (self.X @ (Fbar - np.eye(3)).T).reshape(-1)
        nfull = aff.size
        fixed = np.zeros(nfull, bool)
        fixed[self.vdofs] = True
        keepm = sp.diags((~fixed).astype(float))
        r0 = None
        for it in range(itmax):
            U = aff + self.T @ w
            fint, kval, rc, _ = self.model.evaluate(0.0, U)
            assert rc == 0
            Rf = -fint
            Rf[fixed] = 0.0
            R = self.T.T @ Rf
            nr = np.linalg.norm(R)
            r0 = nr if r0 is None else r0
            if nr <= tol * max(r0, 1e-300) or nr <= 1e-11 * np.linalg.norm(fint):
                break
            K = self._K(kval)
            Km = (keepm @ K @ keepm + sp.diags(fixed.astype(float))).tocsr()
            Kred = (self.T.T @ Km @ self.T).tocsc()
            w += spla.spsolve(Kred, R)
        self.U = U
        self.iters = it
        return self.model.homogenize(U)
