"""Seeded synthetic Hexa8 meshes and the boundary-condition tables of the benchmark
configurations.

Node numbering is x fastest, then y, then z (1-based ids in the connectivity, as the
reference's GiD meshes).  Element node order follows the reference Hexa8
(FEM/Elements/ElementLibrary/ModElementHexa8.f90:185-192):
(-,-,-), (+,-,-), (+,+,-), (-,+,-), (-,-,+), (+,-,+), (+,+,+), (-,+,+).
"""
import numpy as np


def structured_box(nx, ny, nz, lx=1.0, ly=1.0, lz=1.0, jitter=0.05, seed=0):
    """Return (X[n_nodes,3] float64, conn[n_elem,8] int32 1-based).

    Interior nodes are moved uniformly by +-jitter*h per coordinate (h = element size along
    that axis), drawn from numpy.random.default_rng(seed); boundary nodes stay on the faces.
    """
    mx, my, mz = nx + 1, ny + 1, nz + 1
    xs = np.linspace(0.0, lx, mx)
    ys = np.linspace(0.0, ly, my)
    zs = np.linspace(0.0, lz, mz)
    Z, Y, Xg = np.meshgrid(zs, ys, xs, indexing="ij")
    X = np.stack([Xg.ravel(), Y.ravel(), Z.ravel()], axis=1)
    if jitter:
        rng = np.random.default_rng(seed)
        h = np.array([lx / nx, ly / ny, lz / nz])
        d = rng.uniform(-jitter, jitter, size=X.shape) * h
        k, j, i = np.meshgrid(np.arange(mz), np.arange(my), np.arange(mx), indexing="ij")
        interior = ((i > 0) & (i < nx) & (j > 0) & (j < ny) & (k > 0) & (k < nz)).ravel()
        X[interior] += d[interior]
    ke, je, ie = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    ie, je, ke = ie.ravel(), je.ravel(), ke.ravel()

    def nid(i, j, k):
        return (k * my + j) * mx + i + 1

    conn = np.stack([nid(ie, je, ke), nid(ie + 1, je, ke), nid(ie + 1, je + 1, ke), nid(ie, je + 1, ke),
                     nid(ie, je, ke + 1), nid(ie + 1, je, ke + 1), nid(ie + 1, je + 1, ke + 1),
                     nid(ie, je + 1, ke + 1)], axis=1).astype(np.int32)
    return X, conn


def node_grid_index(X, tol=1e-12):
    """Boolean helpers for faces of the unit box meshes."""
    return {
        "x0": np.abs(X[:, 0] - X[:, 0].min()) < tol, "x1": np.abs(X[:, 0] - X[:, 0].max()) < tol,
        "y0": np.abs(X[:, 1] - X[:, 1].min()) < tol, "y1": np.abs(X[:, 1] - X[:, 1].max()) < tol,
        "z0": np.abs(X[:, 2] - X[:, 2].min()) < tol, "z1": np.abs(X[:, 2] - X[:, 2].max()) < tol,
    }


def uniform_steps(t0, t1, n):
    """Time discretization of one load case (ModLoadHistoryData.f90:43-105)."""
    dt = (t1 - t0) / float(n)
    t_init = np.array([t0 + k * dt for k in range(n)])
    return t_init, np.full(n, dt)


def table_values(table, times):
    """Linear interpolation of a (time, value) table (LinearInterpolation in ModMathRoutines)."""
    table = np.asarray(table, dtype=np.float64)
    return np.interp(times, table[:, 0], table[:, 1])


def bc_from_tables(t_init, dt, fixed, presc, presc_tables, force, force_tables):
    """Expand per-DOF tables into the per-step initial/final arrays of GetBoundaryConditions
    (ModBoundaryConditions.f90:540-668).  DOF ids are 1-based; each *_tables entry is a
    (time, value) table for the DOF in the same position."""
    t_fin = t_init + dt
    pi = np.array([table_values(tb, t_init) for tb in presc_tables]) if len(presc) else np.zeros((0, len(t_init)))
    pf = np.array([table_values(tb, t_fin) for tb in presc_tables]) if len(presc) else np.zeros((0, len(t_init)))
    fi = np.array([table_values(tb, t_init) for tb in force_tables]) if len(force) else np.zeros((0, len(t_init)))
    ff = np.array([table_values(tb, t_fin) for tb in force_tables]) if len(force) else np.zeros((0, len(t_init)))
    return {"t0": t_init, "dt": dt, "fixed": np.asarray(fixed, np.int32), "presc": np.asarray(presc, np.int32),
            "presc_init": pi, "presc_final": pf, "force": np.asarray(force, np.int32),
            "force_init": fi, "force_final": ff}


def golden_hexa8_svk_bc(fx):
    """BCs of the reference's NonLinear_FEA_3D_Hexa8_StVenant case from its fixture."""
    t_init, dt = uniform_steps(fx["time"]["t0"], fx["time"]["t1"], fx["time"]["steps"])
    fixed = []
    for row in fx["fixed"]:
        node = row[0]
        for d in range(3):
            if row[1 + d]:
                fixed.append(3 * (node - 1) + d + 1)
    presc, ptabs = [], []
    for row in fx["disps"]:
        node = row[0]
        for d in range(3):
            flag, tab = row[1 + d]
            if flag:
                presc.append(3 * (node - 1) + d + 1)
                ptabs.append(fx["tables"][tab])
    force, ftabs = [], []
    for row in fx["loads"]:
        node = row[0]
        for d in range(3):
            flag, tab = row[1 + d]
            if flag:
                force.append(3 * (node - 1) + d + 1)
                ftabs.append(fx["tables"][tab])
    return bc_from_tables(t_init, dt, sorted(fixed), presc, ptabs, force, ftabs)


def config1_bc(X, n_steps=10, stretch=1.5, extra_rotation_constraint=True):
    """Config 1 BCs: face x=0 fixed in x, corner (0,0,0) pinned, face x=1 displaced to a
    stretch of `stretch` over n_steps equal increments.  One extra constraint, u_z = 0 at the
    corner (0,1,0), removes the rigid rotation about the x-axis through the pinned corner that
    the stated BCs leave free."""
    f = node_grid_index(X)
    t_init, dt = uniform_steps(0.0, 1.0, n_steps)
    L = X[:, 0].max() - X[:, 0].min()
    fixed = set()
    for n in np.nonzero(f["x0"])[0]:
        fixed.add(3 * n + 1)
    corner = np.nonzero(f["x0"] & f["y0"] & f["z0"])[0][0]
    for d in range(3):
        fixed.add(3 * corner + d + 1)
    if extra_rotation_constraint:
        c2 = np.nonzero(f["x0"] & f["y1"] & f["z0"])[0][0]
        fixed.add(3 * c2 + 3)
    presc = [3 * n + 1 for n in np.nonzero(f["x1"])[0]]
    tab = [[0.0, 0.0], [1.0, (stretch - 1.0) * L]]
    return bc_from_tables(t_init, dt, sorted(fixed), presc, [tab] * len(presc), [], [])


def config2_bc(X, n_steps=40, dt=0.025, amplitude=0.3, freq=1.0):
    """Config 2 BCs (project-chosen): cyclic simple shear gamma(t) = amplitude sin(2 pi freq t) of the
    unit cube; bottom face z = 0 fixed, top face z = 1 moved by u_x = gamma(t) (times its height) with
    u_y = u_z = 0; n_steps increments of dt, the table holding gamma at every step end."""
    f = node_grid_index(X)
    t_init = np.array([k * dt for k in range(n_steps)])
    H = X[:, 2].max() - X[:, 2].min()
    fixed = set()
    for n in np.nonzero(f["z0"])[0]:
        for d in range(3):
            fixed.add(3 * n + d + 1)
    top = np.nonzero(f["z1"])[0]
    for n in top:
        fixed.add(3 * n + 2)
        fixed.add(3 * n + 3)
    tk = np.arange(n_steps + 1) * dt
    tab = np.stack([tk, amplitude * np.sin(2.0 * np.pi * freq * tk) * H], axis=1).tolist()
    presc = [3 * n + 1 for n in top]
    return bc_from_tables(t_init, np.full(n_steps, dt), sorted(fixed), presc, [tab] * len(presc), [], [])


def config3_bc(X, n_steps=50, strain=0.05):
    """Config 3 BCs: uniaxial tension of the plate along x to `strain` (engineering) in n_steps equal
    increments of pseudo-time [0, 1]: face x = 0 has u_x = 0, the symmetry planes y = 0 and z = 0
    have u_y = 0 and u_z = 0, face x = L is displaced by strain * L."""
    f = node_grid_index(X)
    t_init, dt = uniform_steps(0.0, 1.0, n_steps)
    L = X[:, 0].max() - X[:, 0].min()
    fixed = set()
    for n in np.nonzero(f["x0"])[0]:
        fixed.add(3 * n + 1)
    for n in np.nonzero(f["y0"])[0]:
        fixed.add(3 * n + 2)
    for n in np.nonzero(f["z0"])[0]:
        fixed.add(3 * n + 3)
    presc = [3 * n + 1 for n in np.nonzero(f["x1"])[0]]
    tab = [[0.0, 0.0], [1.0, strain * L]]
    return bc_from_tables(t_init, dt, sorted(fixed), presc, [tab] * len(presc), [], [])
