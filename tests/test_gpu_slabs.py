"""The host-buffer call (ceos_evaluate) computes in element slabs and copies every finished node-row
prefix to the host while later slabs run.  Its f_int and K equal those of the single-launch device
call (ceos_evaluate_device) up to the summation order of the atomics, for a sweep numbering (rows
finish slab by slab) and for a scrambled one (rows finish only at the end); in mixed precision with
the three K assemblies (two-pass: element loop then conversion per slab; fused: one launch per slab;
banded: element bands on two streams and each band's conversion on a third, rows copied band by band,
two to four bands on these meshes)."""
import numpy as np
import pytest

import ceos_b200 as G
from ceos_b200 import meshgen

pytestmark = pytest.mark.gpu

CNH_P = [1.0, 100.0 - 2.0 / 3.0]


def _mesh(n, scramble):
    X, conn = meshgen.structured_box(n, n, n, jitter=0.05, seed=1)
    if scramble:
        p = np.random.default_rng(5).permutation(len(X))
        Xp = np.empty_like(X)
        Xp[p] = X
        X, conn = Xp, p[conn - 1] + 1
    return X, conn


@pytest.mark.parametrize("n,scramble", [(32, False), (40, True)])
# f_int accumulates in FP64 in both modes (1e-12); mixed-precision K differs between the two calls only
# by the order of the FP32 reductions: at most 2.7e-7 of the largest entry measured on a B200
@pytest.mark.parametrize("precision,ftol,ktol,assembly", [(G.FP64, 1e-12, 1e-12, None),
                                                          (G.MIXED, 1e-12, 1e-6, "two-pass"),
                                                          (G.MIXED, 1e-12, 1e-6, "fused"),
                                                          (G.MIXED, 1e-12, 1e-6, "banded")])
def test_slab_pipelined_host_call_equals_device_call(n, scramble, precision, ftol, ktol, assembly):
    import torch
    X, conn = _mesh(n, scramble)
    g = G.ElementLoop(X, conn, G.CNH, CNH_P, precision=precision)
    try:
        if assembly:
            g.set_assembly(assembly)
        # a smooth deformation (|grad u| <= 0.2) plus a small nodal jitter
        x, y, z = X[:, 0], X[:, 1], X[:, 2]
        rng = np.random.default_rng(2)
        U = (0.03 * np.stack([np.sin(2 * np.pi * y), np.sin(2 * np.pi * z), np.sin(2 * np.pi * x)], 1).reshape(-1)
             + 1e-4 * rng.standard_normal(3 * len(X)))
        f_h, k_h, rc, _ = g.evaluate(0.1, U)
        assert rc == 0
        dU = torch.tensor(U, dtype=torch.float64, device="cuda")
        df = torch.zeros(g.n_dof, dtype=torch.float64, device="cuda")
        dk = torch.zeros(g.nnz, dtype=torch.float64, device="cuda")
        g.evaluate_device(0.1, dU, df, dk)
        torch.cuda.synchronize()
        f_d, k_d = df.cpu().numpy(), dk.cpu().numpy()
        assert np.abs(f_h - f_d).max() <= ftol * np.abs(f_d).max()
        assert np.abs(k_h - k_d).max() <= ktol * np.abs(k_d).max()
        # every K entry was written by the host call: a second call into fresh zeros gives K again
        # (an entry the call skipped would stay 0; exact zero counts are not compared, since a sum of
        # FP32 contributions may cancel to 0.0 in one atomic order and not in another)
        f_h2, k_h2, _, _ = g.evaluate(0.1, U)
        assert np.abs(k_h2 - k_d).max() <= ktol * np.abs(k_d).max()
    finally:
        g.close()
