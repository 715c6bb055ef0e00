"""Failure detection of the fused assembly without a GPU fault.  Every flag wait of
element_assemble_kernel is bounded (200 ms of %globaltimer); when one runs out the kernel sets an
error word, every other waiter gives up too, the launch ends, and ceos_status reports CEOS_E_CUDA.
The test makes one conversion item wait for a flag that nothing sets (ceos_test_stall_conversion),
checks the reported status and the message, restores the item and checks that the next evaluation,
which clears the partly accumulated blocks, gives the same f_int and K as before the failure."""
import numpy as np
import pytest

import ceos_b200 as G
from ceos_b200 import meshgen

pytestmark = pytest.mark.gpu

CNH_P = [1.0, 100.0 - 2.0 / 3.0]


def test_fused_assembly_wait_that_runs_out_reports_an_error_and_recovers():
    import torch
    X, conn = meshgen.structured_box(24, 24, 24, jitter=0.05, seed=4)
    g = G.ElementLoop(X, conn, G.CNH, CNH_P, precision=G.MIXED)
    try:
        g.set_assembly("fused")
        x, y, z = X[:, 0], X[:, 1], X[:, 2]  # a smooth deformation, |grad u| <= 0.2
        U = 0.03 * np.stack([np.sin(2 * np.pi * y), np.sin(2 * np.pi * z), np.sin(2 * np.pi * x)], 1).reshape(-1)
        dU = torch.tensor(U, dtype=torch.float64, device="cuda")
        df = torch.zeros(g.n_dof, dtype=torch.float64, device="cuda")
        dk = torch.zeros(g.nnz, dtype=torch.float64, device="cuda")

        def run():
            g.evaluate_device(0.0, dU, df, dk)
            torch.cuda.synchronize()
            return g.status()

        assert run() == (0, 0)
        f0, k0 = df.cpu().numpy().copy(), dk.cpu().numpy().copy()
        g.test_stall_conversion(3, True)
        rc, _ = run()
        assert rc == -2  # CEOS_E_CUDA: a dependency wait exceeded its bound
        assert "wait exceeded its bound" in g.failed_elements()[1]
        g.test_stall_conversion(3, False)
        assert run() == (0, 0)
        f1, k1 = df.cpu().numpy(), dk.cpu().numpy()
        assert np.abs(f1 - f0).max() <= 1e-5 * np.abs(f0).max()
        assert np.abs(k1 - k0).max() <= 1e-5 * np.abs(k0).max()
    finally:
        g.close()
