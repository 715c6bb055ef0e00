"""Surrogate kernels on the GPU against the FP64 oracle: the BF16 tensor-core training gradient, with
the 128-wide layer GEMMs on tcgen05 (TMEM accumulators) and on mma.sync (oracle with the same BF16
rounding points: 2e-3; plain FP64: 3e-2 relative in norm; 700 samples, so the last 128-sample tile
is partial), the FP32
inference of stress and tangent (1e-4 relative), the training-box flag, and a training run on
an analytic energy."""
import numpy as np
import pytest

import surrogate_oracle as SO
from ceos_b200 import surrogate as SG

pytestmark = pytest.mark.gpu


def _problem(n=700, seed=3):
    rng = np.random.default_rng(seed)
    th = SO.init_params(5) * 0.8
    x = rng.uniform(-1, 1, (n, 7))
    t = rng.normal(scale=0.5, size=(n, 6))
    w = np.array([4.0, 4.0, 4.0, 1.0, 1.0, 1.0])
    return th, x, t, w


@pytest.mark.parametrize("gemm", ["mma", "tcgen05"])
def test_training_gradient_matches_oracle(gemm):
    th, x, t, w = _problem()
    s = SG.Surrogate(batch_max=1024)
    s.set_gemm(gemm)
    s.set_params(th)
    th32 = s.params().astype(np.float64)
    sw = np.random.default_rng(4).uniform(0.2, 3.0, len(x)).astype(np.float32)  # per-sample weights
    loss, g = s.gradient(x, t, w, sw)
    Lb, gb = SO.loss_and_grad(th32, x.astype(np.float32).astype(np.float64), t.astype(np.float32).astype(np.float64),
                              w, bf=True, sw=sw)
    L64, g64 = SO.loss_and_grad(th32, x, t, w, sw=sw)
    assert abs(loss - Lb) <= 1e-4 * Lb
    assert np.linalg.norm(g - gb) <= 2e-3 * np.linalg.norm(gb)
    assert np.linalg.norm(g - g64) <= 3e-2 * np.linalg.norm(g64)
    # every parameter block, not just the norm
    o = 0
    for name, shp in SO.SHAPES[:-1]:
        k = int(np.prod(shp))
        assert np.linalg.norm(g[o:o + k] - gb[o:o + k]) <= 5e-3 * np.linalg.norm(gb[o:o + k]) + 1e-7, name
        o += k
    s.close()


def test_inference_matches_oracle_and_flags_range():
    th, _, _, _ = _problem()
    s = SG.Surrogate(batch_max=256)
    s.set_params(th)
    sC, sW, vf0, svf = 0.15, 2.0, 0.25, 0.15
    s.set_scaling(sC, sW, vf0, svf, lo=-np.ones(7), hi=np.ones(7))
    rng = np.random.default_rng(9)
    F = np.eye(3) + rng.uniform(-0.12, 0.12, (300, 3, 3))
    C6 = SG.voigt_C(F)
    vf = rng.uniform(0.1, 0.4, 300)
    S, Cm, fl = s.evaluate(C6, vf)
    x = s.inputs(C6, vf)
    So, Co = SO.stress_tangent(s.params().astype(np.float64), x, sC, sW)
    assert np.abs(S - So).max() <= 1e-4 * np.abs(So).max()
    assert np.abs(Cm - Co).max() <= 1e-4 * np.abs(Co).max()
    assert np.abs(Cm - np.transpose(Cm, (0, 2, 1))).max() <= 1e-12 * np.abs(Cm).max()
    np.testing.assert_array_equal(fl, np.any(np.abs(x) > 1.0, axis=1))
    s.close()


def test_training_fits_analytic_energy():
    """Train on the stress of a vf-dependent compressible Neo-Hookean energy; the fitted
    network reproduces it to a few percent and the loss falls by two orders of magnitude."""
    rng = np.random.default_rng(0)
    n = 16384
    F = np.eye(3) + rng.uniform(-0.15, 0.15, (n, 3, 3))
    F = F[np.linalg.det(F) > 0.5]
    vf = rng.uniform(0.1, 0.4, len(F))
    mu = 1.0 + 10.0 * vf
    lam = 20.0 * mu
    Cinv = np.linalg.inv(np.einsum("nki,nkj->nij", F, F))
    lnJ = np.log(np.linalg.det(F))
    Sm = mu[:, None, None] * (np.eye(3) - Cinv) + (lam * lnJ)[:, None, None] * Cinv
    S6 = np.stack([Sm[:, i, j] for i, j in SG._IJ], axis=1)
    sC, vf0, svf = 0.15, 0.25, 0.15
    sW = np.sqrt(np.mean(S6 ** 2)) * sC
    s = SG.Surrogate(batch_max=1024)
    s.set_params(SO.init_params(2).astype(np.float32))
    s.set_scaling(sC, sW, vf0, svf)
    C6 = SG.voigt_C(F)
    x = s.inputs(C6, vf)
    t = S6 / (SG.VOIGT_A * (sW / sC))
    hist = s.train(x, t, SG.VOIGT_A ** 2, epochs=40, batch=1024, lr0=3e-3, lr1=1e-4, seed=1)
    assert np.all(np.isfinite(hist))
    assert hist[-1] < 1e-2 * hist[0]
    Sp, _, _ = s.evaluate(C6[:2000], vf[:2000])
    err = np.linalg.norm(Sp - S6[:2000], axis=1) / np.linalg.norm(S6[:2000], axis=1).mean()
    assert np.median(err) < 0.03
    s.close()


def test_reference_state_is_stress_free_and_tangent_unchanged():
    th, _, _, _ = _problem()
    s = SG.Surrogate(batch_max=256)
    s.set_params(th)
    s.set_scaling(0.15, 2.0, 0.25, 0.15)
    rng = np.random.default_rng(2)
    vf = rng.uniform(0.1, 0.4, 50)
    F = np.eye(3) + rng.uniform(-0.1, 0.1, (50, 3, 3))
    S_a, C_a, _ = s.evaluate(SG.voigt_C(F), vf)
    I6 = np.tile([1.0, 1.0, 1.0, 0.0, 0.0, 0.0], (50, 1))
    S_I, _, _ = s.evaluate(I6, vf)
    s.set_reference(0.1, 0.4)
    S_b, C_b, _ = s.evaluate(SG.voigt_C(F), vf)
    S_I2, _, _ = s.evaluate(I6, vf)
    assert np.abs(S_I2).max() <= 1e-4 * np.abs(S_I).max()          # table interpolation in vf
    np.testing.assert_array_equal(C_a, C_b)                           # the tangent is untouched
    assert np.abs((S_a - S_b) - S_I).max() <= 1e-4 * np.abs(S_I).max()
    s.close()


def test_tcgen05_and_mma_gradients_agree():
    """The two GEMM paths see the same BF16 operands and accumulate in FP32: their gradients differ only
    by summation order and the BF16 rounding it can flip (1e-3 relative in norm)."""
    th, x, t, w = _problem(n=1024, seed=8)
    out = {}
    for gemm in ("mma", "tcgen05"):
        s = SG.Surrogate(batch_max=1024)
        s.set_gemm(gemm)
        s.set_params(th)
        out[gemm] = s.gradient(x, t, w)
        s.close()
    (la, ga), (lb, gb) = out["mma"], out["tcgen05"]
    assert abs(la - lb) <= 1e-5 * la
    assert np.linalg.norm(ga - gb) <= 1e-3 * np.linalg.norm(ga)
