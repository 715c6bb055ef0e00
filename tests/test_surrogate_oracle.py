"""CPU checks of the FP64 surrogate oracle that checks the GPU training and inference kernels:
its double-backprop parameter gradient, input gradient and Hessian against central finite
differences."""
import numpy as np

import surrogate_oracle as SO


def _setup(seed=0, n=5):
    th = SO.init_params(1) * 0.7
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, (n, 7))
    t = rng.normal(size=(n, 6))
    w = rng.uniform(0.5, 2, 6)
    return th, x, t, w, rng


def test_loss_gradient_matches_finite_differences():
    th, x, t, w, rng = _setup()
    sw = rng.uniform(0.5, 2.0, len(x))
    _, gr = SO.loss_and_grad(th, x, t, w, sw=sw)
    idx = rng.choice(SO.N_PARAMS, 40, replace=False)
    h = 1e-6
    fd = []
    for i in idx:
        e = np.zeros(SO.N_PARAMS)
        e[i] = h
        fd.append((SO.loss_and_grad(th + e, x, t, w, sw=sw)[0] - SO.loss_and_grad(th - e, x, t, w, sw=sw)[0]) / (2 * h))
    assert np.abs(np.array(fd) - gr[idx]).max() <= 1e-5 * np.abs(gr[idx]).max()


def test_input_gradient_and_hessian_match_finite_differences():
    th, x, _, _, _ = _setup(1)
    h = 1e-6
    _, g, Hs = SO.energy_grad_hess(th, x)
    fdg = np.stack([(SO.energy_grad_hess(th, x + h * np.eye(7)[k])[0] - SO.energy_grad_hess(th, x - h * np.eye(7)[k])[0])
                    / (2 * h) for k in range(7)], axis=1)
    assert np.abs(fdg - g).max() <= 1e-6 * np.abs(g).max()
    fdH = np.stack([(SO.energy_grad_hess(th, x + h * np.eye(7)[k])[1] - SO.energy_grad_hess(th, x - h * np.eye(7)[k])[1])
                    / (2 * h) for k in range(7)], axis=2)
    assert np.abs(fdH - Hs).max() <= 1e-6 * np.abs(Hs).max()
    assert np.abs(Hs - np.transpose(Hs, (0, 2, 1))).max() <= 1e-14 * np.abs(Hs).max()


def test_bf16_rounding_is_round_to_nearest_even():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 3.0e-3])
    r = SO.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6  # ties to even
    assert r[3] == -2.5
    assert abs(r[4] - 3.0e-3) <= 2 ** -8 * 3.0e-3  # 8 significant bits
