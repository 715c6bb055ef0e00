"""Learned FE^2 surrogate (C ABI ceos_sur_*): an MLP energy of (C, vf) trained on the GPU by
BF16 tensor-core kernels on stresses the batched RVE solver produces, evaluated by an FP32
kernel that returns S and the material tangent, with a training-box check that routes points
outside it back to the RVE solve."""
import ctypes as C

import numpy as np

from . import CeosError, _ptr, lib

VOIGT_A = np.array([2.0, 2.0, 2.0, 1.0, 1.0, 1.0])
_IJ = [(0, 0), (1, 1), (2, 2), (0, 1), (1, 2), (0, 2)]


def _setup():
    L = lib()
    P, I, D, F = C.c_void_p, C.c_int, C.c_double, C.c_float
    L.ceos_sur_create.argtypes = [I, I, C.POINTER(P)]
    L.ceos_sur_n_params.restype = I
    L.ceos_sur_set_params.argtypes = [P, P]
    L.ceos_sur_get_params.argtypes = [P, P]
    L.ceos_sur_set_scaling.argtypes = [P, P, P, P]
    L.ceos_sur_gradient.argtypes = [P, I, P, P, P, P, P, P]
    L.ceos_sur_train.argtypes = [P, I, P, P, P, P, I, I, D, D, C.c_uint, P]
    L.ceos_sur_evaluate.argtypes = [P, I, P, P, P, P, P]
    L.ceos_sur_material_device.argtypes = [P, I, P, C.c_longlong, P, P, I, C.c_longlong, P, P]
    L.ceos_sur_set_reference.argtypes = [P, D, D]
    L.ceos_sur_message.argtypes = [P, C.c_char_p, I]
    L.ceos_sur_set_gemm.argtypes = [P, I]
    L.ceos_sur_destroy.argtypes = [P]
    L.ceos_sur_destroy.restype = None
    return L


def voigt_C(F):
    """Right Cauchy-Green tensors [N,6] (C11, C22, C33, C12, C23, C13) of F [N,3,3]."""
    Cm = np.einsum("nki,nkj->nij", F, F)
    return np.stack([Cm[:, i, j] for i, j in _IJ], axis=1)


def voigt_S_from_P(F, P):
    """Second Piola stress S = F^-1 P (symmetric part) in Voigt order, [N,6]."""
    S = np.linalg.solve(F, P)
    S = 0.5 * (S + np.transpose(S, (0, 2, 1)))
    return np.stack([S[:, i, j] for i, j in _IJ], axis=1)


class Surrogate:
    """MLP energy surrogate on one GPU.  Scaling: x = [(C - I)/s_C, (vf - vf0)/s_vf] and
    S = a (s_W/s_C) de/dx; set_scaling() also fixes the training box used by the range check."""

    def __init__(self, batch_max=8192, device=0):
        self._L = _setup()
        h = C.c_void_p()
        rc = self._L.ceos_sur_create(batch_max, device, C.byref(h))
        if rc:
            raise CeosError(rc, "ceos_sur_create")
        self._h = h
        self.n_params = self._L.ceos_sur_n_params()
        self.batch_max = batch_max
        self.scales = np.array([0.15, 1.0, 0.25, 0.15])

    def _check(self, rc):
        if rc:
            buf = C.create_string_buffer(256)
            self._L.ceos_sur_message(self._h, buf, 256)
            raise CeosError(rc, buf.value.decode())

    def set_gemm(self, path):
        """128-wide layer GEMMs of training: "tcgen05" (the default: tensor cores, TMEM accumulators, the
        four passes of 128 samples in one launch) or "mma" (mma.sync on warps, one launch per layer)."""
        self._check(self._L.ceos_sur_set_gemm(self._h, {"mma": 0, "tcgen05": 1}[path]))

    def set_params(self, theta):
        th = np.ascontiguousarray(theta, dtype=np.float32)
        assert th.size == self.n_params
        self._check(self._L.ceos_sur_set_params(self._h, _ptr(th)))

    def params(self):
        th = np.zeros(self.n_params, np.float32)
        self._check(self._L.ceos_sur_get_params(self._h, _ptr(th)))
        return th

    def set_scaling(self, s_C, s_W, vf0, s_vf, lo=None, hi=None):
        self.scales = np.array([s_C, s_W, vf0, s_vf], np.float64)
        lo = None if lo is None else np.ascontiguousarray(lo, np.float64)
        hi = None if hi is None else np.ascontiguousarray(hi, np.float64)
        self._check(self._L.ceos_sur_set_scaling(self._h, _ptr(self.scales), _ptr(lo) if lo is not None else None,
                                                 _ptr(hi) if hi is not None else None))

    def set_reference(self, vf_lo, vf_hi):
        """Make C = I stress-free for vf in [vf_lo, vf_hi] (subtracts the tabulated S(I, vf))."""
        self._check(self._L.ceos_sur_set_reference(self._h, vf_lo, vf_hi))

    def inputs(self, C6, vf):
        s_C, _, vf0, s_vf = self.scales
        x = np.zeros((len(vf), 7))
        x[:, :6] = (C6 - np.array([1, 1, 1, 0, 0, 0])) / s_C
        x[:, 6] = (np.asarray(vf) - vf0) / s_vf
        return x

    def gradient(self, x, t, w, sw=None):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        w = np.ascontiguousarray(w, np.float32)
        sw = None if sw is None else np.ascontiguousarray(sw, np.float32)
        g = np.zeros(self.n_params, np.float32)
        loss = C.c_double()
        self._check(self._L.ceos_sur_gradient(self._h, x.shape[0], _ptr(x), _ptr(t), _ptr(w), _ptr(sw), _ptr(g),
                                              C.byref(loss)))
        return loss.value, g

    def train(self, x, t, w, epochs, batch, lr0=2e-3, lr1=2e-5, seed=0, sw=None):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        w = np.ascontiguousarray(w, np.float32)
        sw = None if sw is None else np.ascontiguousarray(sw, np.float32)
        hist = np.zeros(epochs)
        self._check(self._L.ceos_sur_train(self._h, x.shape[0], _ptr(x), _ptr(t), _ptr(w), _ptr(sw), epochs, batch,
                                           lr0, lr1, seed, _ptr(hist)))
        return hist

    def evaluate(self, C6, vf):
        """S [N,6], material tangent [N,6,6] (Voigt tensor components), out-of-range flags [N]."""
        C6 = np.ascontiguousarray(C6, np.float64)
        vf = np.ascontiguousarray(vf, np.float64)
        n = vf.size
        S = np.zeros((n, 6))
        Cm = np.zeros((n, 36))
        fl = np.zeros(n, np.int32)
        self._check(self._L.ceos_sur_evaluate(self._h, n, _ptr(C6), _ptr(vf), _ptr(S), _ptr(Cm), _ptr(fl)))
        return S, Cm.reshape(n, 6, 6), fl.astype(bool)

    def material_device(self, n_elem, F_ptr, ldF, vf_ptr, state_ptr, state_f32, ld, flags_ptr, stream=0):
        """Fill the external-material state of an element loop from device arrays (pointers)."""
        self._check(self._L.ceos_sur_material_device(self._h, n_elem, F_ptr, ldF, vf_ptr, state_ptr, state_f32, ld,
                                                     flags_ptr, stream))

    def close(self):
        if getattr(self, "_h", None):
            self._L.ceos_sur_destroy(self._h)
            self._h = None

    def __del__(self):
        try:  # at interpreter exit the library binding may already be gone
            self.close()
        except Exception:
            pass


def training_targets(F, P, s_C, s_W):
    """Targets of de/dx for the stress loss: t_k = S_k / (a_k s_W / s_C), weights a_k^2 (the loss
    is then the mean squared stress error in units of s_W / s_C)."""
    S = voigt_S_from_P(F, P)
    t = S / (VOIGT_A * (s_W / s_C))
    return t, VOIGT_A ** 2


def init_params(seed=0):
    """He-style initial parameters (normal, std sqrt(2/fan_in); output layer sqrt(1/128); zero biases)."""
    rng = np.random.default_rng(seed)
    H = 128
    parts = [rng.normal(0, np.sqrt(2.0 / 7), (H, 7)).ravel(), np.zeros(H)]
    for _ in range(3):
        parts += [rng.normal(0, np.sqrt(2.0 / H), (H, H)).ravel(), np.zeros(H)]
    parts += [rng.normal(0, np.sqrt(1.0 / H), H), np.zeros(1)]
    return np.concatenate(parts).astype(np.float32)
