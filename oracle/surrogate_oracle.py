"""FP64 CPU oracle of the MLP energy surrogate (TEST INFRASTRUCTURE ONLY).

The surrogate has no reference counterpart: CEOS obtains the homogenized response of a macro
Gauss point by solving its RVE (MultiScale/ModMultiscaleAnalysis.f90:445-470).  The network is
an energy e(x) of x = [(C11-1, C22-1, C33-1, C12, C23, C13) / s_C, (vf - vf0) / s_vf]:

    z1 = W1 x + b1,  h_l = softplus(z_l),  z_l = W_l h_{l-1} + b_l (l = 2..4),  e = w5 . h4 + b5

with second Piola stress S_k = a_k (s_W / s_C) de/dx_k, a = (2, 2, 2, 1, 1, 1), and material
tangent C_pq = a_p a_q (s_W / s_C^2) d2e/dx_p dx_q (tensor components in Voigt order).

Training fits the stress only (Sobolev loss on de/dx): L = (1/N) sum_n sum_k w_k (g_k - t_k)^2,
g = de/dx.  Its parameter gradient is the forward-over-reverse product d/dtheta (u . g) with
u = dL/dg, written out layer by layer below.  With bf16=True the GEMM operands are rounded to
bfloat16 (round to nearest even) at exactly the points where the GPU kernels round them.
"""
import numpy as np

H = 128
NIN = 7
SHAPES = [("W1", (H, NIN)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (H, H)), ("b3", (H,)),
          ("W4", (H, H)), ("b4", (H,)), ("w5", (H,)), ("b5", (1,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(theta):
    out, o = {}, 0
    for name, shp in SHAPES:
        k = int(np.prod(shp))
        out[name] = np.asarray(theta[o:o + k], dtype=np.float64).reshape(shp)
        o += k
    return out


def pack(p):
    return np.concatenate([np.asarray(p[name], np.float64).reshape(-1) for name, _ in SHAPES])


def init_params(seed=0):
    """He-style initialisation (the GPU trainer is seeded with the same vector)."""
    rng = np.random.default_rng(seed)
    p = {}
    p["W1"] = rng.normal(0, np.sqrt(2.0 / NIN), (H, NIN))
    for l in (2, 3, 4):
        p["W%d" % l] = rng.normal(0, np.sqrt(2.0 / H), (H, H))
    for l in (1, 2, 3, 4):
        p["b%d" % l] = np.zeros(H)
    p["w5"] = rng.normal(0, np.sqrt(1.0 / H), H)
    p["b5"] = np.zeros(1)
    return pack(p)


def bf16(a):
    """Round float64/float32 values to bfloat16 (nearest even), returned as float64."""
    f = np.asarray(a, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def softplus(z):
    return np.maximum(z, 0.0) + np.log1p(np.exp(-np.abs(z)))


def sigmoid(z):
    return 0.5 * (1.0 + np.tanh(0.5 * z))


def energy_grad_hess(theta, x):
    """e [N], g = de/dx [N,7], Hs = d2e/dx2 [N,7,7] in FP64 (no rounding)."""
    p = unpack(theta)
    Ws = [p["W1"], p["W2"], p["W3"], p["W4"]]
    bs = [p["b1"], p["b2"], p["b3"], p["b4"]]
    x = np.atleast_2d(x)
    zs, h = [], x
    for W, b in zip(Ws, bs):
        z = h @ W.T + b
        zs.append(z)
        h = softplus(z)
    e = h @ p["w5"] + p["b5"][0]
    # backward: G_l = de/dh_l, delta_l = de/dz_l
    G = [None] * 4
    G[3] = np.broadcast_to(p["w5"], zs[3].shape)
    deltas = [None] * 4
    for l in range(3, -1, -1):
        deltas[l] = sigmoid(zs[l]) * G[l]
        if l > 0:
            G[l - 1] = deltas[l] @ Ws[l]
    g = deltas[0] @ Ws[0]
    # Hessian: sum_l J_l^T diag(G_l sigma'(z_l)) J_l, J_l = dz_l/dx
    N = x.shape[0]
    Hs = np.zeros((N, NIN, NIN))
    J = np.broadcast_to(Ws[0], (N, H, NIN))
    for l in range(4):
        s = sigmoid(zs[l])
        c = G[l] * s * (1.0 - s)
        Hs += np.einsum("nmi,nm,nmj->nij", J, c, J)
        if l < 3:
            J = np.einsum("ab,nb,nbi->nai", Ws[l + 1], s, J)
    return e, g, Hs


def loss_and_grad(theta, x, t, w, bf=False, sw=None):
    """Sobolev loss on the first 6 input derivatives and its parameter gradient.

    x [N,7], t [N,6] targets of g[:, :6], w [6] component weights, sw [N] sample weights (None: 1).
    Returns (L, dL/dtheta).
    bf=True rounds to bfloat16 where the GPU does: the BF16 weight copies of W1..W4, the padded
    inputs x and seeds u, the activations h_l, tangents hdot_l, adjoints delta_l (l >= 2) and a_l.
    """
    r = bf16 if bf else (lambda v: v)
    p = unpack(theta)
    W = [p["W1"], p["W2"], p["W3"], p["W4"]]
    Wb = [r(Wl) for Wl in W]
    b = [p["b1"], p["b2"], p["b3"], p["b4"]]
    w5 = p["w5"]
    N = x.shape[0]
    X0 = r(x)
    # forward primal
    Z, Hb = [], []
    h = X0
    for l in range(4):
        z = h @ Wb[l].T + b[l]
        Z.append(z)
        h = r(softplus(z))
        Hb.append(h)
    S = [sigmoid(z) for z in Z]
    Sp = [s * (1.0 - s) for s in S]
    # backward primal: G_l (pre-sigmoid adjoint), delta_l
    G = [None] * 4
    D = [None] * 4
    G[3] = np.broadcast_to(w5, Z[3].shape)
    D[3] = r(S[3] * G[3])
    for l in (2, 1, 0):
        G[l] = D[l + 1] @ Wb[l + 1]
        D[l] = r(S[l] * G[l]) if l > 0 else S[0] * G[0]
    d1 = S[0] * G[0]                      # FP32 on the GPU, feeds the stress
    g = d1 @ W[0]                         # master FP32 W1
    res = g[:, :6] - t
    swv = np.ones(N) if sw is None else np.asarray(sw, np.float64)
    L = float(np.sum(swv[:, None] * w * res * res) / N)
    u = np.zeros((N, NIN))
    u[:, :6] = 2.0 * swv[:, None] * w * res / N
    U0 = r(u)
    # forward tangent
    Zd, Hd = [], []
    hd = U0
    for l in range(4):
        zd = hd @ Wb[l].T
        Zd.append(zd)
        hd_full = S[l] * zd
        hd = r(hd_full) if l < 3 else hd_full
        Hd.append(hd)
    # backward tangent: a_l
    A = [None] * 4
    A[3] = r(Sp[3] * Zd[3] * w5)
    for l in (2, 1, 0):
        T = A[l + 1] @ Wb[l + 1]
        A[l] = r(S[l] * T + Sp[l] * Zd[l] * G[l])
    D0 = r(d1)
    grads = {}
    prevH = [X0] + Hb[:3]
    prevHd = [U0] + Hd[:3]
    Dop = [D0, D[1], D[2], D[3]]
    for l in range(4):
        grads["W%d" % (l + 1)] = A[l].T @ prevH[l] + Dop[l].T @ prevHd[l]
        grads["b%d" % (l + 1)] = A[l].sum(axis=0)
    grads["w5"] = Hd[3].sum(axis=0)
    grads["b5"] = np.zeros(1)
    return L, pack(grads)


def stress_tangent(theta, x, s_C, s_W):
    """S [N,6] and material tangent C [N,6,6] (Voigt tensor components) from the energy."""
    _, g, Hs = energy_grad_hess(theta, x)
    a = np.array([2.0, 2.0, 2.0, 1.0, 1.0, 1.0])
    S = a * (s_W / s_C) * g[:, :6]
    C = a[:, None] * a[None, :] * (s_W / s_C ** 2) * Hs[:, :6, :6]
    return S, C
