"""CPU restatement of the learned indicator (TEST INFRASTRUCTURE ONLY: the
checker for spd_k_b200/csrc/spdk_mlp.cu, never the product).

No reference counterpart exists (the reference's detector is a-posteriori
only), so this file pins the GPU kernels to the model's mathematics in FP64:
  - the feature rows of a state (spdk_learned.h), bit for bit;
  - forward pass, weighted binary cross-entropy and its gradient with
    respect to the BF16-rounded parameters, evaluated in FP64 on the same
    BF16 inputs (the GPU accumulates in FP32, so agreement is to FP32
    round-off, not bitwise).
The gradient itself is checked here against central finite differences.
"""
import numpy as np
from scipy.special import erf

H = 64


def bf16_round(a):
    """round float32 values to the nearest BF16 (ties to even), as float64"""
    a = np.ascontiguousarray(a, dtype=np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    lsb = (b >> 16) & 1
    r = ((b + 0x7FFF + lsb) >> 16) & 0xFFFF
    return bits_to_float(r.astype(np.uint16))


def bf16_bits(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    lsb = (b >> 16) & 1
    return (((b + 0x7FFF + lsb) >> 16) & 0xFFFF).astype(np.uint16)


def bits_to_float(bits):
    bits = np.asarray(bits).astype(np.uint16).astype(np.uint32) << 16
    return bits.view(np.float32).astype(np.float64)


def layout(n_in):
    o = {"W1": 0, "b1": n_in * H}
    o["W2"] = o["b1"] + H
    o["b2"] = o["W2"] + H * H
    o["w3"] = o["b2"] + H
    o["b3"] = o["w3"] + H
    o["n"] = o["b3"] + 1
    return o


def unpack(theta, n_in):
    o = layout(n_in)
    W1 = theta[o["W1"]:o["b1"]].reshape(n_in, H)
    b1 = theta[o["b1"]:o["W2"]]
    W2 = theta[o["W2"]:o["b2"]].reshape(H, H)
    b2 = theta[o["b2"]:o["w3"]]
    w3 = theta[o["w3"]:o["b3"]]
    b3 = theta[o["b3"]]
    return W1, b1, W2, b2, w3, b3


def gelu(a):
    return 0.5 * a * (1.0 + erf(a / np.sqrt(2.0)))


def gelu_d(a):
    return 0.5 * (1.0 + erf(a / np.sqrt(2.0))) + a * np.exp(-0.5 * a * a) / np.sqrt(2.0 * np.pi)


def forward(theta, X):
    """theta: FP64 parameter vector; X: FP64 [B][n_in] -> (p, cache)"""
    n_in = X.shape[1]
    W1, b1, W2, b2, w3, b3 = unpack(theta, n_in)
    A1 = X @ W1 + b1
    H1 = gelu(A1)
    A2 = H1 @ W2 + b2
    H2 = gelu(A2)
    z = H2 @ w3 + b3
    p = 1.0 / (1.0 + np.exp(-z))
    return p, (X, A1, H1, A2, H2, z)


def loss_grad(theta, X, y, w=None):
    """weighted BCE / sum(w) and its gradient (FP64)"""
    n_in = X.shape[1]
    W1, b1, W2, b2, w3, b3 = unpack(theta, n_in)
    w = np.ones(len(y)) if w is None else np.asarray(w, dtype=np.float64)
    p, (X, A1, H1, A2, H2, z) = forward(theta, X)
    ws = w.sum()
    loss = np.sum(w * (np.maximum(z, 0) - z * y + np.log1p(np.exp(-np.abs(z))))) / ws
    dz = w * (p - y) / ws
    g = np.zeros_like(theta)
    o = layout(n_in)
    g[o["b3"]] = dz.sum()
    g[o["w3"]:o["b3"]] = H2.T @ dz
    D2 = np.outer(dz, w3) * gelu_d(A2)
    g[o["b2"]:o["w3"]] = D2.sum(0)
    g[o["W2"]:o["b2"]] = (H1.T @ D2).reshape(-1)
    D1 = (D2 @ W2.T) * gelu_d(A1)
    g[o["b1"]:o["W2"]] = D1.sum(0)
    g[o["W1"]:o["b1"]] = (X.T @ D1).reshape(-1)
    return loss, g


def features(u, D, p, N, bc, gm):
    """feature rows of a solver state u [E][D+2][NPT] (solver layout) ->
    BF16 bit patterns [E][2 NPT + 4 D] (spd_k_b200/csrc/spdk_mlp.cu k_features)"""
    n = p + 1
    NPT = n ** D
    V = D + 2
    E = u.shape[0]
    u = u.reshape(E, V, NPT).astype(np.float64)
    r = u[:, 0]
    m2 = np.zeros_like(r)
    for d in range(1, V - 1):
        m2 = m2 + u[:, d] * u[:, d]
    pr = (u[:, V - 1] - 0.5 * m2 / r) * (gm - 1.0)
    # sums in point order, as the kernel does
    sr = np.zeros(E)
    sp = np.zeros(E)
    for pt in range(NPT):
        sr = sr + r[:, pt]
        sp = sp + pr[:, pt]
    mr = (sr / NPT).astype(np.float32).astype(np.float64)
    mp = (sp / NPT).astype(np.float32).astype(np.float64)

    def ratio(a, b):
        with np.errstate(all="ignore"):
            out = np.where((b > 0) & np.isfinite(b), a / b - 1.0, 0.0)
        return np.where(np.isfinite(out), out, 0.0).astype(np.float32)

    rows = np.zeros((E, 2 * NPT + 4 * D), dtype=np.float32)
    rows[:, :NPT] = ratio(r, mr[:, None])
    rows[:, NPT:2 * NPT] = ratio(pr, mp[:, None])
    Nx, Ny, Nz = N[0], N[1], (N[2] if D == 3 else 1)
    e = np.arange(E)
    c = [e % Nx, (e // Nx) % Ny, e // (Nx * Ny)]
    Nd = [Nx, Ny, Nz]
    for d in range(D):
        nbs = []
        for sd in (-1, 1):
            cc = [c[0].copy(), c[1].copy(), c[2].copy()]
            cc[d] = cc[d] + sd
            out = (cc[d] < 0) | (cc[d] >= Nd[d])
            if bc[d] == 0:
                cc[d] = np.where(cc[d] < 0, cc[d] + Nd[d], np.where(cc[d] >= Nd[d], cc[d] - Nd[d], cc[d]))
            else:
                cc[d] = np.where(out, c[d], cc[d])
            nbs.append((cc[2] * Ny + cc[1]) * Nx + cc[0])
        r0, r1 = ratio(mr[nbs[0]], mr), ratio(mr[nbs[1]], mr)
        p0, p1 = ratio(mp[nbs[0]], mp), ratio(mp[nbs[1]], mp)
        rows[:, 2 * NPT + 4 * d + 0] = np.minimum(r0, r1)
        rows[:, 2 * NPT + 4 * d + 1] = np.maximum(r0, r1)
        rows[:, 2 * NPT + 4 * d + 2] = np.minimum(p0, p1)
        rows[:, 2 * NPT + 4 * d + 3] = np.maximum(p0, p1)
    return bf16_bits(rows)
