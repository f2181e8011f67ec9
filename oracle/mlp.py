"""FP64 numpy restatement of the SOAP -> per-atom-energy MLP surrogate.

TEST INFRASTRUCTURE ONLY: the checker the CUDA training and inference kernels
(turbogap_b200/csrc/tgb_mlp.cu) are compared with. The reference has no learned
model; the network and its training objective are specified here:

    x   = (q - mu) / sigma_x                       (D inputs, zero-padded to Dp)
    z1  = W1 x + b1,  h1 = silu(z1)                (H)
    z2  = W2 h1 + b2, h2 = silu(z2)                (H)
    E   = w3 . h2 + b3                             (normalised energy)
    G   = dE/dx = W1^T [ (W2^T (w3 * silu'(z2))) * silu'(z1) ]
    L   = 1/B sum_b (E_b - y_b)^2 + lam/(B D) sum_b |G_b - Gref_b|^2

The weight gradient of the G term is the second-order ("double") back-
propagation written out in ``loss_and_grads``. With ``bf16=True`` every GEMM
operand is rounded to bfloat16 (round to nearest even) at the same points as
the GPU path, so the two agree to fp32-accumulation level rather than to the
bf16 resolution.
"""
from __future__ import annotations

import numpy as np


def round_bf16(a):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    u = (u + 0x7FFF + lsb) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def sigmoid(z):
    return 0.5 * (1.0 + np.tanh(0.5 * z))


def silu(z):
    return z * sigmoid(z)


def dsilu(z):
    s = sigmoid(z)
    return s * (1.0 + z * (1.0 - s))


def d2silu(z):
    s = sigmoid(z)
    return s * (1.0 - s) * (2.0 + z * (1.0 - 2.0 * s))


class Params:
    """One ensemble member: W1 (H, Dp), b1 (H), W2 (H, H), b2 (H), w3 (H), b3 ()."""

    def __init__(self, W1, b1, W2, b2, w3, b3):
        self.W1, self.b1, self.W2, self.b2, self.w3 = (np.array(v, np.float64)
                                                      for v in (W1, b1, W2, b2, w3))
        self.b3 = float(b3)

    @staticmethod
    def random(D, Dp, H, seed):
        rng = np.random.default_rng(seed)
        W1 = np.zeros((H, Dp))
        W1[:, :D] = rng.normal(0.0, 1.0 / np.sqrt(D), size=(H, D))
        W2 = rng.normal(0.0, 1.0 / np.sqrt(H), size=(H, H))
        w3 = rng.normal(0.0, 1.0 / np.sqrt(H), size=H)
        return Params(W1, rng.normal(0, 0.1, H), W2, rng.normal(0, 0.1, H), w3, 0.05)


def _mm(a, b, bf16):
    """a @ b with both operands rounded to bf16 when bf16 (GPU GEMM inputs)."""
    if bf16:
        return round_bf16(a) @ round_bf16(b)
    return a @ b


def forward(p: Params, X, bf16=False, s1_bf16=False):
    """Energies E (B) and input gradients G (B, Dp) of a batch X (B, Dp).

    s1_bf16 rounds silu'(z1) to bf16 before it scales v1, as the GPU inference
    path does (it stores silu'(z1) in bf16 from the layer-1 GEMM epilogue)."""
    z1 = _mm(X, p.W1.T, bf16) + p.b1
    h1 = silu(z1)
    z2 = _mm(h1, p.W2.T, bf16) + p.b2
    E = silu(z2) @ p.w3 + p.b3
    u2 = dsilu(z2) * p.w3
    v1 = _mm(u2, p.W2, bf16)
    s1 = round_bf16(dsilu(z1)) if s1_bf16 else dsilu(z1)
    u1 = v1 * s1
    G = _mm(u1, p.W1, bf16)
    return E, G


def loss_and_grads(p: Params, X, y, Gref, lam, D, bf16=False):
    """Loss and its gradient with respect to every parameter (dict), plus E, G."""
    B = X.shape[0]
    z1 = _mm(X, p.W1.T, bf16) + p.b1
    s1, t1 = dsilu(z1), d2silu(z1)
    h1 = silu(z1)
    z2 = _mm(h1, p.W2.T, bf16) + p.b2
    s2, t2 = dsilu(z2), d2silu(z2)
    h2 = silu(z2)
    E = h2 @ p.w3 + p.b3
    u2 = s2 * p.w3
    v1 = _mm(u2, p.W2, bf16)
    u1 = v1 * s1
    G = _mm(u1, p.W1, bf16)

    dE = E - y
    mask = np.zeros(G.shape[1])
    mask[:D] = 1.0
    dG = (G - Gref) * mask
    loss = float(np.sum(dE * dE) / B + lam * np.sum(dG * dG) / (B * D))
    e = 2.0 * dE / B
    R = 2.0 * lam * dG / (B * D)

    a1 = _mm(R, p.W1.T, bf16)              # dL/du1
    dv1 = a1 * s1
    dz1 = a1 * v1 * t1                     # through u1 = v1 * silu'(z1)
    du2 = _mm(dv1, p.W2.T, bf16)           # dL/du2
    dw3 = np.sum(du2 * s2, axis=0) + e @ h2
    dz2 = du2 * p.w3 * t2 + e[:, None] * p.w3 * s2
    db2 = dz2.sum(axis=0)
    db3 = float(e.sum())
    dW2 = _mm(dz2.T, h1, bf16) + _mm(u2.T, dv1, bf16)
    dh1 = _mm(dz2, p.W2, bf16)
    dz1 = dz1 + dh1 * s1
    db1 = dz1.sum(axis=0)
    dW1 = _mm(dz1.T, X, bf16) + _mm(u1.T, R, bf16)
    grads = dict(W1=dW1, b1=db1, W2=dW2, b2=db2, w3=dw3, b3=db3)
    return loss, grads, E, G


def loss_only(p: Params, X, y, Gref, lam, D):
    E, G = forward(p, X)
    dG = (G - Gref)[:, :D]
    return float(np.sum((E - y) ** 2) / X.shape[0] + lam * np.sum(dG * dG) / (X.shape[0] * D))


def adam_step(p: Params, g: dict, state: dict, lr, beta1=0.9, beta2=0.999, eps=1e-8):
    """In-place Adam update; state holds m, v per name and the step count t."""
    state["t"] = state.get("t", 0) + 1
    t = state["t"]
    for k in ("W1", "b1", "W2", "b2", "w3", "b3"):
        w = getattr(p, k)
        m = state.setdefault("m_" + k, np.zeros_like(np.asarray(w, np.float64)))
        v = state.setdefault("v_" + k, np.zeros_like(np.asarray(w, np.float64)))
        m[...] = beta1 * m + (1 - beta1) * g[k]
        v[...] = beta2 * v + (1 - beta2) * np.square(g[k])
        mh = m / (1 - beta1 ** t)
        vh = v / (1 - beta2 ** t)
        new = w - lr * mh / (np.sqrt(vh) + eps)
        setattr(p, k, float(new) if k == "b3" else new)
