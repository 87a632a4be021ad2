"""CPU oracle of the learned peak proposal (TEST INFRASTRUCTURE ONLY: used
by tests/ to check the library's forward and backward kernels, never by
the product).

The network has no counterpart in the reference (its output only seeds the
extremizer, sh_series_extremize.c:273-360), so this oracle is pinned by
the mathematics instead: ``check_gradients`` compares ``backward`` with
central finite differences of ``forward`` in plain FP64.

Layout: parameters are the FP32 masters in the library's order W1 [512][338],
b1, W2 [512][512], b2, W3 [512][512], b3, W4 [3][512], b4.  With
``bf16=True`` the oracle rounds to bf16 exactly where the GPU kernels do
(inputs, weights, hidden activations, dY and dZ) and accumulates in FP64;
the GPU accumulates in FP32, so the two agree to FP32 rounding plus the
occasional one-ulp bf16 flip that it causes.
"""
from __future__ import annotations

import math

import numpy as np

F_IN, HID, D_OUT = 338, 512, 3
SHAPES = [(HID, F_IN), (HID, HID), (HID, HID), (D_OUT, HID)]


def n_params() -> int:
    return sum(o * i + o for o, i in SHAPES)


def unpack(theta: np.ndarray):
    out, k = [], 0
    for o, i in SHAPES:
        W = theta[k:k + o * i].reshape(o, i)
        k += o * i
        b = theta[k:k + o]
        k += o
        out.append((W, b))
    return out


def pack(layers) -> np.ndarray:
    return np.concatenate([np.concatenate([W.ravel(), b.ravel()]) for W, b in layers])


def bf16(x) -> np.ndarray:
    """Round to the nearest bf16 (ties to even) and return as float64."""
    a = np.asarray(x, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def _erf(x):
    return np.vectorize(math.erf, otypes=[np.float64])(x)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def forward(theta, X, bf=True):
    """Returns (Y [n][3], cache)."""
    r = bf16 if bf else (lambda v: np.asarray(v, np.float64))
    layers = unpack(np.asarray(theta, np.float64))
    a = r(X)
    cache = {"A": [a], "Z": []}
    for W, b in layers[:3]:
        z = a @ r(W).T + b
        a = r(gelu(z))
        cache["Z"].append(z)
        cache["A"].append(a)
    W4, b4 = layers[3]
    Y = a @ r(W4).T + b4
    return Y, cache


def loss_and_dY(Y, T, bf=True):
    """Mean of 1 - y.t/|y| over rows and its gradient (rounded as the GPU's
    dY is)."""
    n = Y.shape[0]
    ny = np.linalg.norm(Y, axis=1, keepdims=True) + 1e-12
    c = np.sum(Y * T, axis=1, keepdims=True) / ny
    L = float(np.mean(1.0 - c))
    dY = -(T - c * Y / ny) / (ny * n)
    return L, (bf16(dY) if bf else dY)


def backward(theta, X, T, bf=True):
    """Gradient of the mean cosine loss, packed like theta."""
    r = bf16 if bf else (lambda v: np.asarray(v, np.float64))
    layers = unpack(np.asarray(theta, np.float64))
    Y, cache = forward(theta, X, bf)
    L, dY = loss_and_dY(Y, T, bf)
    grads = [None] * 4
    A = cache["A"]
    grads[3] = (dY.T @ A[3], dY.sum(axis=0))
    d = dY
    Wnext = r(layers[3][0])
    for i in (2, 1, 0):
        dz = r((d @ Wnext) * gelu_grad(cache["Z"][i]))
        grads[i] = (dz.T @ A[i], dz.sum(axis=0))
        d = dz
        Wnext = r(layers[i][0])
    return L, pack(grads)


def init_params(seed: int, scale: float = 1.0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    layers = []
    for o, i in SHAPES:
        lim = scale / math.sqrt(i)
        layers.append((rng.uniform(-lim, lim, (o, i)), rng.uniform(-0.1, 0.1, o)))
    return pack(layers)


def check_gradients(theta, X, T, n_probe=40, h=1e-5, seed=0):
    """Largest relative error of backward() against central differences of
    the FP64 loss along random parameter directions and single
    coordinates."""
    rng = np.random.default_rng(seed)
    _, g = backward(theta, X, T, bf=False)
    worst = 0.0

    def loss(th):
        Y, _ = forward(th, X, bf=False)
        return loss_and_dY(Y, T, bf=False)[0]

    for _ in range(n_probe):
        v = rng.normal(size=theta.size)
        v /= np.linalg.norm(v)
        fd = (loss(theta + h * v) - loss(theta - h * v)) / (2 * h)
        an = float(g @ v)
        worst = max(worst, abs(fd - an) / max(abs(fd), abs(an), 1e-12))
    return worst
