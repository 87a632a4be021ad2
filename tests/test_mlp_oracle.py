"""The learned proposal's CPU oracle is pinned by finite differences
(the network has no reference counterpart), and its bf16 rounding
matches torch's round-to-nearest-even conversion."""
import numpy as np

from oracle import mlp_oracle as M


def test_bf16_rounding_matches_torch():
    import torch
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.normal(size=4000) * 10.0 ** rng.integers(-6, 6, 4000), [0.0, -0.0, 1.0, 1.00390625, 1.01171875, -3.5e-3]])
    ref = torch.tensor(x, dtype=torch.float32).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(M.bf16(x), ref)


def test_oracle_backward_matches_finite_differences():
    rng = np.random.default_rng(1)
    theta = M.init_params(3, scale=2.0)
    X = rng.normal(size=(6, M.F_IN)) / np.sqrt(M.F_IN)
    T = rng.normal(size=(6, 3))
    T /= np.linalg.norm(T, axis=1, keepdims=True)
    assert M.check_gradients(theta, X, T, n_probe=24, h=1e-4) < 1e-6


def test_oracle_layout_round_trip():
    theta = M.init_params(4)
    assert theta.size == M.n_params()
    assert np.array_equal(M.pack(M.unpack(theta)), theta)
