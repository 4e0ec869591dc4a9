"""The FP64 CPU network oracle (oracle/mlp_oracle.py): its backward pass against central
differences of its forward pass (pins the oracle used by the GPU gradient check)."""
import sys

import numpy as np

from conftest import ROOT

sys.path.insert(0, str(ROOT / "oracle"))
import mlp_oracle as mo  # noqa: E402


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = mo.random_params(rng)
    pts = np.concatenate([rng.uniform(-1, 1, (64, 3)), rng.normal(0, 0.3, (64, 1))], 1)
    idx = np.concatenate([rng.choice(np.arange(mo.W1, mo.B1), 8), rng.choice(np.arange(mo.B1, mo.W2), 4),
                          rng.choice(np.arange(mo.W2, mo.B2), 16), rng.choice(np.arange(mo.B2, mo.W3), 4),
                          rng.choice(np.arange(mo.W3, mo.B3), 8), [mo.B3]])
    assert mo.finite_difference_check(p, pts, idx) < 1e-6


def test_oracle_forward_matches_loss_path():
    rng = np.random.default_rng(4)
    p = mo.random_params(rng)
    pts = np.concatenate([rng.uniform(-1, 1, (32, 3)), np.zeros((32, 1))], 1)
    loss, _, y = mo.loss_and_grad(p, pts)
    assert np.allclose(y, mo.forward(p, pts[:, :3]))
    assert np.isclose(loss, np.mean(y * y))
