"""The CPU restatement of the learned preconditioner's network: its float64
gradients against central finite differences (pinning the backward pass the
GPU kernels are checked against), and its BF16 rounding."""
import numpy as np

from oracle import learn_oracle as lo


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, -2.5, 3.0e-3], dtype=np.float32)
    y = lo.bf16(x)
    # ties go to even: 1 + 2^-8 -> 1, 1 + 3 2^-8 -> 1 + 2^-6
    assert y[0] == 1.0 and y[1] == 1.0 and y[2] == np.float32(1.0 + 2.0 ** -6)
    assert y[3] == -2.5
    assert abs(y[4] - 3.0e-3) <= 3.0e-3 * 2.0 ** -8


def test_gradients_match_finite_differences():
    ops = lo.graph(widths=(3, 4, 5, 6), in_channels=4)
    rng = np.random.default_rng(11)
    params = rng.normal(scale=0.4, size=lo.param_count(ops))
    x = rng.normal(size=(2, 4, 8, 16))
    target = rng.normal(size=(2, 8, 16))
    R, npl = 7, 13
    loss, grad = lo.loss_and_grads(params, x, target, R, npl, ops, bf16_mode=False)
    assert grad.shape == params.shape
    idx = rng.choice(params.size, size=60, replace=False)
    eps = 1e-6
    for i in idx:
        p = params.copy()
        p[i] += eps
        lp, _ = lo.loss_and_grads(p, x, target, R, npl, ops, bf16_mode=False)
        p[i] -= 2 * eps
        lm, _ = lo.loss_and_grads(p, x, target, R, npl, ops, bf16_mode=False)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - grad[i]) <= 1e-6 * max(1.0, abs(grad).max()), (i, fd, grad[i])


def test_parameter_count():
    # the network of the library: 16/32/48/64 channels, 4 input channels
    assert lo.param_count() == 194769
