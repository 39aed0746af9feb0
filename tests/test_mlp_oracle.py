"""The FP64 CPU MLP used to check the tensor-core backward pass is itself checked
against central finite differences of its own loss (CPU only)."""
import numpy as np

import mlp_oracle as M


def test_parameter_count_matches_the_c_abi():
    assert M.PARAMETERS == 5059


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = rng.standard_normal(M.PARAMETERS) * 0.2
    x = rng.standard_normal((16, M.IN))
    y = rng.standard_normal((16, M.OUT))
    _, g = M.loss_and_gradient(p, x, y, round_bf16=False)
    for k in list(rng.choice(M.PARAMETERS, 40, replace=False)) + [0, 639, 640, 5058]:
        e = np.zeros_like(p)
        e[k] = 1e-6
        fd = (M.loss_and_gradient(p + e, x, y, False)[0] -
              M.loss_and_gradient(p - e, x, y, False)[0]) / 2e-6
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(g[k])), k


def test_bf16_rounding_is_nearest_even():
    v = np.array([1.0, 1.00390625, 1.0078125, 1.01171875, -2.5], dtype=np.float32)
    r = M.bf16(v)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7 -> even (1.0); 1 + 3*2^-8 -> 1 + 2^-6
    assert list(r) == [1.0, 1.0, 1.0078125, 1.015625, -2.5]
