"""CPU checks of the CNN oracle: its analytic gradients against finite differences, BF16
rounding, and the subspace channel packing (the oracle itself, before it is used to check the GPU)."""
import numpy as np
import pytest

from oracle import cnn_oracle as CO


def test_bf16_round_nearest_even():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 3.0e-3], dtype=np.float32)
    r = CO.bf16_round(v)
    assert r[0] == 1.0
    assert r[1] == 1.0                      # halfway: ties to the even mantissa
    assert r[2] == 1.0 + 2 ** -6            # 1 + 3/256 -> 1 + 4/256
    assert r[3] == -2.5
    assert abs(r[4] - 3.0e-3) <= 3.0e-3 * 2 ** -8


@pytest.mark.parametrize("channels", [(2, 3, 2), (3, 4, 4, 3)])
def test_oracle_gradients_match_finite_differences(channels):
    rng = np.random.default_rng(3)
    _, n = CO.layer_slices(channels)
    p = rng.standard_normal(n) * 0.4
    x = rng.standard_normal((3, 4, 5, channels[0]))
    t = rng.standard_normal((3, 4, 5, channels[0]))
    _, g = CO.loss_and_grads(p, channels, x, t, round_weights=False)
    h = 1e-6
    for i in rng.choice(n, 25, replace=False):
        e = np.zeros(n)
        e[i] = h
        lp, _ = CO.loss_and_grads(p + e, channels, x, t, round_weights=False)
        lm, _ = CO.loss_and_grads(p - e, channels, x, t, round_weights=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_subspace_channels_round_trip():
    rng = np.random.default_rng(4)
    S, _ = np.linalg.qr(rng.standard_normal((9, 3)) + 1j * rng.standard_normal((9, 3)))
    c = rng.standard_normal((4, 5, 6, 6))
    x = CO.subspace_image(c, S, 2.0)
    assert x.shape == (6, 5, 4, 9)
    np.testing.assert_allclose(CO.subspace_channels(x, S, 2.0), c, atol=1e-12)
