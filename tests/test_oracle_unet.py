"""CPU pin of the learned-preconditioner oracle: its analytic gradient against
central differences of its own loss (exact for a loss quadratic in every
single weight, up to rounding), linearity of the network, and identity at a
zero last layer."""
import numpy as np
import pytest

from oracle import oracle as O

N3 = (8, 8, 16)


def _weights(seed):
    rng = np.random.default_rng(seed)
    w = np.zeros(O.unet_num_params(), dtype=np.float32)
    for name, (sl, (_, cout, cin)) in O.unet_layer_slices().items():
        w[sl] = rng.normal(0.0, 1.0 / np.sqrt(27 * cin), sl.stop - sl.start)
    return w


def test_param_count():
    assert O.unet_num_params() == 27 * sum(cin * cout for _, _, cin, cout in O.UNET_LAYERS) == 360288


def test_gradient_matches_central_differences():
    rng = np.random.default_rng(0)
    w = _weights(1)
    N = int(np.prod(N3))
    r = rng.normal(size=(2, N))
    e = rng.normal(size=(2, N))
    _, g = O.unet_loss_grad(N3, w, r, e, bf16=False)
    for name, (sl, _) in O.unet_layer_slices().items():
        for idx in rng.integers(sl.start, sl.stop, 2):
            h = np.float32(0.01 * max(abs(w[idx]), 0.01))
            wp, wm = w.copy(), w.copy()
            wp[idx] += h
            wm[idx] -= h
            lp, _ = O.unet_loss_grad(N3, wp, r, e, bf16=False, want_grad=False)
            lm, _ = O.unet_loss_grad(N3, wm, r, e, bf16=False, want_grad=False)
            fd = (lp - lm) / (float(wp[idx]) - float(wm[idx]))
            assert abs(g[idx] - fd) <= 1e-6 * max(abs(fd), 1e-3), (name, idx, g[idx], fd)


def test_network_is_linear():
    rng = np.random.default_rng(2)
    w = _weights(3)
    N = int(np.prod(N3))
    a, b = rng.normal(size=N), rng.normal(size=N)
    za = O.unet_forward(N3, w, a, bf16=False) - a
    zb = O.unet_forward(N3, w, b, bf16=False) - b
    zab = O.unet_forward(N3, w, 2.0 * a - 3.0 * b, bf16=False) - (2.0 * a - 3.0 * b)
    np.testing.assert_allclose(zab, 2.0 * za - 3.0 * zb, rtol=0, atol=1e-10 * np.abs(zab).max())


def test_zero_last_layer_is_identity():
    w = _weights(4)
    w[O.unet_layer_slices()["dec0"][0]] = 0.0
    u = np.random.default_rng(5).normal(size=int(np.prod(N3)))
    np.testing.assert_array_equal(O.unet_forward(N3, w, u, bf16=False), u)


def test_bad_grid_rejected():
    with pytest.raises(ValueError):
        O.unet_forward((8, 8, 12), _weights(0), np.zeros(8 * 8 * 12))
