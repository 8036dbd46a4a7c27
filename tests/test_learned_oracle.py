"""CPU checks of the network oracle (oracle/cnn_oracle.py): its analytic
gradients against central finite differences in float64, the transposed
convolution against the adjoint identity, and its bfloat16 rounding."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import cnn_oracle as C  # noqa: E402


def _params(rng, widths):
    return [(rng.normal(0, 0.4, (co, 9, ci)), rng.normal(0, 0.1, co)) for ci, co in zip(widths[:-1], widths[1:])]


def test_bf16_rounding_is_round_to_nearest_even():
    vals = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, -2.5, 1e-3, 3.0e38], dtype=np.float32)
    bits = C.to_bf16_bits(vals)
    assert list(bits[:4]) == [0x3F80, 0x3F80, 0x3F82, 0xC020]
    back = C.from_bf16_bits(bits)
    assert np.all(np.abs(back - vals) <= np.abs(vals) * 2.0 ** -8)


def test_adjoint_of_the_convolution():
    rng = np.random.default_rng(1)
    x = rng.normal(size=(2, 5, 7, 3))
    dz = rng.normal(size=(2, 5, 7, 4))
    W = rng.normal(size=(4, 9, 3))
    lhs = np.sum(dz * C.conv3x3(x, W))
    rhs = np.sum(x * C.conv3x3_backward_input(dz, W))
    assert abs(lhs - rhs) < 1e-10 * abs(lhs)


def test_network_gradients_match_finite_differences():
    rng = np.random.default_rng(2)
    widths = [3, 4, 4, 2]
    params = _params(rng, widths)
    x = rng.normal(size=(1, 4, 5, 3))
    target = rng.normal(size=(1, 4, 5, 2))
    loss, grads = C.net_loss_and_grads(x, params, target, 2)
    h = 1e-6
    for li, (W, b) in enumerate(params):
        for idx in [(0, 0, 0), (1, 4, 2), (W.shape[0] - 1, 8, W.shape[2] - 1)]:
            Wp = [(w.copy(), bb.copy()) for w, bb in params]
            Wm = [(w.copy(), bb.copy()) for w, bb in params]
            Wp[li][0][idx] += h
            Wm[li][0][idx] -= h
            fd = (C.net_loss_and_grads(x, Wp, target, 2)[0] - C.net_loss_and_grads(x, Wm, target, 2)[0]) / (2 * h)
            assert abs(fd - grads[li][0][idx]) < 1e-6 * max(1.0, abs(fd)), (li, idx)
        Wp = [(w.copy(), bb.copy()) for w, bb in params]
        Wm = [(w.copy(), bb.copy()) for w, bb in params]
        Wp[li][1][0] += h
        Wm[li][1][0] -= h
        fd = (C.net_loss_and_grads(x, Wp, target, 2)[0] - C.net_loss_and_grads(x, Wm, target, 2)[0]) / (2 * h)
        assert abs(fd - grads[li][1][0]) < 1e-6 * max(1.0, abs(fd)), (li, "bias")


def test_gelu_derivative_matches_finite_differences():
    z = np.linspace(-5, 5, 41)
    h = 1e-6
    fd = (C.gelu(z + h) - C.gelu(z - h)) / (2 * h)
    np.testing.assert_allclose(C.gelu_grad(z), fd, atol=1e-8)


def test_learned_config_defaults_and_argument_checks(pmhd_lib):
    import ctypes
    c = pmhd_lib.LearnedConfig()
    assert pmhd_lib.load().pmhd_learned_config_default(ctypes.byref(c)) == pmhd_lib.OK
    assert (c.nx, c.ny, c.refine, c.precision, c.max_pairs) == (64, 64, 4, pmhd_lib.MIXED, 512)
    assert (c.relax, c.train_noise, c.shrink) == (0.25, 0.03, 0.0)
    h = ctypes.c_void_p(1)
    bad = pmhd_lib.LearnedConfig.from_buffer_copy(c)
    bad.shrink = -0.5
    assert pmhd_lib.load().pmhd_learned_create(ctypes.byref(bad), ctypes.byref(h)) == pmhd_lib.ERR_ARG
    assert h.value is None
    bad = pmhd_lib.LearnedConfig.from_buffer_copy(c)
    bad.refine = 1
    assert pmhd_lib.load().pmhd_learned_create(ctypes.byref(bad), ctypes.byref(h)) == pmhd_lib.ERR_ARG
    assert h.value is None
    bad = pmhd_lib.LearnedConfig.from_buffer_copy(c)
    bad.precision = pmhd_lib.FP32
    assert pmhd_lib.load().pmhd_learned_create(ctypes.byref(bad), ctypes.byref(h)) == pmhd_lib.ERR_UNSUPPORTED
    L = pmhd_lib.load()
    assert L.pmhd_learned_train(None, 10, 4, 1e-3, None) == pmhd_lib.ERR_ARG
    assert L.pmhd_learned_destroy(None) == pmhd_lib.OK
    assert L.pmhd_learned_num_pairs(None) == 0


def test_curl_loss_gradient_matches_finite_differences():
    """The correction loss (direct channels plus the field through the curl
    of the potential channel) against central finite differences in every
    output entry, on a small periodic batch."""
    rng = np.random.default_rng(5)
    out = rng.normal(size=(2, 4, 5, 16))
    tgt = rng.normal(size=(2, 4, 5, 16))
    cx, cy = 0.5, 0.7
    _, g = C.curl_loss_and_grad(out, tgt, cx, cy)
    h = 1e-6
    it = np.nditer(out, flags=["multi_index"])
    for _ in it:
        idx = it.multi_index
        p = out.copy()
        m = out.copy()
        p[idx] += h
        m[idx] -= h
        fd = (C.curl_loss_and_grad(p, tgt, cx, cy)[0] - C.curl_loss_and_grad(m, tgt, cx, cy)[0]) / (2 * h)
        assert abs(fd - g[idx]) < 1e-7, (idx, fd, g[idx])
    # Channels outside the loss get no gradient.
    assert np.all(g[..., 8:] == 0)


def test_curl_of_a_potential_has_no_central_difference_divergence():
    """The field correction dBx = dA/dy, dBy = -dA/dx (central differences,
    periodic) leaves the central-difference div B unchanged: the property the
    corrected run relies on."""
    rng = np.random.default_rng(6)
    A = rng.normal(size=(1, 8, 9))
    dx, dy = 0.3, 0.2
    dbx = (np.roll(A, -1, axis=1) - np.roll(A, 1, axis=1)) / (2 * dy)
    dby = -(np.roll(A, -1, axis=2) - np.roll(A, 1, axis=2)) / (2 * dx)
    div = (np.roll(dbx, -1, axis=2) - np.roll(dbx, 1, axis=2)) / (2 * dx) + \
          (np.roll(dby, -1, axis=1) - np.roll(dby, 1, axis=1)) / (2 * dy)
    assert np.abs(div).max() < 1e-12 * np.abs(A).max() / (dx * dy)


def test_four_layer_network_with_curl_loss_matches_finite_differences():
    rng = np.random.default_rng(7)
    widths = [3, 4, 4, 4, 16]
    params = [(rng.normal(0, 0.3, (co, 9, ci)), rng.normal(0, 0.1, co)) for ci, co in zip(widths[:-1], widths[1:])]
    x = rng.normal(size=(1, 4, 5, 3))
    tgt = rng.normal(size=(1, 4, 5, 16))
    _, grads = C.net_curl_loss_and_grads(x, params, tgt, 0.5, 0.5)
    h = 1e-6
    for li in (0, 3):
        W, b = params[li]
        for idx in [(0, 4, 0), (2, 7, 1), (3, 0, 2)] if li == 0 else [(0, 4, 0), (5, 7, 1), (8, 0, 2)]:
            Wp, Wm = W.copy(), W.copy()
            Wp[idx] += h
            Wm[idx] -= h
            pp = list(params)
            pm = list(params)
            pp[li] = (Wp, b)
            pm[li] = (Wm, b)
            fd = (C.net_curl_loss_and_grads(x, pp, tgt, 0.5, 0.5)[0] -
                  C.net_curl_loss_and_grads(x, pm, tgt, 0.5, 0.5)[0]) / (2 * h)
            assert abs(fd - grads[li][0][idx]) < 1e-6 * max(1.0, abs(fd)), (li, idx, fd, grads[li][0][idx])
