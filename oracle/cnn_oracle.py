"""CPU float64 oracle of the learned coarse-grid correction's network.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the BF16
tensor-core kernels (precision-study_b200/csrc/learned/); never used by the
product.

The reference has no implementation of this part (it is named in the
project's plan only), so there is no reference code to follow; this module
states the mathematics directly and its gradients are pinned by central
finite differences in float64 (tests/test_learned_oracle.py).

Conventions (the kernels' own): images are NHWC arrays [batch, h, w, c],
periodic in y and x; weights W[c_out, 9, c_in] with tap t = (dy+1)*3 +
(dx+1) and out(y, x) = sum_t W[:, t, :] @ x(y+dy, x+dx) + b; GELU is the
tanh form 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3))), written as
z / (1 + exp(-2 sqrt(2/pi) (z + 0.044715 z^3))) (the same function; no
cancellation in the left tail).
"""
import math

import numpy as np

TAPS = [(t // 3 - 1, t % 3 - 1) for t in range(9)]


def bf16_round(a):
    """Round to the nearest bfloat16 (ties to even), returned as float32."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def to_bf16_bits(a):
    """bfloat16 bit patterns (uint16) of bf16_round(a)."""
    return (bf16_round(a).view(np.uint32) >> 16).astype(np.uint16)


def from_bf16_bits(u):
    return (np.asarray(u, dtype=np.uint32) << 16).view(np.float32)


# y2 = 2 sqrt(2/pi) (z + 0.044715 z^3) = z (GELU_A + GELU_B z^2)
GELU_A = 2.0 * math.sqrt(2.0 / math.pi)
GELU_B = GELU_A * 0.044715


def _gelu_sigmoid(z):
    z = np.asarray(z, dtype=np.float64)
    y2 = z * (GELU_A + GELU_B * z * z)
    with np.errstate(over="ignore"):
        return 1.0 / (1.0 + np.exp(-y2))


def gelu(z):
    return np.asarray(z, dtype=np.float64) * _gelu_sigmoid(z)


def gelu_grad(z):
    z = np.asarray(z, dtype=np.float64)
    s = _gelu_sigmoid(z)
    return s + z * s * (1.0 - s) * (GELU_A + 3.0 * GELU_B * z * z)


def shift(x, dy, dx):
    """x(y+dy, x+dx) with periodic wrap, for NHWC x."""
    return np.roll(np.roll(x, -dy, axis=1), -dx, axis=2)


def conv3x3(x, W, b=None):
    x = np.asarray(x, dtype=np.float64)
    W = np.asarray(W, dtype=np.float64)
    out = np.zeros(x.shape[:3] + (W.shape[0],))
    for t, (dy, dx) in enumerate(TAPS):
        out += shift(x, dy, dx) @ W[:, t, :].T
    if b is not None:
        out += np.asarray(b, dtype=np.float64)
    return out


def conv3x3_backward_input(dz, W):
    """Gradient of sum(dz * conv3x3(x, W)) with respect to x."""
    dz = np.asarray(dz, dtype=np.float64)
    W = np.asarray(W, dtype=np.float64)
    dx_ = np.zeros(dz.shape[:3] + (W.shape[2],))
    for t, (dy, dx) in enumerate(TAPS):
        dx_ += shift(dz, -dy, -dx) @ W[:, t, :]
    return dx_


def conv3x3_backward_weight(x, dz):
    """Gradients (dW[c_out, 9, c_in], db[c_out]) of sum(dz * conv3x3(x, W) + b)."""
    x = np.asarray(x, dtype=np.float64)
    dz = np.asarray(dz, dtype=np.float64)
    co, ci = dz.shape[3], x.shape[3]
    dW = np.zeros((co, 9, ci))
    for t, (dy, dx) in enumerate(TAPS):
        dW[:, t, :] = np.einsum("bhwo,bhwi->oi", dz, shift(x, dy, dx))
    return dW, dz.sum(axis=(0, 1, 2))


def net_forward(x, params):
    """Network of len(params) layers: conv-GELU ..., then conv (linear).
    params is a list of (W, b) per layer.  Returns (output, cache)."""
    cache = []
    a = np.asarray(x, dtype=np.float64)
    for i, (W, b) in enumerate(params):
        z = conv3x3(a, W, b)
        cache.append((a, z))
        a = gelu(z) if i < len(params) - 1 else z
    return a, cache


def net_loss_and_grads(x, params, target, nvar):
    """Mean squared error over the first nvar output channels and its
    gradients with respect to every (W, b)."""
    out, cache = net_forward(x, params)
    n = out.shape[0] * out.shape[1] * out.shape[2] * nvar
    diff = np.zeros_like(out)
    diff[..., :nvar] = out[..., :nvar] - np.asarray(target, dtype=np.float64)[..., :nvar]
    loss = float((diff ** 2).sum() / n)
    dz = 2.0 * diff / n
    grads = [None] * len(params)
    for i in range(len(params) - 1, -1, -1):
        a_in, _ = cache[i]
        grads[i] = conv3x3_backward_weight(a_in, dz)
        if i > 0:
            da = conv3x3_backward_input(dz, params[i][0])
            dz = da * gelu_grad(cache[i - 1][1])
    return loss, grads


DIRECT = [0, 1, 2, 3, 4, 6, 7]  # channels compared directly with the target
CH_A, CH_BX, CH_BY = 5, 8, 9     # potential; target field change


def curl_loss_and_grad(out, target, cx, cy):
    """Training loss of the correction network (the kernels' loss_grad):
    squared differences of the direct channels, plus the field change
    (target channels 8, 9) against the central-difference curl of the
    potential in channel 5, dBx = cy (A(y+1) - A(y-1)), dBy = -cx (A(x+1) -
    A(x-1)), periodic; divided by 9 x pixels.  Returns (loss, d loss / d out)
    for NHWC arrays of 16 channels."""
    out = np.asarray(out, dtype=np.float64)
    target = np.asarray(target, dtype=np.float64)
    n = 9 * out.shape[0] * out.shape[1] * out.shape[2]
    d = np.zeros_like(out)
    d[..., DIRECT] = out[..., DIRECT] - target[..., DIRECT]
    A = out[..., CH_A]
    rx = cy * (np.roll(A, -1, axis=1) - np.roll(A, 1, axis=1)) - target[..., CH_BX]
    ry = -cx * (np.roll(A, -1, axis=2) - np.roll(A, 1, axis=2)) - target[..., CH_BY]
    loss = float(((d ** 2).sum() + (rx ** 2).sum() + (ry ** 2).sum()) / n)
    g = 2.0 * d / n
    g[..., CH_A] = 2.0 / n * (cy * (np.roll(rx, 1, axis=1) - np.roll(rx, -1, axis=1)) +
                              cx * (np.roll(ry, -1, axis=2) - np.roll(ry, 1, axis=2)))
    return loss, g


def net_curl_loss_and_grads(x, params, target, cx, cy):
    """curl_loss_and_grad of the network output and its gradients with
    respect to every (W, b)."""
    out, cache = net_forward(x, params)
    loss, dz = curl_loss_and_grad(out, target, cx, cy)
    grads = [None] * len(params)
    for i in range(len(params) - 1, -1, -1):
        a_in, _ = cache[i]
        grads[i] = conv3x3_backward_weight(a_in, dz)
        if i > 0:
            da = conv3x3_backward_input(dz, params[i][0])
            dz = da * gelu_grad(cache[i - 1][1])
    return loss, grads
