"""NumPy restatement of the learned column selector's network — test infrastructure.

The reference has no learned component; this oracle is the CPU check of the
library's hand-written kernels (kernels_mlp.cuh): the same 6 -> 64 -> 64 -> 2
perceptron with ReLU activations, BF16-rounded weights and FP32 biases, its
squared-error loss and the loss gradient with respect to every parameter
(weights as the BF16 values in use), and the per-column features.  The
arithmetic here is FP64 (a tighter reference than the kernels' FP32), and
``finite_difference`` checks the analytic gradient itself (weights taken at
their BF16 values, biases at their FP32 values).

Parameter order (as in the kernels): W1[64][6], W2[64][64], W3[2][64], then
b1[64], b2[64], b3[2].
"""

from __future__ import annotations

import numpy as np

N_IN, N_HID, N_OUT = 6, 64, 2
W1, W2, W3 = N_HID * N_IN, N_HID * N_HID, N_OUT * N_HID
N_WEIGHTS = W1 + W2 + W3
N_BIASES = N_HID + N_HID + N_OUT
N_PARAMS = N_WEIGHTS + N_BIASES


def bf16_round(x: np.ndarray) -> np.ndarray:
    """Round FP32 values to the nearest BF16 value (ties to even), returned as FP32."""
    bits = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    rounded = ((bits + 0x7FFF + ((bits >> 16) & 1)) >> 16) << 16
    return rounded.astype(np.uint32).view(np.float32)


def bf16_bits(x: np.ndarray) -> np.ndarray:
    """BF16 bit patterns (uint16) of FP32 values, rounded to nearest even."""
    return (bf16_round(x).view(np.uint32) >> 16).astype(np.uint16)


def unpack(params: np.ndarray):
    """Split a flat parameter vector; weights are rounded to BF16 as the kernels use them."""
    p = np.asarray(params, dtype=np.float32)
    w = bf16_round(p[:N_WEIGHTS]).astype(np.float64)
    b = p[N_WEIGHTS:].astype(np.float64)
    return (w[:W1].reshape(N_HID, N_IN), w[W1:W1 + W2].reshape(N_HID, N_HID),
            w[W1 + W2:].reshape(N_OUT, N_HID), b[:N_HID], b[N_HID:2 * N_HID], b[2 * N_HID:])


def forward(params, x):
    """out[count][2] for x[count][6]."""
    w1, w2, w3, b1, b2, b3 = unpack(params)
    x = np.asarray(x, dtype=np.float64)
    h1 = np.maximum(x @ w1.T + b1, 0.0)
    h2 = np.maximum(h1 @ w2.T + b2, 0.0)
    return h2 @ w3.T + b3


def loss_and_grad(params, x, y, c0=1.0, c1=1.0, scale=1.0):
    """scale * sum_i c0 (out0 - y0)^2 + c1 (out1 - y1)^2 and its gradient (flat, kernel order)."""
    w1, w2, w3, b1, b2, b3 = unpack(params)
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    z1 = x @ w1.T + b1
    h1 = np.maximum(z1, 0.0)
    z2 = h1 @ w2.T + b2
    h2 = np.maximum(z2, 0.0)
    out = h2 @ w3.T + b3
    r = out - y
    c = np.array([c0, c1])
    loss = scale * float(np.sum(c * r * r))
    d3 = 2.0 * c * r * scale
    d2 = (d3 @ w3) * (z2 > 0.0)
    d1 = (d2 @ w2) * (z1 > 0.0)
    grad = np.concatenate([(d1.T @ x).ravel(), (d2.T @ h1).ravel(), (d3.T @ h2).ravel(),
                           d1.sum(axis=0), d2.sum(axis=0), d3.sum(axis=0)])
    return loss, grad


def adam(master, m1, m2, grad, step, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, decay=0.0):
    """One Adam step (decoupled weight decay on the weights), as k_mlp_adam, in FP64."""
    master = np.array(master, dtype=np.float64)
    m1 = beta1 * np.asarray(m1, dtype=np.float64) + (1.0 - beta1) * grad
    m2 = beta2 * np.asarray(m2, dtype=np.float64) + (1.0 - beta2) * grad * grad
    master[:N_WEIGHTS] -= lr * decay * master[:N_WEIGHTS]
    master -= lr * (m1 / (1.0 - beta1 ** step)) / (np.sqrt(m2 / (1.0 - beta2 ** step)) + eps)
    return master, m1, m2


def finite_difference(params, x, y, index, c0=1.0, c1=1.0, h=1e-4):
    """Central difference of the loss in one parameter, in FP64.  A weight is
    perturbed after its BF16 rounding (the gradient is taken with respect to
    the BF16 value in use), a bias directly."""
    base = np.concatenate([bf16_round(np.asarray(params, dtype=np.float32)[:N_WEIGHTS]).astype(np.float64),
                           np.asarray(params, dtype=np.float64)[N_WEIGHTS:]])

    def loss64(q):
        w1 = q[:W1].reshape(N_HID, N_IN)
        w2 = q[W1:W1 + W2].reshape(N_HID, N_HID)
        w3 = q[W1 + W2:N_WEIGHTS].reshape(N_OUT, N_HID)
        b1, b2, b3 = q[N_WEIGHTS:N_WEIGHTS + N_HID], q[N_WEIGHTS + N_HID:N_WEIGHTS + 2 * N_HID], q[-N_OUT:]
        h1 = np.maximum(x @ w1.T + b1, 0.0)
        h2 = np.maximum(h1 @ w2.T + b2, 0.0)
        r = h2 @ w3.T + b3 - y
        return float(np.sum(np.array([c0, c1]) * r * r))

    plus, minus = base.copy(), base.copy()
    plus[index] += h
    minus[index] -= h
    return (loss64(plus) - loss64(minus)) / (2.0 * h)


def features(A, candidates, theta, scores, core_flags, mu):
    """The six inputs per candidate column (k_mlp_features), in FP64."""
    A = A.tocsc()
    nnz = np.diff(A.indptr)[candidates].astype(np.float64)
    sq = np.asarray(A.multiply(A).sum(axis=0)).ravel()[candidates]
    out = np.empty((candidates.size, N_IN))
    out[:, 0] = 0.1 * np.log(theta[candidates])
    out[:, 1] = np.log(nnz)
    out[:, 2] = 0.5 * np.log(np.maximum(sq, 1e-300))
    out[:, 3] = 0.1 * np.log(max(mu, 1e-300))
    out[:, 4] = 0.0 if core_flags is None else core_flags
    out[:, 5] = 0.1 * np.log(np.maximum(scores, 1e-300))
    return out
