"""oracle/mlp_oracle.py -- TEST INFRASTRUCTURE ONLY: the CPU reference of the surrogate MLP.

A float64 numpy forward and backward pass of the library's MLP (din -> dh -> dh -> dh -> dout,
GELU in its tanh form between layers, mean squared error over the first `nvalid` outputs), used
only by tests to check the gradients the library's tensor-core kernels compute. With
``emulate_bf16`` it rounds to bfloat16 at exactly the points where the device stores bfloat16
(weights, activations, the pre-activations kept for the backward pass, gradients between
layers), so the remaining difference is the order of the FP32 sums and the device's tanh
approximation; without it every intermediate is float64.

The reference (ww3-gpu) has no learned component, so there is no reference file to cite: the
algorithm is the textbook backpropagation of this network.
"""

import numpy as np

GELU_C = 0.7978845608028654
GELU_A = 0.044715


def bf16(x):
    """Round to the nearest bfloat16 (ties to even), returned as float32."""
    x = np.ascontiguousarray(x, np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def gelu(z):
    return 0.5 * z * (1.0 + np.tanh(GELU_C * (z + GELU_A * z ** 3)))


def dgelu(z):
    t = np.tanh(GELU_C * (z + GELU_A * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * GELU_C * (1.0 + 3.0 * GELU_A * z * z)


def forward_backward(layers, x, t, nvalid=None, emulate_bf16=True):
    """layers: [(W (n x k), b (n))] * 4 in float32 (the device's fp32 master copy); x (m x din)
    bf16-representable; t (m x >= nvalid). Returns (loss, [(dW, db)] * 4) in float64."""
    r = bf16 if emulate_bf16 else (lambda v: np.asarray(v, np.float64))
    f64 = lambda v: np.asarray(v, np.float64)  # noqa: E731
    W = [f64(bf16(w)) for w, _ in layers]  # the device computes with bf16 weights
    B = [f64(b) for _, b in layers]
    m = x.shape[0]
    nvalid = nvalid or W[3].shape[0]
    acts = [f64(x)]
    zs = []
    h = f64(x)
    for l in range(3):
        z = h @ W[l].T + B[l]
        zs.append(f64(r(z)))          # pre-activation kept for GELU'
        h = f64(r(gelu(z)))
        acts.append(h)
    out = h @ W[3].T + B[3]
    d = out[:, :nvalid] - f64(t)[:, :nvalid]
    loss = float(np.mean(d * d))
    g = np.zeros_like(out)
    g[:, :nvalid] = 2.0 * d / (m * nvalid)
    g = f64(r(g))
    grads = [None] * 4
    for l in range(3, -1, -1):
        grads[l] = (g.T @ acts[l], g.sum(axis=0))
        if l == 0:
            break
        g = f64(r((g @ W[l]) * dgelu(zs[l - 1])))
    return loss, grads


def adamw_step(w, g, lr, wd, step=1, beta1=0.9, beta2=0.999, eps=1e-8, m=None, v=None):
    """One AdamW update of float32 master weights (decoupled decay), float64 arithmetic."""
    w = np.asarray(w, np.float64)
    g = np.asarray(g, np.float64)
    m = np.zeros_like(w) if m is None else m
    v = np.zeros_like(w) if v is None else v
    m = beta1 * m + (1 - beta1) * g
    v = beta2 * v + (1 - beta2) * g * g
    mh = m / (1 - beta1 ** step)
    vh = v / (1 - beta2 ** step)
    return w - lr * (mh / (np.sqrt(vh) + eps) + wd * w), m, v
