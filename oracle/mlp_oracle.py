"""CPU oracle of the surrogate MLP (test infrastructure only).

FP64 restatement of the forward and backward passes that the tensor-core
kernels in lcurve-rs_b200/csrc/lcb_mlp.cu compute, rounding to bfloat16 at the
same points the device does (packed input, weights, hidden activations, and
the gradients flowing between layers), so the two agree to accumulation-order
and transcendental rounding.  The reference has no surrogate, so nothing here
follows a reference file; the network is n_in -> width x n_hidden (exact erf
GELU) -> n_out with mean-squared-error loss.

Parameter layout (same as lcb_mlp_get_params): [W0 (width x n_in), b0,
W1 (width x width), b1, ..., W_last (n_out x width), b_last].
"""
import numpy as np
from scipy.special import erf


def bf16(a):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    a32 = np.ascontiguousarray(a, dtype=np.float32)
    u = a32.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def dgelu(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def unpack(params, n_in, width, n_hidden, n_out):
    """Flat parameter vector -> list of (W, b)."""
    shapes = [(width, n_in)] + [(width, width)] * (n_hidden - 1) + [(n_out, width)]
    out, k = [], 0
    for (o, i) in shapes:
        W = np.asarray(params[k:k + o * i], dtype=np.float64).reshape(o, i)
        k += o * i
        b = np.asarray(params[k:k + o], dtype=np.float64)
        k += o
        out.append((W, b))
    assert k == len(params)
    return out


def forward(layers, x):
    """Returns (prediction, inputs of every layer, pre-activations)."""
    a = bf16(x)
    xs, zs = [], []
    for l, (W, b) in enumerate(layers):
        xs.append(a)
        z = a @ bf16(W).T + b
        if l + 1 < len(layers):
            zs.append(z)
            a = bf16(gelu(z))
        else:
            return z, xs, zs


def loss_and_grads(params, x, target, n_in, width, n_hidden, n_out):
    """Mean-squared error and its gradient, in the flat parameter layout."""
    layers = unpack(params, n_in, width, n_hidden, n_out)
    pred, xs, zs = forward(layers, x)
    n = pred.size
    loss = float(np.mean((pred - target) ** 2))
    dz = bf16(2.0 * (pred - target) / n)
    grads = [None] * len(layers)
    for l in range(len(layers) - 1, -1, -1):
        W, _ = layers[l]
        grads[l] = (dz.T @ xs[l], dz.sum(axis=0))
        if l > 0:
            dz = bf16((dz @ bf16(W)) * dgelu(zs[l - 1]))
    flat = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])
    return loss, flat, pred
