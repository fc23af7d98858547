"""CPU oracle (FP64 numpy) for the sine-activated perceptron of the
station-beam surrogate: parameter layout, forward pass, mean-squared-error
loss and its gradient by backpropagation. Test infrastructure only; it is
itself checked against central finite differences in tests/test_mlp_oracle.py.

Layout (as the CUDA library's): per layer W [out][in] then b [out], one flat
array; every layer but the last is followed by sin(omega0 z)."""
import numpy as np


def unpack(params, dims):
    out, off = [], 0
    for a, b in zip(dims[:-1], dims[1:]):
        W = params[off:off + a * b].reshape(b, a)
        off += a * b
        bias = params[off:off + b]
        off += b
        out.append((W, bias))
    assert off == params.size
    return out


def forward(params, dims, omega0, x):
    """Returns (y, cache); cache holds each layer's input and pre-activation."""
    layers = unpack(np.asarray(params, np.float64), dims)
    a = np.asarray(x, np.float64)
    cache = []
    for i, (W, b) in enumerate(layers):
        z = a @ W.T + b
        cache.append((a, z))
        a = np.sin(omega0 * z) if i < len(layers) - 1 else z
    return a, cache


def mse(y, t):
    d = y - t
    return float(np.mean(d * d)), 2.0 * d / d.size


def backward(params, dims, omega0, cache, dy):
    layers = unpack(np.asarray(params, np.float64), dims)
    grads = []
    g = np.asarray(dy, np.float64)
    for i in range(len(layers) - 1, -1, -1):
        W, _ = layers[i]
        a_in, z = cache[i]
        if i < len(layers) - 1:
            g = g * omega0 * np.cos(omega0 * z)
        grads.append((g.T @ a_in, g.sum(axis=0)))
        g = g @ W
    flat = []
    for dW, db in reversed(grads):
        flat += [dW.ravel(), db]
    return np.concatenate(flat)


def loss_and_grad(params, dims, omega0, x, t):
    y, cache = forward(params, dims, omega0, x)
    loss, dy = mse(y, t)
    return loss, backward(params, dims, omega0, cache, dy)
