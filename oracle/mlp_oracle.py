"""FP64 CPU oracle of the collision-likelihood MLP: forward pass, mean binary
cross-entropy and its gradient with respect to every parameter.

TEST INFRASTRUCTURE ONLY: the GPU training kernel's gradients are checked
against it.  It applies the kernels' BF16 rounding of the weights, inputs,
hidden activations and back-propagated errors (rounding treated as identity in
the derivative), so the comparison isolates the tensor-core arithmetic.
"""
import numpy as np


def _bf16(a):
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unflatten(p, n_in=48, hid=128):
    shapes = [("W1", (n_in, hid)), ("b1", (hid,)), ("W2", (hid, hid)), ("b2", (hid,)),
              ("W3", (hid, hid)), ("b3", (hid,)), ("w4", (hid,)), ("b4", (1,))]
    out, o = {}, 0
    for name, shape in shapes:
        k = int(np.prod(shape))
        out[name] = np.asarray(p[o:o + k], np.float64).reshape(shape)
        o += k
    return out, shapes


def loss_and_grads(p, x, y):
    """Returns (summed BCE loss, flat gradient of the MEAN BCE) in FP64."""
    P, shapes = unflatten(p)
    n = len(x)
    X = _bf16(x)
    W1, W2, W3 = _bf16(P["W1"]), _bf16(P["W2"]), _bf16(P["W3"])
    h1 = _bf16(np.maximum(X @ W1 + P["b1"], 0))
    h2 = _bf16(np.maximum(h1 @ W2 + P["b2"], 0))
    z3 = h2 @ W3 + P["b3"]
    h3 = np.maximum(z3, 0)
    z = h3 @ P["w4"] + P["b4"][0]
    y = np.asarray(y, np.float64)
    loss = np.sum(np.maximum(z, 0) - z * y + np.log1p(np.exp(-np.abs(z))))
    dz = (1.0 / (1.0 + np.exp(-z)) - y) / n
    g = {}
    g["w4"] = h3.T @ dz
    g["b4"] = np.array([dz.sum()])
    dz3 = np.outer(dz, P["w4"]) * (h3 > 0)
    g["b3"] = dz3.sum(0)
    dz3b = _bf16(dz3)
    g["W3"] = h2.T @ dz3b
    dh2 = dz3b @ W3.T
    dz2 = dh2 * (h2 > 0)
    g["b2"] = dz2.sum(0)
    dz2b = _bf16(dz2)
    g["W2"] = h1.T @ dz2b
    dh1 = dz2b @ W2.T
    dz1 = dh1 * (h1 > 0)
    g["b1"] = dz1.sum(0)
    g["W1"] = X.T @ _bf16(dz1)
    flat = np.concatenate([g[name].ravel() for name, _ in shapes])
    return loss, flat
