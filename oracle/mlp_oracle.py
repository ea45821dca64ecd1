"""ORACLE - test infrastructure only.  float64 numpy restatement of the
surrogate MLP (in -> h -> h -> out, exact-erf GELU on the hidden layers),
its parameter gradient for a given output gradient, and one Adam step
(Kingma & Ba 2015), used to check libaq's aq_mlp_* kernels.  Every operand
of every contraction, weights and activations alike (x, a1, a2 in the
forward pass; dy, dz2, dz1 and the activations they multiply in the
backward pass), enters the dot products rounded to bf16 (round to nearest
even), as the kernels' tensor-core products read them; biases, bias
gradients, pre-activations and GELU stay unrounded."""
import math

import numpy as np

_erf = np.vectorize(math.erf)


def bf16(a):
    a = np.asarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def unpack(p, n_in, n_h, n_out):
    o = 0
    out = []
    for fan_in, fan_out in ((n_in, n_h), (n_h, n_h), (n_h, n_out)):
        W = p[o:o + fan_in * fan_out].reshape(fan_out, fan_in)
        o += fan_in * fan_out
        b = p[o:o + fan_out]
        o += fan_out
        out.append((W, b))
    return out


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2 * math.pi)


def r(a):
    """an operand as the tensor cores read it: bf16, widened back to float64"""
    return bf16(a).astype(np.float64)


def forward(p, x, dims):
    (W1, b1), (W2, b2), (W3, b3) = unpack(np.asarray(p, np.float32), *dims)
    x = np.asarray(x, np.float64)
    z1 = r(x) @ r(W1).T + b1
    a1 = gelu(z1)
    z2 = r(a1) @ r(W2).T + b2
    a2 = gelu(z2)
    y = r(a2) @ r(W3).T + b3
    return y, (x, z1, a1, z2, a2)


def backward(p, x, dy, dims):
    (W1, _), (W2, _), (W3, _) = unpack(np.asarray(p, np.float32), *dims)
    _, (x, z1, a1, z2, a2) = forward(p, x, dims)
    dy = np.asarray(dy, np.float64)
    gW3, gb3 = r(dy).T @ r(a2), dy.sum(0)
    dz2 = (r(dy) @ r(W3)) * gelu_grad(z2)
    gW2, gb2 = r(dz2).T @ r(a1), dz2.sum(0)
    dz1 = (r(dz2) @ r(W2)) * gelu_grad(z1)
    gW1, gb1 = r(dz1).T @ r(x), dz1.sum(0)
    return np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])


def adam(p, m, v, g, t, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    p = p - lr * (m / (1 - b1 ** t)) / (np.sqrt(v / (1 - b2 ** t)) + eps)
    return p, m, v
