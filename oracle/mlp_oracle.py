"""NumPy FP64 restatement of the warm-start MLP: forward, backward and Adam.

Test infrastructure only: the parity tests compare the tensor-core kernels of
gp5_b200/csrc/mlp.cu against these functions; nothing in the product imports this file.
The reference has no learned component (it starts every solve from a Gaussian,
python/test/regressionTests/LHY_imaginary.py:14), so the oracle is pinned by its own
finite-difference test instead of a reference golden.

Network: 3 -> 256 -> 256 -> 256 -> 64, GELU (exact, erf form) on the hidden layers, linear
output.  Loss: sum((y - t)^2) / (B * 64).  Parameter vector layout: for each layer, W row-major
[fan_out][fan_in] then b [fan_out].

`quantize=True` rounds the operands the GPU feeds its BF16 GEMMs (inputs, weights, hidden
activations and back-propagated gradients) to BF16 at the same points, so the two agree to
FP32-accumulation error rather than BF16 error.
"""
import math

import numpy as np

SHAPES = [(256, 3), (256, 256), (256, 256), (64, 256)]


def num_params(shapes=SHAPES):
    return sum(o * i + o for o, i in shapes)


def unpack(p, shapes=SHAPES):
    out, off = [], 0
    for o, i in shapes:
        W = p[off:off + o * i].reshape(o, i)
        off += o * i
        b = p[off:off + o]
        off += o
        out.append((W, b))
    return out


def bf16(a):
    """Round to the nearest BF16 value (ties to even); float64 result."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


_erf = np.vectorize(math.erf, otypes=[np.float64])


def gelu(x):
    return 0.5 * x * (1.0 + _erf(x / math.sqrt(2.0)))


def gelu_grad(x):
    cdf = 0.5 * (1.0 + _erf(x / math.sqrt(2.0)))
    pdf = np.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)
    return cdf + x * pdf


def forward(p, x, quantize=False, shapes=SHAPES):
    """Returns (y, cache) for inputs x [B][3]."""
    q = bf16 if quantize else (lambda a: np.asarray(a, dtype=np.float64))
    layers = unpack(np.asarray(p, dtype=np.float64), shapes)
    h = q(x)
    cache = {"inputs": [], "pre": []}
    for l, (W, b) in enumerate(layers):
        cache["inputs"].append(h)
        z = h @ q(W).T + b
        if l < len(layers) - 1:
            cache["pre"].append(z)
            h = q(gelu(z))
        else:
            h = z
    return h, cache


def loss_and_grad(p, x, t, quantize=False, shapes=SHAPES):
    """MSE loss and its gradient (same layout as p)."""
    q = bf16 if quantize else (lambda a: np.asarray(a, dtype=np.float64))
    y, cache = forward(p, x, quantize, shapes)
    B, n_out = y.shape
    loss = float(np.sum((y - t) ** 2) / (B * n_out))
    d = 2.0 * (y - t) / (B * n_out)
    layers = unpack(np.asarray(p, dtype=np.float64), shapes)
    grads = [None] * len(layers)
    for l in range(len(layers) - 1, -1, -1):
        W, _ = layers[l]
        dq = q(d)
        grads[l] = (dq.T @ cache["inputs"][l], d.sum(axis=0))
        if l == 0:
            break
        d = (dq @ q(W)) * gelu_grad(cache["pre"][l - 1])
    g = np.concatenate([np.concatenate([gw.ravel(), gb]) for gw, gb in grads])
    return loss, g


def adam_step(p, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update (bias-corrected, no weight decay); returns new (p, m, v)."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    c1 = 1 - b1 ** step
    c2 = 1 - b2 ** step
    p = p - lr * (m / c1) / (np.sqrt(v / c2) + eps)
    return p, m, v


def init_params(seed, shapes=SHAPES):
    """Seeded uniform initialisation of the same scale as the device's (zero biases); the
    device draws its own numbers, so tests that compare the two set the device's parameters."""
    rng = np.random.default_rng(seed)
    parts = []
    for l, (o, i) in enumerate(shapes):
        lim = math.sqrt(6.0 / i) * (0.5 if l == len(shapes) - 1 else 1.0)
        parts.append(rng.uniform(-lim, lim, o * i))
        parts.append(np.zeros(o))
    return np.concatenate(parts)
