"""CPU reference of the warm-start MLP (numpy) -- test infrastructure.

Same parameter layout and quantization points as the device: X, W1, W2 and
the first hidden activation rounded to bf16 (round to nearest even) before
their products; products and sums in f64 here (f32 on the device); GELU in
tanh form; sigmoid output.  Gradients by backpropagation, checked against
central finite differences of the same function in tests.
"""
import numpy as np

IN, H = 32, 64
W1, B1 = 0, H * IN
W2 = B1 + H
B2 = W2 + H * H
W3 = B2 + H
B3 = W3 + H
NPARAM = B3 + 1
K = 0.7978845608028654


def bf16(a):
    """Round f32 values to bf16 (nearest even), returned as f32/f64 values."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def unpack(p):
    p = np.asarray(p, np.float64)
    return (p[W1:B1].reshape(H, IN), p[B1:W2], p[W2:B2].reshape(H, H), p[B2:W3], p[W3:B3], p[B3])


def gelu(z):
    return 0.5 * z * (1.0 + np.tanh(K * (z + 0.044715 * z ** 3)))


def gelu_grad(z):
    th = np.tanh(K * (z + 0.044715 * z ** 3))
    return 0.5 * (1.0 + th) + 0.5 * z * (1.0 - th * th) * K * (1.0 + 3 * 0.044715 * z * z)


def forward(p, x, quantize=True):
    w1, b1, w2, b2, w3, b3 = unpack(p)
    q = bf16 if quantize else (lambda a: np.asarray(a, np.float64))
    xq = q(x).astype(np.float64)
    z1 = xq @ q(w1).astype(np.float64).T + b1
    a1 = gelu(z1)
    a1q = q(a1).astype(np.float64) if quantize else a1
    z2 = a1q @ q(w2).astype(np.float64).T + b2
    a2 = gelu(z2)
    y = a2 @ w3 + b3
    t = 1.0 / (1.0 + np.exp(-y))
    return t, dict(xq=xq, z1=z1, a1q=a1q, z2=z2, a2=a2, y=y)


def loss_and_grad(p, x, target, quantize=True):
    """Mean squared error of t and its gradient over the parameter vector."""
    w1, b1, w2, b2, w3, b3 = unpack(p)
    q = bf16 if quantize else (lambda a: np.asarray(a, np.float64))
    t, c = forward(p, x, quantize)
    n = len(x)
    loss = np.mean((t - target) ** 2)
    dy = 2.0 * (t - target) * t * (1.0 - t) / n
    g = np.zeros(NPARAM)
    g[W3:B3] = c["a2"].T @ dy
    g[B3] = dy.sum()
    dz2 = (dy[:, None] * w3[None, :]) * gelu_grad(c["z2"])
    dz2q = q(dz2).astype(np.float64)
    g[W2:B2] = (dz2q.T @ c["a1q"]).reshape(-1)
    g[B2:W3] = dz2.sum(0)
    da1 = dz2q @ q(w2).astype(np.float64)
    dz1 = da1 * gelu_grad(c["z1"])
    dz1q = q(dz1).astype(np.float64)
    g[W1:B1] = (dz1q.T @ c["xq"]).reshape(-1)
    g[B1:W2] = dz1.sum(0)
    return loss, g


def init_params(seed=0):
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM, np.float32)
    p[W1:B1] = rng.normal(0, 1 / np.sqrt(IN), H * IN)
    p[W2:B2] = rng.normal(0, 1 / np.sqrt(H), H * H)
    p[W3:B3] = rng.normal(0, 1 / np.sqrt(H), H)
    return p
