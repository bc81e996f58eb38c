"""CPU FP64 restatement of the learned star proposal's network (test
infrastructure: the checker of the tensor-core kernels, never the product).

The model (16 -> 64 -> 64 -> 64 -> 1, ReLU, binary cross-entropy on the
logit) and its parameter layout follow gstar4d_b200/csrc/g4d_mlp.cu. The model
itself has no counterpart in the reference; its labels come from the
reference's algorithm (final Delaunay edges of the plain star splaying).

forward_backward(..., rounding=True) rounds to BF16 where the kernels round:
weights, inputs, a1 and a2 entering a GEMM, and dz3, dz2, dz1 entering a GEMM;
everything else is computed in FP64. With rounding=False it is the exact
function, whose gradient a finite-difference test checks.
"""
import numpy as np

H, K0 = 64, 16
P_W1 = 0
P_B1 = P_W1 + H * K0
P_W2 = P_B1 + H
P_B2 = P_W2 + H * H
P_W3 = P_B2 + H
P_B3 = P_W3 + H * H
P_W4 = P_B3 + H
P_B4 = P_W4 + H
NPARAMS = P_B4 + 1


def bf16_bits(a):
    """Round-to-nearest-even BF16 encoding (uint16) of float32 values."""
    b = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = (b + 0x7FFF + ((b >> 16) & 1)) >> 16
    return r.astype(np.uint16)


def from_bf16(bits):
    return (np.asarray(bits, dtype=np.uint16).astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def bf16(a):
    """Values rounded to BF16 (through float32), as float64."""
    return from_bf16(bf16_bits(np.asarray(a, dtype=np.float64).astype(np.float32)))


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[P_W1:P_B1].reshape(H, K0), p[P_B1:P_W2], p[P_W2:P_B2].reshape(H, H), p[P_B2:P_W3],
            p[P_W3:P_B3].reshape(H, H), p[P_B3:P_W4], p[P_W4:P_B4], p[P_B4])


def pack(W1, b1, W2, b2, W3, b3, w4, b4):
    return np.concatenate([W1.ravel(), b1, W2.ravel(), b2, W3.ravel(), b3, w4, [b4]])


def forward_backward(x, y, params, rounding=True):
    """x: (m, 16) float64 inputs (already BF16 values when rounding), y: (m,)
    labels. Returns (mean loss, gradient vector, logits)."""
    r = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
    W1, b1, W2, b2, W3, b3, w4, b4 = unpack(params)
    W1r, W2r, W3r = r(W1), r(W2), r(W3)
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    m = len(x)
    z1 = x @ W1r.T + b1
    a1 = r(np.maximum(z1, 0.0))
    z2 = a1 @ W2r.T + b2
    a2 = r(np.maximum(z2, 0.0))
    z3 = a2 @ W3r.T + b3
    a3 = np.maximum(z3, 0.0)
    logit = a3 @ w4 + b4
    loss = np.mean(np.maximum(logit, 0.0) - logit * y + np.log1p(np.exp(-np.abs(logit))))
    dl = (1.0 / (1.0 + np.exp(-logit)) - y) / m
    g_w4 = a3.T @ dl
    g_b4 = dl.sum()
    dz3 = dl[:, None] * w4[None, :] * (z3 > 0)
    g_b3 = dz3.sum(0)
    dz3r = r(dz3)
    dz2 = (dz3r @ W3r) * (z2 > 0)
    g_b2 = dz2.sum(0)
    dz2r = r(dz2)
    dz1 = (dz2r @ W2r) * (z1 > 0)
    g_b1 = dz1.sum(0)
    dz1r = r(dz1)
    g_W3 = dz3r.T @ a2
    g_W2 = dz2r.T @ a1
    g_W1 = dz1r.T @ x
    return loss, pack(g_W1, g_b1, g_W2, g_b2, g_W3, g_b3, g_w4, g_b4), logit


def logits(x, params, rounding=True):
    return forward_backward(x, np.zeros(len(x)), params, rounding)[2]


def init_params(seed=0, scale=1.0):
    rng = np.random.default_rng(seed)
    W1 = rng.uniform(-1, 1, (H, K0)) * np.sqrt(6 / 6) * scale
    W2 = rng.uniform(-1, 1, (H, H)) * np.sqrt(6 / 64) * scale
    W3 = rng.uniform(-1, 1, (H, H)) * np.sqrt(6 / 64) * scale
    w4 = rng.uniform(-1, 1, H) * np.sqrt(6 / 64) * scale
    b1, b2, b3 = (rng.uniform(-0.1, 0.1, H) for _ in range(3))
    return pack(W1, b1, W2, b2, W3, b3, w4, 0.05)


def sample_rows(m, seed=0):
    """Feature rows shaped like the ring features (6 live columns in grid
    units, 10 zero columns), as BF16 bits and their float64 values."""
    rng = np.random.default_rng(seed)
    f = np.zeros((m, K0), np.float32)
    d = rng.normal(0, 1.2, (m, 3))
    f[:, 0:3] = d
    f[:, 3] = np.linalg.norm(d, axis=1) / 2
    f[:, 4] = rng.integers(1, 40, m) / 16.0
    f[:, 5] = rng.integers(2, 30, m) / 16.0
    bits = bf16_bits(f)
    return bits, from_bf16(bits)
