"""Oracle (test infrastructure only): FP64 numpy restatement of the warm-start
MLP of mochii_b200/csrc/mlp.cu -- the forward pass, the loss and its
gradients -- with the operands of every matrix product rounded to BF16 at the
points where the device kernels round them (their FP32 accumulation is exact
here).  There is no reference counterpart: the MLP is this library's
addition, so the oracle is pinned by finite differences of itself."""
import numpy as np
from math import erf, sqrt, pi

DIMS = [16, 128, 128, 128, 4]


def bf16(x):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


_erf = np.vectorize(erf)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / sqrt(2.0))) + z * np.exp(-0.5 * z * z) / sqrt(2.0 * pi)


def unpack(p):
    W, b, o = [], [], 0
    for l in range(4):
        no, ni = DIMS[l + 1], DIMS[l]
        W.append(np.asarray(p[o:o + no * ni], dtype=np.float64).reshape(no, ni))
        o += no * ni
        b.append(np.asarray(p[o:o + no], dtype=np.float64))
        o += no
    return W, b


def head(o):
    p = np.zeros_like(o)
    p[:, 0] = 1.0 / (1.0 + np.exp(-o[:, 0]))
    z = np.stack([np.zeros(len(o)), o[:, 1], o[:, 2]], axis=1)
    z = np.exp(z - z.max(axis=1, keepdims=True))
    z /= z.sum(axis=1, keepdims=True)
    p[:, 1], p[:, 2] = z[:, 1], z[:, 2]
    p[:, 3] = o[:, 3]
    return p


def forward(p, X, rounding=True):
    r = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
    W, b = unpack(p)
    H, Z = [np.asarray(X, dtype=np.float64)], [None]
    for l in range(3):
        z = r(H[l]) @ r(W[l]).T + b[l]
        Z.append(z)
        H.append(gelu(z))
    out = r(H[3]) @ r(W[3]).T + b[3]
    return H, Z, out


def loss(p, X, Y, rounding=True):
    _, _, out = forward(p, X, rounding)
    e = head(out) - Y
    return float(np.mean(np.sum(e * e, axis=1) * 0.25))


def gradients(p, X, Y, rounding=True):
    r = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
    W, b = unpack(p)
    H, Z, out = forward(p, X, rounding)
    B = X.shape[0]
    pr = head(out)
    dp = 0.5 * (pr - Y) / B
    d = np.zeros_like(out)
    d[:, 0] = dp[:, 0] * pr[:, 0] * (1 - pr[:, 0])
    d[:, 1] = dp[:, 1] * pr[:, 1] * (1 - pr[:, 1]) - dp[:, 2] * pr[:, 2] * pr[:, 1]
    d[:, 2] = dp[:, 2] * pr[:, 2] * (1 - pr[:, 2]) - dp[:, 1] * pr[:, 1] * pr[:, 2]
    d[:, 3] = dp[:, 3]
    gW, gb = [None] * 4, [None] * 4
    dZ = d
    for l in range(3, -1, -1):
        gW[l] = r(dZ).T @ r(H[l])
        gb[l] = dZ.sum(axis=0)
        if l == 0:
            break
        dH = r(dZ) @ r(W[l])
        dZ = dH * gelu_grad(Z[l])
    out = []
    for l in range(4):
        out.append(gW[l].ravel())
        out.append(gb[l])
    return np.concatenate(out)
