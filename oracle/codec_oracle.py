"""numpy restatement of the learned wavefield codec -- TEST INFRASTRUCTURE ONLY.

Only tests/ use this module; the product never imports it. It restates, in float64 with the
kernels' BF16 roundings, the network of the CUDA codec (4^3/s4 conv 1->16 + leaky ReLU, 2^3/s2
conv 16->32 = the latent, and the two transposed convolutions back; per-8^3-block max-|value|
scaling), its loss (mean squared error of the normalised blocks) and its gradient, so that the
GPU training kernel's gradient and the GPU encode/decode can be checked. The codec has no
counterpart in the reference (CvxCompress, which it replaces in src/compressedio.jl:1-137, is not
in the reference tree and is not restated), so parity is pinned on the network's own definition:
`grad` is checked against finite differences of `loss` in tests/test_codec_oracle.py.

Also the non-learned method the network is compared with: an orthonormal 3D DCT-II of each 8^3
block keeping the 32 lowest-frequency coefficients (BF16) and the block scale -- the same code size.
"""
from __future__ import annotations

import numpy as np

# parameter layout of the CUDA codec (W*t[n][k]: output n, input k)
SHAPES = [("W1", (16, 64)), ("b1", (16,)), ("W2", (32, 128)), ("b2", (32,)), ("W3", (128, 32)), ("b3", (128,)),
          ("W4", (64, 16)), ("b4", (64,))]
OFFSETS = {}
_o = 0
for _n, _s in SHAPES:
    OFFSETS[_n] = (_o, _s)
    _o += int(np.prod(_s))
NPARAM = _o
LEAK = 0.5


def bf16(x):
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32)


def unpack(w, rounding=True):
    """Weights as float64 arrays; with rounding, matrices rounded to BF16 as the kernels read them and
    biases to FP32."""
    out = {}
    for n, (o, s) in OFFSETS.items():
        if rounding:
            a = np.asarray(w[o:o + int(np.prod(s))], np.float32).reshape(s)
            if n.startswith("W"):
                a = bf16(a)
        else:  # exact float64 (the finite-difference check)
            a = np.asarray(w[o:o + int(np.prod(s))], np.float64).reshape(s)
        out[n] = a.astype(np.float64)
    return out


def _act(x):
    return np.where(x >= 0, x, LEAK * x)


def _dact(x):
    return np.where(x >= 0, 1.0, LEAK)


def _q(x, rounding):
    return bf16(x.astype(np.float32)).astype(np.float64) if rounding else x


def forward(w, X, rounding=True):
    """X: (n, 512) normalised blocks in the codec's cell order. Returns (Y, cache)."""
    P = unpack(w, rounding)
    X = np.asarray(X, np.float64)
    n = X.shape[0]
    Xq = _q(X, rounding).reshape(n, 8, 64)
    H1p = np.einsum("nsk,ck->nsc", Xq, P["W1"]) + P["b1"]
    H1q = _q(_act(H1p), rounding).reshape(n, 128)
    Z = H1q @ P["W2"].T + P["b2"]
    Zq = _q(Z, rounding)
    H2p = Zq @ P["W3"].T + P["b3"]
    H2q = _q(_act(H2p), rounding).reshape(n, 8, 16)
    Y = (np.einsum("nsj,kj->nsk", H2q, P["W4"]) + P["b4"]).reshape(n, 512)
    return Y, dict(P=P, X=X, Xq=Xq, H1p=H1p, H1q=H1q, Zq=Zq, H2p=H2p, H2q=H2q, Y=Y)


def loss(w, X, rounding=True):
    Y, _ = forward(w, X, rounding)
    return float(np.mean((Y - np.asarray(X, np.float64)) ** 2))


def grad(w, X, rounding=True):
    """Gradient of `loss` with respect to the FP32 master weights (straight-through roundings)."""
    Y, c = forward(w, X, rounding)
    P, n = c["P"], c["X"].shape[0]
    dY = (2.0 * (Y - c["X"]) / (n * 512)).reshape(n, 8, 64)
    g = {}
    g["W4"] = np.einsum("nsk,nsj->kj", dY, c["H2q"])
    g["b4"] = dY.sum(axis=(0, 1))
    dH2 = (np.einsum("nsk,kj->nsj", dY, P["W4"]).reshape(n, 128)) * _dact(c["H2p"])
    g["W3"] = dH2.T @ c["Zq"]
    g["b3"] = dH2.sum(axis=0)
    dZ = dH2 @ P["W3"]
    g["W2"] = dZ.T @ c["H1q"]
    g["b2"] = dZ.sum(axis=0)
    dH1 = (dZ @ P["W2"]).reshape(n, 8, 16) * _dact(c["H1p"])
    g["W1"] = np.einsum("nsc,nsk->ck", dH1, c["Xq"])
    g["b1"] = dH1.sum(axis=(0, 1))
    out = np.zeros(NPARAM)
    for k, (o, s) in OFFSETS.items():
        out[o:o + int(np.prod(s))] = g[k].ravel()
    return out


# ---- whole fields -------------------------------------------------------------------------------------
def _cell_index():
    """(x, y, z) offsets of the 512 cells of a block in the codec's cell order."""
    j = np.arange(512)
    s, k = j >> 6, j & 63
    x = (s >> 2) * 4 + (k >> 4)
    y = ((s >> 1) & 1) * 4 + ((k >> 2) & 3)
    z = (s & 1) * 4 + (k & 3)
    return x, y, z


def blocks_of(field):
    """field (nx, ny, nz) -> (blocks (nb, 512) in block order (bx, by, bz), zero padded), padded shape."""
    nx, ny, nz = field.shape
    px, py, pz = -(-nx // 8) * 8, -(-ny // 8) * 8, -(-nz // 8) * 8
    f = np.zeros((px, py, pz), np.float32)
    f[:nx, :ny, :nz] = field
    cx, cy, cz = _cell_index()
    b = f.reshape(px // 8, 8, py // 8, 8, pz // 8, 8).transpose(0, 2, 4, 1, 3, 5)
    b = b.reshape(-1, 8, 8, 8)
    return np.ascontiguousarray(b[:, cx, cy, cz]), (px, py, pz)


def field_of(blocks, shape):
    nx, ny, nz = shape
    px, py, pz = -(-nx // 8) * 8, -(-ny // 8) * 8, -(-nz // 8) * 8
    cx, cy, cz = _cell_index()
    b = np.zeros((blocks.shape[0], 8, 8, 8), np.float64)
    b[:, cx, cy, cz] = blocks
    f = b.reshape(px // 8, py // 8, pz // 8, 8, 8, 8).transpose(0, 3, 1, 4, 2, 5).reshape(px, py, pz)
    return f[:nx, :ny, :nz]


def roundtrip(w, field):
    """Encode and decode a whole field with the network (the kernels' roundings)."""
    B, _ = blocks_of(field)
    m = np.abs(B).max(axis=1).astype(np.float32)
    inv = np.where(m > 0, np.float32(1.0) / np.where(m > 0, m, 1), 0).astype(np.float32)
    Xn = (B * inv[:, None]).astype(np.float32)
    Y, _ = forward(w, Xn)
    return field_of(Y * m[:, None].astype(np.float64), field.shape)


def dct_matrix(n=8):
    k = np.arange(n)[:, None]
    i = np.arange(n)[None, :]
    C = np.cos(np.pi * (2 * i + 1) * k / (2 * n)) * np.sqrt(2.0 / n)
    C[0] /= np.sqrt(2.0)
    return C


def dct_keep(ncoef=32):
    idx = [(i, j, k) for i in range(8) for j in range(8) for k in range(8)]
    idx.sort(key=lambda t: (sum(t), t[0] ** 2 + t[1] ** 2 + t[2] ** 2, t))
    return idx[:ncoef]


def dct_roundtrip(field, ncoef=32, raw_frac=0.01):
    """The non-learned codec of the same size: per 8^3 block, scale by max |value|, orthonormal
    3D DCT-II, keep the ncoef lowest-frequency coefficients in BF16, invert; then, like the learned
    codec, the raw_frac of blocks with the largest error energy are kept exactly."""
    nx, ny, nz = field.shape
    px, py, pz = -(-nx // 8) * 8, -(-ny // 8) * 8, -(-nz // 8) * 8
    f = np.zeros((px, py, pz), np.float64)
    f[:nx, :ny, :nz] = field
    b = f.reshape(px // 8, 8, py // 8, 8, pz // 8, 8).transpose(0, 2, 4, 1, 3, 5).reshape(-1, 8, 8, 8)
    m = np.abs(b).max(axis=(1, 2, 3))
    bn = b / np.where(m > 0, m, 1)[:, None, None, None]
    C = dct_matrix()
    c = np.einsum("ai,bj,ck,nijk->nabc", C, C, C, bn)
    keep = np.zeros((8, 8, 8), bool)
    for t in dct_keep(ncoef):
        keep[t] = True
    c = np.where(keep, bf16(c.astype(np.float32)).astype(np.float64), 0.0)
    r = np.einsum("ai,bj,ck,nabc->nijk", C, C, C, c) * m[:, None, None, None]
    if raw_frac > 0:
        err = ((r - b) ** 2).sum(axis=(1, 2, 3))
        cap = max(1, int(len(err) * raw_frac))
        worst = np.argsort(-err)[:cap]
        r[worst] = b[worst]
    r = r.reshape(px // 8, py // 8, pz // 8, 8, 8, 8).transpose(0, 3, 1, 4, 2, 5).reshape(px, py, pz)
    return r[:nx, :ny, :nz]


def init_weights(seed=0):
    """Glorot-uniform matrices and zero biases (the same scheme as the CUDA codec, another RNG)."""
    rng = np.random.default_rng(seed)
    w = np.zeros(NPARAM, np.float32)
    for n, (o, s) in OFFSETS.items():
        if n.startswith("W"):
            a = np.sqrt(6.0 / (s[0] + s[1]))
            w[o:o + s[0] * s[1]] = rng.uniform(-a, a, s[0] * s[1])
    return w
