"""The codec's numpy restatement pinned on its own definition (CPU): the analytic gradient against
central finite differences of the loss (no roundings, float64), the block layout round trip, and the
BF16 rounding helper against torch's conversion."""
import numpy as np
import pytest

from oracle import codec_oracle as co


def test_block_layout_roundtrip():
    rng = np.random.default_rng(0)
    for shape in [(16, 8, 24), (13, 9, 20)]:
        f = rng.standard_normal(shape).astype(np.float32)
        B, _ = co.blocks_of(f)
        assert B.shape == (np.prod([-(-n // 8) for n in shape]), 512)
        assert np.array_equal(co.field_of(B, shape), f.astype(np.float64))
    # cell order: s = (sx*2+sy)*2+sz, k = (dx*4+dy)*4+dz
    f = np.arange(8 * 8 * 8, dtype=np.float32).reshape(8, 8, 8)
    B, _ = co.blocks_of(f)
    j = (((1 * 2 + 0) * 2 + 1) * 64) + ((2 * 4 + 3) * 4 + 1)  # s=(1,0,1), k=(2,3,1) -> (6, 3, 5)
    assert B[0, j] == f[6, 3, 5]


def test_bf16_rounding_matches_torch():
    import torch
    rng = np.random.default_rng(1)
    x = (rng.standard_normal(10000) * 10.0 ** rng.uniform(-5, 5, 10000)).astype(np.float32)
    want = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(co.bf16(x), want)


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(2)
    w = co.init_weights(3).astype(np.float64)
    w += rng.standard_normal(co.NPARAM) * 0.05  # non-zero biases
    X = rng.standard_normal((3, 512))
    X /= np.abs(X).max(axis=1, keepdims=True)
    g = co.grad(w, X, rounding=False)
    idx = np.concatenate([rng.choice(np.arange(o, o + int(np.prod(s))), 6, replace=False)
                          for o, s in co.OFFSETS.values()])
    h = 1e-6
    for i in idx:
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        fd = (co.loss(wp, X, rounding=False) - co.loss(wm, X, rounding=False)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])


def test_dct_codec_keeps_32_coefficients_and_is_exact_for_smooth_blocks():
    keep = co.dct_keep(32)
    assert len(keep) == 32 and keep[0] == (0, 0, 0)
    x, y, z = np.meshgrid(np.arange(8.0), np.arange(16.0), np.arange(24.0), indexing="ij")
    f = 1.0 + 0.01 * x  # constant plus a gentle ramp: captured up to BF16 rounding
    r = co.dct_roundtrip(f)
    assert np.abs(r - f).max() < 2e-2
