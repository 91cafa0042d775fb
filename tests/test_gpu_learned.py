"""The learned preconditioner's tensor-core convolution (tcgen05 + TMEM)
against a numpy restatement.

The numpy side rounds inputs and weights to BF16 exactly as the device does
(round to nearest even) and accumulates in FP64; the device accumulates in
FP32 and rounds its output to BF16, so the bound is 2^-8 of the output scale.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 2.0 ** -8


def _bf16(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(torch.bfloat16).to(torch.float32).numpy()


def conv_ref(x, w):
    """y[h, j, o] = sum_{dy, dx, i} x[h+dy-1, (j+dx-1) mod W, i] w[3 dy + dx, i, o],
    zero outside 0 <= h < H."""
    H, W, C = x.shape
    x, w = _bf16(x).astype(np.float64), _bf16(w).astype(np.float64)
    y = np.zeros((H, W, w.shape[2]))
    for dy in range(3):
        for dx in range(3):
            sh = np.roll(x, -(dx - 1), axis=1)               # sh[:, j] = x[:, j + dx - 1]
            pad = np.zeros_like(sh)
            lo, hi = max(0, 1 - dy), min(H, H + 1 - dy)      # rows h with 0 <= h + dy - 1 < H
            pad[lo:hi] = sh[lo + dy - 1:hi + dy - 1]
            y += pad @ w[3 * dy + dx]
    return y


def adjoint_weights(w):
    return np.stack([w[8 - t].T for t in range(9)])


@pytest.fixture(scope="module")
def G():
    from vvm_b200 import build, gpu
    build.build()
    return gpu


@pytest.mark.parametrize("H,W", [(3, 128), (5, 200), (4, 64), (2, 384)])
def test_conv_matches_reference(G, H, W):
    rng = np.random.default_rng(H * 1000 + W)
    x = rng.standard_normal((H, W, 32)).astype(np.float32)
    w = (rng.standard_normal((9, 32, 32)) / 16).astype(np.float32)
    y = G.conv3x3_c32(x, w)
    ref = conv_ref(x, w)
    assert np.abs(y - ref).max() <= TOL * np.abs(ref).max(), np.abs(y - ref).max()


def test_adjoint_conv_matches_reference_and_transposes(G):
    rng = np.random.default_rng(7)
    H, W = 6, 256
    x = rng.standard_normal((H, W, 32)).astype(np.float32)
    u = rng.standard_normal((H, W, 32)).astype(np.float32)
    w = (rng.standard_normal((9, 32, 32)) / 16).astype(np.float32)
    ya = G.conv3x3_c32(u, w, adjoint=True)
    ref = conv_ref(u, adjoint_weights(w))
    assert np.abs(ya - ref).max() <= TOL * np.abs(ref).max()
    # <A x, u> = <x, A^T u> up to the BF16 rounding of both results
    lhs = float(np.sum(G.conv3x3_c32(x, w).astype(np.float64) * _bf16(u)))
    rhs = float(np.sum(_bf16(x).astype(np.float64) * ya))
    assert abs(lhs - rhs) <= 1e-2 * abs(lhs)
