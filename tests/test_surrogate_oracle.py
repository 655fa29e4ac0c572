"""CPU checks of the surrogate's oracle (oracle/surrogate.py): the split is
exact up to binning noise, psi is C2 at the split radius, and the network's
backward pass is the adjoint of its forward pass."""
import numpy as np
import pytest

from oracle import surrogate as S


def test_psi_matches_outer_kernel_to_second_order():
    a = 10.0
    h = 1e-3
    assert abs(S.psi(a - 1e-9, a) - S.g_outer(a)) < 1e-9
    d1_in = (S.psi(a, a) - S.psi(a - h, a)) / h
    d1_out = (S.psi(a + h, a) - S.psi(a, a)) / h
    assert abs(d1_in - d1_out) < 1e-4
    d2_in = (S.psi(a - 2 * h, a) - 2 * S.psi(a - h, a) + S.psi(a, a)) / h ** 2
    d2_out = (S.psi(a, a) - 2 * S.psi(a + h, a) + S.psi(a + 2 * h, a)) / h ** 2
    assert abs(d2_in - d2_out) < 1e-3 * abs(d2_out) + 1e-6


def test_series_matches_dielectric_table():
    x = np.linspace(8.0, 81.91, 500)
    exact = np.interp(x, np.arange(8192) / 100.0, S.ddd_table())
    assert np.max(np.abs(S.tau(x) - exact) / exact) < 1e-5


def _receptor(n, seed):
    rng = np.random.default_rng(seed)
    r = 20.0 * (n / 2000.0) ** (1 / 3)
    p = rng.normal(size=(4 * n, 3))
    p = p / np.linalg.norm(p, axis=1)[:, None] * r * rng.random((4 * n, 1)) ** (1 / 3)
    p = p[:n]
    q = np.clip(rng.normal(0, 0.2, n), -0.7, 0.7)
    q -= q.mean()
    return np.concatenate([p, (q * 0.1465)[:, None]], axis=1)


def test_split_is_exact_up_to_binning_noise():
    x = _receptor(600, 1)
    pts = S.points(9, 9, 9, 0.375)
    a = 10.0
    d = S.direct(pts, x)
    n = S.near_field(pts, x, a)
    far = np.array([(S.psi(np.sqrt(((p - x[:, :3]) ** 2).sum(1)), a) * x[:, 3]).sum() for p in pts])
    assert np.max(np.abs(d - n - far)) < 5e-4


def test_trilinear_far_field_and_leading_correction():
    x = _receptor(600, 2)
    nx, ny, nz, h, a = 13, 11, 9, 0.375, 10.0
    fld = S.coarse_field(x, nx, ny, nz, h, a)
    feat, F = S.features_and_flin(fld, nx, ny, nz, h)
    pts = S.points(nx, ny, nz, h)
    far = np.array([(S.psi(np.sqrt(((p - x[:, :3]) ** 2).sum(1)), a) * x[:, 3]).sum() for p in pts])
    err = np.abs(F - far)
    corr = -0.5 * (feat[:, 0] + feat[:, 1] + feat[:, 2]) + feat[:, 6] / 6 + feat[:, 7] / 24
    err2 = np.abs(F + corr - far)
    # coarse nodes are exact; the leading-order terms remove most of the rest
    assert err2.max() < 0.5 * err.max()


def test_network_backward_is_adjoint_of_forward():
    rng = np.random.default_rng(3)
    shape = (3, 4, 5)
    P = int(np.prod(shape))
    w = rng.normal(0, 0.3, S.W1 + S.W2 + S.W3)
    feat = rng.normal(size=(P, 8))
    tgt = rng.normal(size=P)
    o, loss, g = S.net_grad(feat, w, shape, tgt, emulate_bf16=False)
    for idx in [5, S.W1 + 100, S.W1 + S.W2 + 7, S.W1 - 1, S.W1 + S.W2 - 3]:
        e = 1e-5
        wp, wm = w.copy(), w.copy()
        wp[idx] += e
        wm[idx] -= e
        _, lp, _ = S.net_grad(feat, wp, shape, tgt, emulate_bf16=False)
        _, lm, _ = S.net_grad(feat, wm, shape, tgt, emulate_bf16=False)
        num = (lp - lm) / (2 * e)
        assert abs(num - g[idx]) <= 1e-5 * max(1.0, abs(num)), (idx, num, g[idx])


def test_conv_adjoint_identity():
    rng = np.random.default_rng(4)
    x = rng.normal(size=(4, 3, 5, 8))
    W = rng.normal(size=(27, 8, 6))
    gr = rng.normal(size=(4, 3, 5, 6))
    lhs = (S.conv(x, W) * gr).sum()
    assert abs(lhs - (x * S.conv_t(gr, W)).sum()) < 1e-9 * abs(lhs) + 1e-9
    assert abs(lhs - (W * S.conv_w(x, gr)).sum()) < 1e-9 * abs(lhs) + 1e-9


def test_bf16_rounding_is_nearest_even():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 1e-30], dtype=np.float32)
    r = S.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6 and r[3] == -2.5
