"""GPU: the learned far-field surrogate of the e-map.

* its exact parts (near field, coarse far field, trilinear interpolation and
  the corrector's input features) against the numpy oracle;
* the corrector's forward pass and weight gradient (hand-written tensor-core
  kernels) against the oracle's BF16-emulating forward and backward;
* a short training run lowers the loss;
* with the shipped weights, on a held-out 20,000-atom receptor on a 161^3
  grid: the error against the direct sum (all points) and the FP64 oracle
  (samples) stays within 0.01 kcal/mol/e, the corrector beats the trilinear
  far field alone, and the residual probes send a box back to the direct sum
  when they should.
"""
import json

import numpy as np
import pytest

import fastgrid_b200 as fg
import oracle
from oracle import surrogate as S

pytestmark = pytest.mark.gpu


def test_exact_parts_match_oracle():
    x = fg.surrogate_receptor(11, 1200)
    nx, ny, nz, h, a = 25, 23, 21, 0.375, 10.0
    g = fg.Grid(nx, ny, nz, h)
    ctx = fg.Context(0)
    feat, base = ctx.surrogate_features(g, x, fg.ddd_table())
    ctx.close()
    pts = S.points(nx, ny, nz, h)
    near = S.near_field(pts, x, a)
    fld = S.coarse_field(x, nx, ny, nz, h, a)
    ofeat, F = S.features_and_flin(fld, nx, ny, nz, h)
    assert np.max(np.abs(base - (near + F))) < 2e-4
    for k in range(8):
        tol = 0.01 * np.abs(ofeat[:, k]) + 2e-3 * np.sqrt(np.mean(ofeat[:, k] ** 2)) + 1e-7
        assert np.all(np.abs(feat[:, k] - ofeat[:, k]) <= tol), k


def test_corrector_forward_and_gradient_match_oracle():
    rng = np.random.default_rng(7)
    nx, ny, nz = 20, 9, 5  # partial tiles on every axis
    g = fg.Grid(nx, ny, nz, 0.375)
    P = nx * ny * nz
    w = np.concatenate([rng.normal(0, 0.15, S.W1), rng.normal(0, 0.06, S.W2), rng.normal(0, 0.05, S.W3)])
    w = S.bf16(w).astype(np.float32)
    feat = rng.normal(size=(P, 8)).astype(np.float32)
    tgt = rng.normal(size=P).astype(np.float32)
    ctx = fg.Context(0)
    ctx.surrogate_weights(w, (1.0, 1.0))
    o, grad, loss = ctx.surrogate_net_grad(g, feat, tgt)
    ctx.close()
    ro, rloss, rgrad = S.net_grad(feat, w, (nz, ny, nx), tgt)
    assert np.max(np.abs(o - ro)) <= 5e-3 * np.max(np.abs(ro))
    assert abs(loss - rloss) <= 1e-2 * rloss
    for lo, hi in ((0, S.W1), (S.W1, S.W1 + S.W2), (S.W1 + S.W2, S.W1 + S.W2 + S.W3)):
        d = np.abs(grad[lo:hi] - rgrad[lo:hi])
        scale = np.max(np.abs(rgrad[lo:hi]))
        assert np.max(d) <= 2e-2 * scale, (lo, float(np.max(d)), float(scale))
        cos = np.dot(grad[lo:hi], rgrad[lo:hi]) / (np.linalg.norm(grad[lo:hi]) * np.linalg.norm(rgrad[lo:hi]))
        assert cos > 0.999


def test_short_training_lowers_the_loss():
    ctx = fg.Context(0)
    rep = ctx.surrogate_train(n_receptors=4, min_atoms=1500, max_atoms=3000, points=33, spacing=0.375, epochs=8,
                              lr=3e-3, seed=3)
    ctx.close()
    print("TRAIN_SMALL " + json.dumps(rep))
    assert rep["steps"] == 32
    assert rep["last_epoch_loss"] < 0.5 * rep["first_epoch_loss"]


def _heldout(seed=900001, n=20000):
    return fg.surrogate_receptor(seed, n)


def test_shipped_weights_accuracy_and_gain():
    x = _heldout()
    g = fg.Grid(161, 161, 161, 0.375)
    eps = fg.ddd_table()
    ctx = fg.Context(0)
    direct = ctx.emap(g, x, eps)
    ctx.surrogate_load()
    ctx.surrogate_set(probe_tol=0.0)  # probes off: the network's own error
    surr, _ = ctx.emap_surrogate(g, x, eps)
    ctx.surrogate_set(probe_tol=0.0, use_corrector=False)
    tri, _ = ctx.emap_surrogate(g, x, eps)
    ctx.surrogate_set()  # defaults: probes and fallback on
    final, st = ctx.emap_surrogate(g, x, eps)
    ctx.close()
    err = np.abs(surr.astype(np.float64) - direct)
    err_tri = np.abs(tri.astype(np.float64) - direct)
    err_final = np.abs(final.astype(np.float64) - direct)
    rng = np.random.default_rng(1)
    idx = np.unique(np.concatenate([rng.choice(direct.size, 1500, replace=False), np.argsort(-err_final)[:200]]))
    ref = oracle.emap_points(g, x, eps, idx)
    err64 = np.abs(final[idx].astype(np.float64) - ref)
    rep = {"max_err_net": float(err.max()), "rms_err_net": float(np.sqrt(np.mean(err ** 2))),
           "max_err_trilinear": float(err_tri.max()), "rms_err_trilinear": float(np.sqrt(np.mean(err_tri ** 2))),
           "max_err_final": float(err_final.max()), "max_err_final_vs_fp64": float(err64.max()), **st}
    print("SURROGATE " + json.dumps(rep))
    assert rep["rms_err_net"] < 0.5 * rep["rms_err_trilinear"]
    assert rep["max_err_net"] < rep["max_err_trilinear"]
    assert rep["max_err_final"] <= 0.01
    assert rep["max_err_final_vs_fp64"] <= 0.01


def test_probe_fallback_reproduces_direct_sum():
    x = fg.surrogate_receptor(5, 3000)
    g = fg.Grid(49, 47, 45, 0.375)
    eps = fg.ddd_table()
    ctx = fg.Context(0)
    direct = ctx.emap(g, x, eps)
    # every probe fails at a zero tolerance: every box is recomputed directly
    ctx.surrogate_set(probe_tol=1e-12, use_corrector=False)
    out, st = ctx.emap_surrogate(g, x, eps)
    ctx.close()
    assert st["fallback_boxes"] == st["boxes"] > 0
    assert np.max(np.abs(out.astype(np.float64) - direct)) <= 1e-4


def test_tcgen05_corrector_matches_mma_sync():
    """The corrector's forward convolutions on tcgen05 (tensor memory
    accumulators) give the same map as the mma.sync kernels, up to the
    rounding of the BF16 activations between layers."""
    x = fg.surrogate_receptor(21, 6000)
    g = fg.Grid(45, 41, 37, 0.375)  # partial tiles on every axis
    eps = fg.ddd_table()
    ctx = fg.Context(0)
    ctx.surrogate_load()
    ctx.surrogate_set(probe_tol=0.0)
    ctx.tune(fg.AG_TUNE_SURROGATE_TCGEN05, 0)
    ref, _ = ctx.emap_surrogate(g, x, eps)
    ctx.tune(fg.AG_TUNE_SURROGATE_TCGEN05, 1)
    tc, _ = ctx.emap_surrogate(g, x, eps)
    tc2, _ = ctx.emap_surrogate(g, x, eps)
    ctx.close()
    assert np.array_equal(tc, tc2)
    assert np.max(np.abs(tc.astype(np.float64) - ref)) <= 2e-4
