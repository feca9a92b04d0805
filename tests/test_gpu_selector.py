"""The learned strategy selector on the GPU: the device MLP kernels against the numpy oracle,
training with them, the device features, and AUTO with the selector giving exact results."""

import numpy as np
import pytest

from helpers import as_dict, assert_results_match
from oracle import mlp
from polars_b200 import _abi as A
from polars_b200 import selector as S
from polars_b200._native import ColumnData, Handle, groupby, mlp_adam_step, mlp_forward, mlp_gradient, \
    selector_features

pytestmark = pytest.mark.gpu


def _t(a, dtype=None):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a, dtype=dtype)).cuda()


def test_forward_gradient_and_adam_match_the_oracle():
    rng = np.random.default_rng(1)
    h = Handle(0, selector=None)
    p = S.init_params(5)
    X = rng.random((200, mlp.NF)).astype(np.float32)
    cls = rng.integers(0, mlp.NS, 200).astype(np.int32)
    y = (rng.random(200) * 25).astype(np.float32)
    sw = (rng.random(200) + 0.5).astype(np.float32)
    out = mlp_forward(_t(p), _t(X), handle=h).cpu().numpy()
    np.testing.assert_allclose(out, mlp.forward(p, X), rtol=1e-4, atol=1e-5)
    g, loss = mlp_gradient(_t(p), _t(X), _t(cls), _t(y), _t(sw), wreg=0.1, handle=h)
    want_loss, want_g = mlp.loss_and_grad(p, X, cls, y, sw, wreg=0.1)
    assert loss == pytest.approx(want_loss, rel=1e-4)
    np.testing.assert_allclose(g.cpu().numpy(), want_g, rtol=1e-3, atol=1e-6)
    pd, m, v = _t(p), _t(np.zeros_like(p)), _t(np.zeros_like(p))
    mlp_adam_step(pd, g, m, v, 1, 1e-2, handle=h)
    want_p, _, _ = mlp.adam_step(p.astype(np.float64), g.cpu().numpy().astype(np.float64), 0, 0, 1, 1e-2)
    np.testing.assert_allclose(pd.cpu().numpy(), want_p, rtol=1e-5, atol=1e-6)


def test_training_with_the_device_kernels_learns_a_rule():
    rng = np.random.default_rng(2)
    n = 2048
    X = rng.random((n, mlp.NF)).astype(np.float32)
    # the fastest strategy follows feature 4 (sample distinct fraction), like a cardinality rule
    T = np.stack([1 + 4 * X[:, 4], 2 - X[:, 4], 1 + 3 * (1 - X[:, 4]), 1.5 + 2 * np.abs(X[:, 4] - 0.5)], axis=1)
    G = (2 ** (20 * X[:, 13])).astype(np.int64)
    p, hist = S.train(X, T, G, epochs=60, batch=256, lr=5e-3)
    assert hist[-1] < 0.5 * hist[0]
    pred = np.argmax(mlp.forward(p, X)[:, :mlp.NS], axis=1)
    assert np.mean(pred == np.argmin(T, axis=1)) > 0.9


def test_features_of_known_tables():
    h = Handle(0, selector=None)
    n = 200_000
    rng = np.random.default_rng(3)
    v = ColumnData(rng.standard_normal(n))
    aggs = [("Sum", "v", "s"), ("Len", None, "n")]
    f = selector_features({"k": ColumnData(np.arange(n, dtype=np.int64)), "v": v}, ["k"], aggs, handle=h)
    assert f[4] == pytest.approx(1.0) and f[22] == 1.0 and f[5] == pytest.approx(1.0)  # all distinct
    f = selector_features({"k": ColumnData(np.arange(n, dtype=np.int64) % 10), "v": v}, ["k"], aggs, handle=h)
    assert f[4] == pytest.approx(10 / 4096) and f[22] == 0.0 and f[2] == 0.0
    valid = rng.random(n) > 0.3
    k = ColumnData(rng.integers(0, 1000, n).astype(np.int32), np.packbits(valid, bitorder="little"))
    f = selector_features({"k": k, "v": v}, ["k"], aggs, handle=h)
    assert f[2] == pytest.approx(0.3, abs=0.03) and f[1] == pytest.approx(33 / 128)
    pred = {"kind": "Compare", "op": "Gt", "lhs": {"kind": "Column", "name": "v"}, "rhs": {"kind": "LiteralF64", "value": 0.0}}
    f = selector_features({"k": k, "v": v}, ["k"], aggs, pred, handle=h)
    assert f[3] == pytest.approx(0.5, abs=0.03) and f[20] == 1.0


@pytest.mark.skipif(S.default_params() is None, reason="no shipped selector")
def test_auto_with_the_selector_is_exact():
    learned, plain = Handle(0), Handle(0, selector=None)
    for sp in S.sample_specs(12, seed=99, max_rows=3e6):
        cols, keys = S.make_table(sp)
        a = groupby(cols, keys, S.AGGS, handle=learned)
        b = groupby(cols, keys, S.AGGS, handle=plain)
        assert_results_match(as_dict(a), as_dict(b), len(keys), S.AGGS, f"{sp} ({a.strategy} vs {b.strategy})")
