"""GPU parity of the batched path (pmb_groupby_batched): many queries of one signature in one
persistent launch, each against the CPU oracle."""

import numpy as np
import pytest

from helpers import as_dict, assert_results_match, pack
from oracle import pyoracle
from polars_b200 import datagen
from polars_b200._native import ColumnData, Handle, groupby_batched

pytestmark = pytest.mark.gpu


def _np_query(rng, n, card, s, with_pred=True):
    ranks = np.minimum((rng.zipf(1.0 + s, n) if s > 0 else rng.integers(1, card + 1, n)) - 1, card - 1)
    key = ((ranks * 2654435761 + 12345) & 0x7FFFFFFF).astype(np.int32)
    v = rng.standard_normal(n)
    valid = rng.random(n) > 0.01
    cols = {"key": (key, None), "v": (v, pack(valid))}
    pred = datagen.PRED_BATCH if with_pred else None
    return cols, ["key"], datagen.AGGS_BATCH, pred


def _device_to_host(r):
    """A device-output result with its columns copied to host numpy arrays (CUDA runtime)."""
    import ctypes as C

    from polars_b200 import _abi as A

    rt = C.CDLL("libcudart.so.12")
    rt.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
    n = r.n_groups
    vb = max(4, ((n + 7) // 8 + 3) // 4 * 4)
    data, valid = [], []
    for ptr, vptr, dt in zip(r.data, r.validity, r.dtypes):
        nb = vb if dt == A.BOOL else n * A.DTYPE_BYTES[dt]
        d = np.zeros(max(nb, 1), np.uint8)
        v = np.zeros(vb, np.uint8)
        if nb:
            assert rt.cudaMemcpy(d.ctypes.data, ptr, nb, 2) == 0
        assert rt.cudaMemcpy(v.ctypes.data, vptr, (n + 7) // 8, 2) == 0
        data.append(d if dt == A.BOOL else d[:nb].view(A.NUMPY_NAME[dt]))
        valid.append(v)
    r.data, r.validity = data, valid
    return r


def _check(queries, results, label):
    for i, ((cols, keys, aggs, pred), got) in enumerate(zip(queries, results)):
        want = pyoracle.groupby(cols, keys, aggs, pred)
        assert_results_match(as_dict(got), want, len(keys), aggs, f"{label} query {i}")


def _product(q):
    cols, keys, aggs, pred = q
    return ({n: ColumnData(*c) for n, c in cols.items()}, keys, aggs, pred)


@pytest.mark.parametrize("output", ["host", "device"])
def test_batch_of_uneven_queries(output):
    rng = np.random.default_rng(1)
    sizes = [1, 50, 127, 128, 129, 1000, 4096, 30_000, 250_000, 1_200_000, 77, 65_536]
    cards = [1, 10, 100, 7, 129, 1000, 3000, 20_000, 200_000, 50, 5, 60_000]
    skews = [0.0, 0.5, 1.0, 1.5, 0.2, 1.1, 0.0, 0.8, 1.3, 0.0, 0.7, 1.0]
    queries = [_np_query(rng, n, c, s) for n, c, s in zip(sizes, cards, skews)]
    h = Handle(0)
    res = groupby_batched([_product(q) for q in queries], output=output, handle=h)
    if output == "device":
        res = [_device_to_host(r) for r in res]
    _check(queries, res, f"batch {output}")


def test_batch_matches_single_queries_and_reruns_wider_float_range():
    rng = np.random.default_rng(2)
    queries = [_np_query(rng, n, c, 1.0) for n, c in [(100_000, 1000), (300_000, 50_000), (20_000, 10)]]
    # a float outside the sampled range (row 1 is not sampled): the query re-runs with a wider range
    queries[1][0]["v"][0][1] = 3.0e30
    res = groupby_batched([_product(q) for q in queries], handle=Handle(0))
    _check(queries, res, "rerun")


def test_mixed_signatures_run_one_by_one():
    rng = np.random.default_rng(3)
    a = _np_query(rng, 10_000, 100, 0.5)
    b = _np_query(rng, 10_000, 100, 0.5, with_pred=False)
    res = groupby_batched([_product(a), _product(b)], handle=Handle(0))
    _check([a, b], res, "mixed")
    with pytest.raises(NotImplementedError):
        groupby_batched([_product(a), _product(b)], output="device", handle=Handle(0))


def test_overflow_in_batch_reruns_larger(monkeypatch):
    # a capacity far below the group count: the query's table overflows and it runs again
    monkeypatch.setenv("PMB_GCAP_MULT", "0.02")
    rng = np.random.default_rng(4)
    queries = [_np_query(rng, 200_000, 150_000, 0.0), _np_query(rng, 50_000, 100, 1.0)]
    res = groupby_batched([_product(q) for q in queries], handle=Handle(0))
    _check(queries, res, "overflow")


def test_prepared_batch_twice_and_the_plain_loop_switch():
    # a batch prepared once gives the same results on two calls; with batching off the same
    # batch runs query by query inside the library, with the same results again
    from polars_b200._native import prepare_batched

    rng = np.random.default_rng(41)
    qs = []
    for n, card, s in [(30_000, 50, 0.8), (120_000, 5_000, 0.0), (70_000, 900, 1.2)]:
        cols, keys, aggs, pred = _np_query(rng, n, card, s)
        qs.append(({k: ColumnData(*v) for k, v in cols.items()}, keys, aggs, pred))
    prep = prepare_batched(qs, output="host")
    first = groupby_batched(prep)
    second = groupby_batched(prep)
    h = Handle(0)
    h.set_batching(False)
    loop = groupby_batched(prep, handle=h)
    h.close()
    for (cols, keys, aggs, pred), a, b, c in zip(qs, first, second, loop):
        np_cols = {k: (v.data, v.validity) for k, v in cols.items()}
        want = pyoracle.groupby(np_cols, keys, aggs, pred)
        for got, label in ((a, "prepared 1"), (b, "prepared 2"), (c, "plain loop")):
            assert_results_match(as_dict(got), want, 1, aggs, label)
