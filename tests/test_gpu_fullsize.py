"""GPU parity at the benchmarked sizes: the hash workload at its full 100M rows (Zipf hot keys
holding tens of millions of rows, fixed-point sum widths of 100M rows), the sort workload at
200M rows with ~49M groups, and every query of the 4096-query batch, each against the CPU
oracle on the same seeded inputs. Inputs are generated on the GPU and copied to the host for the
oracle."""

import pytest

from helpers import as_dict, assert_results_match
from oracle import pyoracle
from polars_b200 import datagen
from polars_b200._native import groupby, groupby_batched

pytestmark = pytest.mark.gpu


def _free():
    import torch

    torch.cuda.synchronize()
    torch.cuda.empty_cache()


def test_hash_workload_parity_at_100m_rows():
    t = datagen.make_hash(100_000_000, seed=1234, device="cuda")
    got = groupby(datagen.to_column_data(t), t.keys, t.aggs, t.predicate)
    want = pyoracle.groupby(datagen.to_numpy_columns(t), t.keys, t.aggs, t.predicate)
    assert got.n_groups > 900_000
    assert_results_match(as_dict(got), want, 1, t.aggs, "hash 100M")
    del t
    _free()


@pytest.mark.parametrize("strategy", ["auto", "sort"])
def test_sort_workload_parity_at_200m_rows(strategy):
    t = datagen.make_sort(200_000_000, seed=1234, device="cuda")
    got = groupby(datagen.to_column_data(t), t.keys, t.aggs, None, strategy=strategy)
    want = pyoracle.groupby(datagen.to_numpy_columns(t), t.keys, t.aggs, None)
    assert got.n_groups > 40_000_000
    assert_results_match(as_dict(got), want, len(t.keys), t.aggs, f"sort 200M {strategy}")
    del t
    _free()


def test_every_query_of_the_full_batch():
    tables = datagen.make_batch(4096, seed=4, device="cuda", max_total=500_000_000)
    qs = [(datagen.to_column_data(b), b.keys, b.aggs, b.predicate) for b in tables]
    res = groupby_batched(qs)
    assert len(res) == 4096
    for i, (b, got) in enumerate(zip(tables, res)):
        want = pyoracle.groupby(datagen.to_numpy_columns(b), b.keys, b.aggs, b.predicate)
        assert_results_match(as_dict(got), want, 1, b.aggs, f"batch query {i}")
    del tables, qs
    _free()
