"""Seeded synthetic tables with the shapes and value distributions of the benchmark workloads.

Generation runs in torch (on the GPU when `device="cuda"`, which is what makes a 100M-row
table quick to build) and is excluded from every timed region. Null masks are Bernoulli per
cell; validity bitmaps are Arrow-layout (LSB first, 1 = valid). Zipf keys are bounded: ranks
1..K with P(k) ~ k^-s, mapped to key values by a fixed random permutation so hot keys are not
numerically adjacent.

Workloads:
  small    1M rows; key int64 U[0,1000); v1 float64 N(0,1); v2 int64 U[-1e6,1e6];
           1% nulls on v1, v2; filter v1 > 0; sum/mean(v1), min/max(v2), len
  hash     100M rows; key int32 Zipf(s=1.1) over 1M values; v1, v2 float64 N(0,1);
           v3 int64 U[0,1e9); 5% nulls on v1, v2, v3; filter (v1 > -0.5) & (v3 % 7 != 0);
           sum/mean(v1), min/max(v2), sum(v3), len
  sort     200M rows; keys int64 drawn from 781,250 values in [0, 2^40) and int32 U[0,64)
           (about 50M distinct pairs); v float32 U(0,1), vi int64; no filter; sum/min/max/len
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _abi as A


def _torch():
    import torch

    return torch


def pack_bits(mask) -> "object":
    """Bool tensor (n,) -> uint8 bitmap, LSB first (torch, same device)."""
    torch = _torch()
    n = mask.numel()
    pad = (-n) % 8
    m = mask.to(torch.uint8)
    if pad:
        m = torch.cat([m, torch.zeros(pad, dtype=torch.uint8, device=m.device)])
    w = torch.tensor([1, 2, 4, 8, 16, 32, 64, 128], dtype=torch.uint8, device=m.device)
    return (m.view(-1, 8) * w).sum(dim=1, dtype=torch.uint8)


def unpack_bits(bitmap: np.ndarray, n: int) -> np.ndarray:
    return np.unpackbits(np.asarray(bitmap, dtype=np.uint8), bitorder="little")[:n].astype(bool)


def zipf_keys(n: int, n_values: int, s: float, gen, device, dtype):
    torch = _torch()
    ranks = torch.arange(1, n_values + 1, dtype=torch.float64, device=device)
    p = ranks.pow(-s)
    cdf = torch.cumsum(p, 0)
    cdf = cdf / cdf[-1]
    u = torch.rand(n, generator=gen, dtype=torch.float64, device=device)
    idx = torch.searchsorted(cdf, u).clamp_(max=n_values - 1)
    perm = torch.randperm(n_values, generator=gen, device=device)
    return perm[idx].to(dtype)


@dataclass
class Table:
    """Columns as (data, validity-bitmap-or-None) torch tensors, plus the query to run."""

    columns: dict
    keys: list
    aggs: list
    predicate: dict | None
    n_rows: int
    name: str

    def bytes_per_row(self) -> float:
        """Algorithmic input bytes per row: every touched column read once (values + validity bits)."""
        total = 0.0
        for data, valid in self.columns.values():
            total += data.element_size()
            if valid is not None:
                total += 1.0 / 8.0
        return total

    def to(self, device):
        cols = {k: (d.to(device), None if v is None else v.to(device)) for k, (d, v) in self.columns.items()}
        return Table(cols, self.keys, self.aggs, self.predicate, self.n_rows, self.name)

    def slice(self, n: int) -> "Table":
        """First n rows (n a multiple of 8 keeps bitmaps byte-aligned)."""
        assert n % 8 == 0 or n == self.n_rows
        cols = {k: (d[:n], None if v is None else v[: (n + 7) // 8]) for k, (d, v) in self.columns.items()}
        return Table(cols, self.keys, self.aggs, self.predicate, n, self.name)


def _gen(seed: int, device):
    torch = _torch()
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    return g


def _nulls(n, frac, gen, device):
    torch = _torch()
    if frac <= 0:
        return None
    keep = torch.rand(n, generator=gen, device=device) >= frac
    return pack_bits(keep)


PRED_SMALL = {
    "kind": "Compare",
    "op": "Gt",
    "dtype": "F64",
    "lhs": {"kind": "Column", "name": "v1", "dtype": "F64"},
    "rhs": {"kind": "LiteralF64", "value": 0.0},
}

PRED_HASH = {
    "kind": "And",
    "lhs": {
        "kind": "Compare",
        "op": "Gt",
        "dtype": "F64",
        "lhs": {"kind": "Column", "name": "v1", "dtype": "F64"},
        "rhs": {"kind": "LiteralF64", "value": -0.5},
    },
    "rhs": {
        "kind": "Compare",
        "op": "Ne",
        "dtype": "I64",
        "lhs": {
            "kind": "Arith",
            "op": "Mod",
            "dtype": "I64",
            "lhs": {"kind": "Column", "name": "v3", "dtype": "I64"},
            "rhs": {"kind": "LiteralI64", "value": 7},
        },
        "rhs": {"kind": "LiteralI64", "value": 0},
    },
}


def make_small(n: int = 1_000_000, seed: int = 1, device="cpu", null_frac: float = 0.01) -> Table:
    torch = _torch()
    g = _gen(seed, device)
    key = torch.randint(0, 1000, (n,), generator=g, device=device, dtype=torch.int64)
    v1 = torch.randn(n, generator=g, device=device, dtype=torch.float64)
    v2 = torch.randint(-1_000_000, 1_000_001, (n,), generator=g, device=device, dtype=torch.int64)
    cols = {
        "key": (key, None),
        "v1": (v1, _nulls(n, null_frac, g, device)),
        "v2": (v2, _nulls(n, null_frac, g, device)),
    }
    aggs = [("Sum", "v1", "v1_sum"), ("Mean", "v1", "v1_mean"), ("Min", "v2", "v2_min"), ("Max", "v2", "v2_max"),
            ("Len", None, "count")]
    return Table(cols, ["key"], aggs, PRED_SMALL, n, "small")


def make_hash(n: int = 100_000_000, seed: int = 2, device="cpu", n_values: int = 1_000_000, s: float = 1.1,
              null_frac: float = 0.05) -> Table:
    torch = _torch()
    g = _gen(seed, device)
    key = zipf_keys(n, n_values, s, g, device, torch.int32)
    v1 = torch.randn(n, generator=g, device=device, dtype=torch.float64)
    v2 = torch.randn(n, generator=g, device=device, dtype=torch.float64)
    v3 = torch.randint(0, 1_000_000_000, (n,), generator=g, device=device, dtype=torch.int64)
    cols = {
        "key": (key, None),
        "v1": (v1, _nulls(n, null_frac, g, device)),
        "v2": (v2, _nulls(n, null_frac, g, device)),
        "v3": (v3, _nulls(n, null_frac, g, device)),
    }
    aggs = [("Sum", "v1", "v1_sum"), ("Mean", "v1", "v1_mean"), ("Min", "v2", "v2_min"), ("Max", "v2", "v2_max"),
            ("Sum", "v3", "v3_sum"), ("Len", None, "count")]
    return Table(cols, ["key"], aggs, PRED_HASH, n, "hash")


def make_sort(n: int = 200_000_000, seed: int = 3, device="cpu", pool: int = 781_250) -> Table:
    torch = _torch()
    g = _gen(seed, device)
    values = torch.randint(0, 1 << 40, (pool,), generator=g, device=device, dtype=torch.int64)
    k1 = values[torch.randint(0, pool, (n,), generator=g, device=device)]
    k2 = torch.randint(0, 64, (n,), generator=g, device=device, dtype=torch.int32)
    v = torch.rand(n, generator=g, device=device, dtype=torch.float32)
    vi = torch.randint(-(1 << 40), 1 << 40, (n,), generator=g, device=device, dtype=torch.int64)
    cols = {"k1": (k1, None), "k2": (k2, None), "v": (v, None), "vi": (vi, None)}
    aggs = [("Sum", "v", "v_sum"), ("Min", "v", "v_min"), ("Max", "v", "v_max"), ("Sum", "vi", "vi_sum"),
            ("Min", "vi", "vi_min"), ("Max", "vi", "vi_max"), ("Len", None, "count")]
    return Table(cols, ["k1", "k2"], aggs, None, n, "sort")


PRED_BATCH = {"kind": "Compare", "op": "Gt", "lhs": {"kind": "Column", "name": "v"},
              "rhs": {"kind": "LiteralF64", "value": -1.0}}
AGGS_BATCH = [("Sum", "v", "v_sum"), ("Mean", "v", "v_mean"), ("Min", "v", "v_min"), ("Max", "v", "v_max"),
              ("Len", None, "count")]


def batch_sizes(n_queries: int, seed: int, mu: float = 11.512925464970229, sigma: float = 1.5,
                lo: int = 1000, hi: int = 10_000_000):
    """Per-query rows (lognormal(mu = ln 1e5, sigma), clipped), cardinality (log-uniform in
    [10, 1e6], at most the rows) and Zipf skew (uniform in [0, 1.5]) of the batched workload."""
    rng = np.random.default_rng(seed)
    rows = np.clip(np.exp(rng.normal(mu, sigma, n_queries)), lo, hi).astype(np.int64)
    card = np.exp(rng.uniform(np.log(10), np.log(1e6), n_queries)).astype(np.int64)
    card = np.minimum(card, rows)
    s = rng.uniform(0.0, 1.5, n_queries)
    return rows, card, s


def make_batch(n_queries: int = 4096, seed: int = 4, device="cpu", max_total: int | None = None,
               stop_rows: int | None = None):
    """Independent filter -> group_by queries: key int32 (Zipf over its cardinality), v float64
    N(0,1) with 1% nulls; filter v > -1; sum/mean/min/max(v), len. Returns Tables. With
    `stop_rows`, only the leading queries up to that many rows are made (the same ones as in
    the full batch on the same device)."""
    torch = _torch()
    rows, card, s = batch_sizes(n_queries, seed)
    if max_total is not None and rows.sum() > max_total:
        rows = np.maximum(1000, (rows * (max_total / rows.sum())).astype(np.int64))
        card = np.minimum(card, rows)
    g = _gen(seed, device)
    out = []
    made = 0
    for i in range(n_queries):
        if stop_rows is not None and made >= stop_rows:
            break
        made += int(rows[i])
        n, d = int(rows[i]), int(max(card[i], 1))
        k = zipf_keys(n, d, float(s[i]), g, device, torch.int64)
        k = ((k * 0x9E3779B1 + i) & 0x7FFFFFFF).to(torch.int32)
        v = torch.randn(n, generator=g, device=device, dtype=torch.float64)
        cols = {"key": (k, None), "v": (v, _nulls(n, 0.01, g, device))}
        out.append(Table(cols, ["key"], AGGS_BATCH, PRED_BATCH, n, f"batch{i}"))
    return out


def to_column_data(t: Table) -> dict:
    """Table -> {name: ColumnData} (torch tensors; zero-copy when on the GPU)."""
    from ._native import ColumnData

    torch = _torch()
    out = {}
    for name, (d, v) in t.columns.items():
        dt = {
            torch.int8: A.I8,
            torch.int16: A.I16,
            torch.int32: A.I32,
            torch.int64: A.I64,
            torch.uint8: A.U8,
            torch.float32: A.F32,
            torch.float64: A.F64,
        }[d.dtype]
        out[name] = ColumnData(d, v, dtype=dt, length=t.n_rows)
    return out


def to_numpy_columns(t: Table) -> dict:
    """Table -> {name: (numpy data, numpy bitmap or None)} on the host."""
    return {k: (d.cpu().numpy(), None if v is None else v.cpu().numpy()) for k, (d, v) in t.columns.items()}
