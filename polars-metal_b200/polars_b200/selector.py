"""The learned strategy selector: training data, training and evaluation.

The network (include/pmb.h, PMB_SELECTOR_*) reads device-computed features of a 4096-row key
sample and scores the four group-by strategies (shared-memory hash, global hash, sort,
partitioned) and predicts log2 of the group count. This module

  * generates synthetic tables like the learned-selection workload (rows log-uniform, key width
    int32 / int64 / 2 x int64, distinct count log-uniform, Zipf skew, null fraction);
  * collects, per table, the features, the device time of every strategy and the exact group
    count, measured by the engine itself (`collect`);
  * trains the network on the GPU with libpmb's own forward / backward / Adam kernels (`train`);
  * evaluates picks against the plain cardinality heuristic and the best strategy per table
    (`evaluate`), replaying the measured times.

Command line (on a GPU machine):
    python -m polars_b200.selector collect --tables 2000 --out data.npz
    python -m polars_b200.selector train --data data.npz --out selector_params.npy
    python -m polars_b200.selector report --data data.npz
"""

from __future__ import annotations

import argparse
import math
import time
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import _abi as A

PKG = Path(__file__).resolve().parent
PARAMS_FILE = PKG / "data" / "selector_params.npy"
DATASET_FILE = PKG / "data" / "selector_dataset.npz"
# tables of the same distribution with a filter on most of them: the network is applied to filtered
# queries too (the hash workload, the batched queries), so it trains on some
FILTERED_FILE = PKG / "data" / "selector_dataset_filtered.npz"
STRATEGIES = A.SELECTOR_STRATEGIES  # score index -> strategy name
KEY_KINDS = ["i32", "i64", "2xi64"]
_M64 = 0x9E3779B97F4A7C15 - (1 << 64)  # an odd 64-bit multiplier, as a signed int64
AGGS = [("Sum", "v", "s"), ("Mean", "v", "m"), ("Min", "v", "lo"), ("Max", "v", "hi"), ("Len", None, "n")]


def default_params() -> np.ndarray | None:
    """The parameters shipped with the package (None when absent)."""
    if PARAMS_FILE.exists():
        p = np.load(PARAMS_FILE).astype(np.float32)
        if p.size == A.SELECTOR_PARAMS and np.all(np.isfinite(p)):
            return p
    return None


@dataclass
class TableSpec:
    rows: int
    key: str        # one of KEY_KINDS
    distinct: int
    zipf: float
    null_frac: float
    seed: int
    keep: float = 1.0  # < 1: the query filters v > t, keeping this fraction of the rows


def predicate_of(spec: TableSpec) -> dict | None:
    """The filter of a spec: v > t with P(v > t) = keep for v ~ N(0,1); None when keep is 1."""
    if spec.keep >= 1.0:
        return None
    from statistics import NormalDist

    t = NormalDist().inv_cdf(1.0 - spec.keep)
    return {"kind": "Compare", "op": "Gt", "lhs": {"kind": "Column", "name": "v"},
            "rhs": {"kind": "LiteralF64", "value": float(t)}}


def sample_specs(n: int, seed: int, min_rows: float = 1e5, max_rows: float = 1e8, max_distinct: float = 1e8,
                 filter_frac: float = 0.0):
    """Table specs of the learned-selection workload: rows log-uniform in [min_rows, max_rows],
    distinct count log-uniform in [10, min(max_distinct, rows)], Zipf s uniform in [0, 2], null
    fraction uniform in [0, 0.2], key width uniform over int32 / int64 / 2 x int64. With
    `filter_frac` > 0 that fraction of the tables also gets a filter keeping U[0.05, 1) of the rows
    (drawn from a separate stream, so the tables themselves do not change)."""
    rng = np.random.default_rng(seed)
    frng = np.random.default_rng(seed + 7919)
    out = []
    for i in range(n):
        rows = int(math.exp(rng.uniform(math.log(min_rows), math.log(max_rows))))
        hi = min(max_distinct, rows)
        distinct = int(math.exp(rng.uniform(math.log(10), math.log(max(hi, 11)))))
        keep = float(frng.uniform(0.05, 1.0)) if frng.random() < filter_frac else 1.0
        out.append(TableSpec(rows, KEY_KINDS[rng.integers(0, 3)], max(1, distinct), float(rng.uniform(0, 2)),
                             float(rng.uniform(0, 0.2)), int(rng.integers(0, 2**31 - 1)), keep))
    return out


def _ranks(n: int, d: int, s: float, g, device):
    """Ranks in [0, d) with P(rank k) ~ (k + 1)^-s: exact inverse CDF up to 2^21 values, the
    continuous bounded power law beyond."""
    import torch

    if d <= (1 << 21):
        k = torch.arange(1, d + 1, dtype=torch.float64, device=device).pow(-s)
        cdf = torch.cumsum(k, 0)
        cdf /= cdf[-1].clone()
        u = torch.rand(n, generator=g, dtype=torch.float64, device=device)
        return torch.searchsorted(cdf, u).clamp_(max=d - 1)
    u = torch.rand(n, generator=g, dtype=torch.float64, device=device)
    if abs(s - 1.0) < 1e-6:
        x = torch.exp(u * math.log(d))
    else:
        a = 1.0 - s
        x = (u * (d ** a - 1.0) + 1.0).pow(1.0 / a)
    return (x.floor().to(torch.int64) - 1).clamp_(0, d - 1)


def make_table(spec: TableSpec, device="cuda"):
    """Columns {name: ColumnData} of one synthetic table (keys from the spec; v float64 N(0,1))."""
    import torch

    from . import datagen
    from ._native import ColumnData

    g = datagen._gen(spec.seed, device)
    n = spec.rows
    r = _ranks(n, spec.distinct, spec.zipf, g, device)
    cols = {}
    # rank -> key value by an odd multiplier (a bijection), so hot keys are not numerically adjacent
    if spec.key == "i32":
        k = ((r * 0x9E3779B1 + 0x1234567) & 0xFFFFFFFF).to(torch.int64)
        k = torch.where(k >= 2**31, k - 2**32, k).to(torch.int32)
        cols["k1"] = ColumnData(k, datagen._nulls(n, spec.null_frac, g, device), dtype=A.I32, length=n)
        keys = ["k1"]
    elif spec.key == "i64":
        cols["k1"] = ColumnData(r * _M64 + 0x5851F42D, datagen._nulls(n, spec.null_frac, g, device), dtype=A.I64,
                                length=n)
        keys = ["k1"]
    else:
        # two full-width int64 keys fill the 128-bit packed key, so they carry no null bit here; the
        # value column still has nulls
        cols["k1"] = ColumnData(r * _M64 + 0x5851F42D, None, dtype=A.I64, length=n)
        cols["k2"] = ColumnData((r ^ 0x2545F491) * 0x4F1BBCDCBFA53E0B, None, dtype=A.I64, length=n)
        keys = ["k1", "k2"]
    v = torch.randn(n, generator=g, dtype=torch.float64, device=device)
    cols["v"] = ColumnData(v, datagen._nulls(n, spec.null_frac, g, device), dtype=A.F64, length=n)
    return cols, keys


def collect(specs, reps: int = 2, log=None, budget_s: float = 0.0) -> dict:
    """Features, per-strategy device time (ms, best of `reps`), the heuristic's pick and the
    exact group count of every table, measured on the current GPU. With `budget_s` > 0 the
    collection stops after the table that crosses that many seconds (`seconds` in the result
    holds the time taken)."""
    import torch

    from ._native import Handle, groupby, selector_choose, selector_features

    h = Handle(0, selector=None)  # features and the heuristic without a learned selector
    X, T, G, H, S = [], [], [], [], []
    t0 = time.time()
    warmed = set()  # (key width, strategy): the run-time compile happens in the first such call
    for i, sp in enumerate(specs):
        cols, keys = make_table(sp)
        pred = predicate_of(sp)
        torch.cuda.synchronize()
        X.append(selector_features(cols, keys, AGGS, pred, handle=h))
        heur, _ = selector_choose(cols, keys, AGGS, pred, handle=h)
        H.append(STRATEGIES.index(heur) if heur in STRATEGIES else 1)
        times, groups = [], None
        for s in STRATEGIES:
            if (sp.key, s, sp.null_frac > 0) not in warmed:
                groupby(cols, keys, AGGS, pred, strategy=s, output="device", handle=h)  # warm-up (run-time compile)
                warmed.add((sp.key, s, sp.null_frac > 0))
            best = float("inf")
            h.set_profiling(True)
            for _ in range(reps):
                res = groupby(cols, keys, AGGS, pred, strategy=s, output="device", handle=h)
                best = min(best, h.last_stats()["total_ms"])
            h.set_profiling(False)
            groups = res.n_groups if groups is None else groups
            if res.n_groups != groups:
                raise RuntimeError(f"strategies disagree on the group count for {sp}")
            times.append(best)
        T.append(times)
        G.append(groups)
        S.append([sp.rows, KEY_KINDS.index(sp.key), sp.distinct, sp.zipf, sp.null_frac, sp.keep])
        del cols
        if log and (i + 1) % 50 == 0:
            log(f"{i + 1}/{len(specs)} tables, {time.time() - t0:.0f} s")
        if budget_s > 0 and time.time() - t0 > budget_s:
            break
    h.close()
    return {"X": np.array(X, np.float32), "T": np.array(T, np.float64), "G": np.array(G, np.int64),
            "H": np.array(H, np.int32), "S": np.array(S, np.float64), "seconds": np.float64(time.time() - t0)}


def labels(T: np.ndarray, G: np.ndarray):
    """Best strategy per table, a weight per table (how much choosing matters: worst / best time,
    capped) and the regression target log2(groups)."""
    cls = np.argmin(T, axis=1).astype(np.int32)
    sw = np.clip(T.max(axis=1) / np.maximum(T.min(axis=1), 1e-6), 1.0, 10.0).astype(np.float32)
    y = np.log2(np.maximum(G, 1)).astype(np.float32)
    return cls, sw, y


def init_params(seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    F, Hd, O = A.SELECTOR_FEATURES, A.SELECTOR_HIDDEN, A.SELECTOR_OUTPUTS
    parts = [rng.normal(0, math.sqrt(2.0 / F), Hd * F), np.zeros(Hd),
             rng.normal(0, math.sqrt(2.0 / Hd), Hd * Hd), np.zeros(Hd),
             rng.normal(0, math.sqrt(1.0 / Hd), O * Hd), np.zeros(O)]
    return np.concatenate(parts).astype(np.float32)


def train(X, T, G, epochs: int = 400, batch: int = 256, lr: float = 3e-3, wreg: float = 0.05, seed: int = 0,
          log=None) -> tuple[np.ndarray, list]:
    """Trains the selector on the GPU with libpmb's kernels; returns (parameters, loss per epoch)."""
    import torch

    from ._native import Handle, mlp_adam_step, mlp_gradient

    h = Handle(0, selector=None)
    cls, sw, y = labels(T, G)
    dev = torch.device("cuda")
    Xd = torch.from_numpy(np.ascontiguousarray(X, np.float32)).to(dev)
    Cd = torch.from_numpy(cls).to(dev)
    Sd = torch.from_numpy(sw).to(dev)
    Yd = torch.from_numpy(y).to(dev)
    p0 = init_params(seed)
    p0[-1] = float(y.mean())  # the group-count output starts at the mean target
    p = torch.from_numpy(p0).to(dev)
    m = torch.zeros_like(p)
    v = torch.zeros_like(p)
    g = torch.Generator(device="cpu")
    g.manual_seed(seed)
    n = X.shape[0]
    step, hist = 0, []
    for ep in range(epochs):
        perm = torch.randperm(n, generator=g).to(dev)
        tot = 0.0
        for b0 in range(0, n, batch):
            idx = perm[b0:b0 + batch]
            grad, loss = mlp_gradient(p, Xd[idx].contiguous(), Cd[idx].contiguous(), Yd[idx].contiguous(),
                                      Sd[idx].contiguous(), wreg=wreg, handle=h)
            step += 1
            mlp_adam_step(p, grad, m, v, step, lr, handle=h)
            tot += loss * idx.numel()
        hist.append(tot / n)
        if log and (ep + 1) % 50 == 0:
            log(f"epoch {ep + 1}: loss {hist[-1]:.4f}")
    out = p.cpu().numpy()
    h.close()
    return out, hist


def predict(params: np.ndarray, X: np.ndarray) -> np.ndarray:
    """The network's outputs [n, 4] for features X [n, 24], computed by the device kernel."""
    import torch

    from ._native import Handle, mlp_forward

    h = Handle(0, selector=None)
    out = mlp_forward(torch.from_numpy(np.ascontiguousarray(params, np.float32)).cuda(),
                      torch.from_numpy(np.ascontiguousarray(X, np.float32)).cuda(), handle=h)
    res = out.cpu().numpy()
    h.close()
    return res


def evaluate(picks: np.ndarray, T: np.ndarray, H: np.ndarray) -> dict:
    """Total measured time of the picks against the heuristic's picks and the best per table."""
    rows = np.arange(T.shape[0])
    t_pick = float(T[rows, picks].sum())
    t_heur = float(T[rows, H].sum())
    t_best = float(T.min(axis=1).sum())
    return {"tables": int(T.shape[0]), "ms_learned": t_pick, "ms_heuristic": t_heur, "ms_best": t_best,
            "gain_vs_heuristic": t_heur / t_pick, "learned_vs_best": t_pick / t_best,
            "accuracy_learned": float(np.mean(picks == np.argmin(T, axis=1))),
            "accuracy_heuristic": float(np.mean(H == np.argmin(T, axis=1)))}


def evaluate_live(specs, params, reps: int = 2, log=None) -> dict:
    """Measured device time of the AUTO strategy with the selector `params` and with the plain
    heuristic on fresh tables (best of `reps` calls each; the selector's own feature and MLP
    kernels are inside the learned side's time), plus both sides' rehash counts."""
    import torch

    from ._native import Handle, groupby

    learned, plain = Handle(0, selector=params), Handle(0, selector=None)
    tot = {"learned": 0.0, "heuristic": 0.0}
    rehash = {"learned": 0, "heuristic": 0}
    picks = {"learned": {}, "heuristic": {}}
    for i, sp in enumerate(specs):
        cols, keys = make_table(sp)
        pred = predicate_of(sp)
        torch.cuda.synchronize()
        for name, h in (("learned", learned), ("heuristic", plain)):
            groupby(cols, keys, AGGS, pred, output="device", handle=h)
            h.set_profiling(True)
            best = float("inf")
            for _ in range(reps):
                res = groupby(cols, keys, AGGS, pred, output="device", handle=h)
                best = min(best, h.last_stats()["total_ms"])
            h.set_profiling(False)
            tot[name] += best
            rehash[name] += res.rehash_count
            picks[name][res.strategy] = picks[name].get(res.strategy, 0) + 1
        del cols
        if log and (i + 1) % 50 == 0:
            log(f"{i + 1}/{len(specs)} tables")
    learned.close()
    plain.close()
    return {"tables": len(specs), "ms_learned": tot["learned"], "ms_heuristic": tot["heuristic"],
            "gain_vs_heuristic": tot["heuristic"] / tot["learned"], "rehash_learned": rehash["learned"],
            "rehash_heuristic": rehash["heuristic"], "picks": picks}


def split(n: int, test_frac: float = 0.25, seed: int = 7):
    rng = np.random.default_rng(seed)
    perm = rng.permutation(n)
    k = int(n * (1 - test_frac))
    return perm[:k], perm[k:]


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m polars_b200.selector")
    sub = ap.add_subparsers(dest="cmd", required=True)
    c = sub.add_parser("collect")
    c.add_argument("--tables", type=int, default=2000)
    c.add_argument("--seed", type=int, default=1)
    c.add_argument("--max-rows", type=float, default=2e7)
    c.add_argument("--out", default=str(DATASET_FILE))
    c.add_argument("--budget-s", type=float, default=0.0, help="stop after this many seconds of collection")
    c.add_argument("--filter-frac", type=float, default=0.0, help="fraction of the tables that get a filter")
    t = sub.add_parser("train")
    t.add_argument("--data", default=str(DATASET_FILE))
    t.add_argument("--out", default=str(PARAMS_FILE))
    t.add_argument("--epochs", type=int, default=400)
    r = sub.add_parser("report")
    r.add_argument("--data", default=str(DATASET_FILE))
    r.add_argument("--params", default=str(PARAMS_FILE))
    lv = sub.add_parser("live")
    lv.add_argument("--params", default=str(PARAMS_FILE))
    lv.add_argument("--tables", type=int, default=200)
    lv.add_argument("--seed", type=int, default=12345)
    lv.add_argument("--max-rows", type=float, default=1e8)
    lv.add_argument("--filter-frac", type=float, default=0.0)
    a = ap.parse_args(argv)
    if a.cmd == "collect":
        specs = sample_specs(a.tables, a.seed, max_rows=a.max_rows, filter_frac=a.filter_frac)
        d = collect(specs, log=print, budget_s=a.budget_s)
        print(f"collected {d['X'].shape[0]} tables in {float(d['seconds']):.0f} s")
        Path(a.out).parent.mkdir(parents=True, exist_ok=True)
        np.savez_compressed(a.out, **d)
        print("wrote", a.out)
    elif a.cmd == "train":
        # several datasets (comma-separated): the network trains on the training split of each
        parts = [np.load(x) for x in a.data.split(",")]
        X, T, G = [], [], []
        for d in parts:
            tr, _te = split(d["X"].shape[0])
            X.append(d["X"][tr])
            T.append(d["T"][tr])
            G.append(d["G"][tr])
        p, hist = train(np.concatenate(X), np.concatenate(T), np.concatenate(G), epochs=a.epochs, log=print)
        Path(a.out).parent.mkdir(parents=True, exist_ok=True)
        np.save(a.out, p)
        print("wrote", a.out, "final loss", hist[-1])
    elif a.cmd == "live":
        specs = sample_specs(a.tables, a.seed, max_rows=a.max_rows, filter_frac=a.filter_frac)
        print(evaluate_live(specs, np.load(a.params), log=print))
    else:
        p = np.load(a.params)
        for path in a.data.split(","):
            d = np.load(path)
            tr, te = split(d["X"].shape[0])
            out = predict(p, d["X"][te])
            print(Path(path).name, evaluate(np.argmax(out[:, :len(STRATEGIES)], axis=1), d["T"][te], d["H"][te]))


if __name__ == "__main__":
    main()
