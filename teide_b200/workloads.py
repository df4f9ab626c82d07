"""Seeded synthetic inputs with the shapes of the benchmark workloads.

No public dataset backs these workloads (the H2O.ai db-benchmark data and the
external teide-bench scripts are not available), so every column is drawn
from a seeded generator with the stated distribution.  Generators return
numpy arrays; `device="cuda"` draws on the GPU with torch for the large
configurations and copies to host memory (the values then differ from the
numpy draws of the same seed, but every consumer -- kernel and checker --
reads the same arrays).
"""
from __future__ import annotations

import math

import numpy as np

ZIPF_S = 1.1
ZIPF_N = 1 << 24
# rank r (0 = most frequent) maps to key (r * ZIPF_MULT) mod 2^24: a bijection
# that scatters the hot keys over the whole key range.
ZIPF_MULT = 0x9E3779 | 1


def _zipf_cdf(n=ZIPF_N, s=ZIPF_S):
    w = np.arange(1, n + 1, dtype=np.float64) ** (-s)
    c = np.cumsum(w)
    return c / c[-1]


def readme_table(n=10_000_000, seed=1):
    """README pipeline: flag U{0..3}, region U[0,64), amount U[0,1000)."""
    r = np.random.default_rng(seed)
    return {
        "flag": r.integers(0, 4, n, dtype=np.int64),
        "region": r.integers(0, 64, n, dtype=np.int64),
        "amount": r.random(n) * 1000.0,
    }


def zipf_group_table(n=200_000_000, seed=2, device=None, nkeys=ZIPF_N):
    """Radix group-by: key Zipf(1.1) over `nkeys` values, v1 U[-1e6,1e6],
    v2 N(0,1)."""
    if device is not None:
        import torch
        g = torch.Generator(device=device).manual_seed(seed)
        w = torch.arange(1, nkeys + 1, dtype=torch.float64, device=device).pow(-ZIPF_S)
        cdf = torch.cumsum(w, 0)
        cdf /= cdf[-1].clone()
        out = {}
        keys = torch.empty(n, dtype=torch.int64, device=device)
        step = 1 << 26
        for i in range(0, n, step):
            m = min(step, n - i)
            u = torch.rand(m, dtype=torch.float64, device=device, generator=g)
            rank = torch.searchsorted(cdf, u).clamp_(max=nkeys - 1)
            keys[i:i + m] = (rank * ZIPF_MULT) % nkeys
        out["key"] = keys.cpu().numpy()
        del keys
        out["v1"] = torch.randint(-1_000_000, 1_000_001, (n,), dtype=torch.int64, device=device,
                                  generator=g).cpu().numpy()
        out["v2"] = torch.randn(n, dtype=torch.float64, device=device, generator=g).cpu().numpy()
        return out
    r = np.random.default_rng(seed)
    cdf = _zipf_cdf(nkeys)
    rank = np.minimum(np.searchsorted(cdf, r.random(n)), nkeys - 1).astype(np.int64)
    return {
        "key": (rank * ZIPF_MULT) % nkeys,
        "v1": r.integers(-1_000_000, 1_000_001, n, dtype=np.int64),
        "v2": r.standard_normal(n),
    }


def join_tables(n_build=10_000_000, n_probe=100_000_000, seed=3, device=None):
    """Filter -> join -> group: build pk = permutation of [0,n_build),
    cat U[0,1000); probe fk U[0, 1.2 n_build), qty U[1,100], price U[1,500)."""
    fk_hi = int(round(n_build * 1.2))
    if device is not None:
        import torch
        g = torch.Generator(device=device).manual_seed(seed)
        build = {
            "pk": torch.randperm(n_build, device=device, generator=g).to(torch.int64).cpu().numpy(),
            "cat": torch.randint(0, 1000, (n_build,), dtype=torch.int64, device=device,
                                 generator=g).cpu().numpy(),
        }
        probe = {
            "fk": torch.randint(0, fk_hi, (n_probe,), dtype=torch.int64, device=device,
                                generator=g).cpu().numpy(),
            "qty": torch.randint(1, 101, (n_probe,), dtype=torch.int64, device=device,
                                 generator=g).cpu().numpy(),
            "price": (torch.rand(n_probe, dtype=torch.float64, device=device, generator=g)
                      * 499.0 + 1.0).cpu().numpy(),
        }
        return build, probe
    r = np.random.default_rng(seed)
    build = {
        "pk": r.permutation(n_build).astype(np.int64),
        "cat": r.integers(0, 1000, n_build, dtype=np.int64),
    }
    probe = {
        "fk": r.integers(0, fk_hi, n_probe, dtype=np.int64),
        "qty": r.integers(1, 101, n_probe, dtype=np.int64),
        "price": r.random(n_probe) * 499.0 + 1.0,
    }
    return build, probe


def batch_shapes(n_queries=4096, seed=4, rows=(1_000, 2_000_000), groups=(16, 65_536)):
    """Per-query (rows, K): both log-uniform."""
    r = np.random.default_rng(seed)
    lr = r.uniform(math.log(rows[0]), math.log(rows[1]), n_queries)
    lk = r.uniform(math.log(groups[0]), math.log(groups[1]), n_queries)
    return np.exp(lr).astype(np.int64), np.exp(lk).astype(np.int64)


def batch_query(rows, k, seed):
    """One batched query's table: key U[0,K), val U[0,1)."""
    r = np.random.default_rng(seed)
    return {"key": r.integers(0, k, rows, dtype=np.int64), "val": r.random(rows)}


def serve_requests(n, rate=2000.0, seed=5, group_rows=200_000_000, probe_rows=100_000_000,
                     join_frac=0.3, len_range=(100_000, 50_000_000)):
    """The served mix: n requests with Poisson arrivals at `rate` per second.
    70% filter + group-by over the group table (v1 > t, t ~ U[-1e6, 1e6]),
    30% filter + join + group-by over the probe table (qty > t, t ~ U{1..100});
    each reads a contiguous row range [off, off + len) with len ~ U[100K, 50M]
    (clipped to the table) and off uniform over the valid starts.
    Returns a list of (kind, off, len, threshold, arrival_seconds)."""
    r = np.random.default_rng(seed)
    arrivals = np.cumsum(r.exponential(1.0 / rate, n))
    out = []
    for i in range(n):
        join = r.random() < join_frac
        rows = probe_rows if join else group_rows
        ln = int(min(r.integers(len_range[0], len_range[1] + 1), rows))
        off = int(r.integers(0, rows - ln + 1))
        t = int(r.integers(1, 101)) if join else int(r.integers(-1_000_000, 1_000_001))
        out.append(("join" if join else "group", off, ln, t, float(arrivals[i])))
    return out
