"""Seeded synthetic inputs with the shapes of the benchmark workloads.

Every value is a pure function of (seed, stream, row index) through
splitmix64, so any row range can be generated independently and the CPU and
GPU paths see identical inputs. There is no dataset: these stand in for the
reference's h2o-style benchmark shapes.
"""

from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np

M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(x: np.ndarray) -> np.ndarray:
    """splitmix64 finaliser (Steele, Lea & Flood 2014) over a uint64 array."""
    with np.errstate(over="ignore"):
        z = x.astype(np.uint64) + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def uniform_u64(seed: int, stream: int, n: int, start: int = 0) -> np.ndarray:
    base = splitmix64(np.array([(seed * 0x100000001B3 + stream * 0x9E3779B1) & 0xFFFFFFFFFFFFFFFF],
                               dtype=np.uint64))[0]
    with np.errstate(over="ignore"):
        idx = np.arange(start, start + n, dtype=np.uint64) + base
    return splitmix64(idx)


def unit_f64(u: np.ndarray) -> np.ndarray:
    """Top 53 bits -> [0, 1)."""
    return (u >> np.uint64(11)).astype(np.float64) * (1.0 / (1 << 53))


def normal_f64(seed: int, stream: int, n: int, sigma: float, start: int = 0) -> np.ndarray:
    """Box-Muller normal N(0, sigma)."""
    u1 = unit_f64(uniform_u64(seed, stream, n, start))
    u2 = unit_f64(uniform_u64(seed, stream + 1000, n, start))
    r = np.sqrt(-2.0 * np.log1p(-u1))
    return sigma * r * np.cos(2.0 * np.pi * u2)


# ---------------------------------------------------------------------------
# Plain single-key GROUP BY: k int32 U[0,1024), v int64 U[-1e6, 1e6]
# ---------------------------------------------------------------------------
def groupby_small(n: int = 1_000_000, seed: int = 1, n_keys: int = 1024):
    k = (uniform_u64(seed, 1, n) >> np.uint64(32)) % np.uint64(n_keys)
    v = (uniform_u64(seed, 2, n) % np.uint64(2_000_001)).astype(np.int64) - 1_000_000
    return {"k": k.astype(np.int32), "v": v}


# ---------------------------------------------------------------------------
# Filtered two-key GROUP BY: (a, b) int32 pairs of Zipf(s) ranks, f < 50 filter
# ---------------------------------------------------------------------------
CHUNK = 1 << 22


def _threads() -> int:
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)


def _chunked(n: int, fn) -> None:
    """Runs fn(start, stop) over row chunks on every host thread (numpy's
    ufuncs and searchsorted release the GIL). The generators are pure
    functions of the row index, so the chunking does not change any value."""
    spans = [(s, min(n, s + CHUNK)) for s in range(0, n, CHUNK)]
    if len(spans) <= 1:
        for s, e in spans:
            fn(s, e)
        return
    with ThreadPoolExecutor(max_workers=min(_threads(), len(spans))) as pool:
        for f in [pool.submit(fn, s, e) for s, e in spans]:
            f.result()


def zipf_cdf(n_ranks: int, s: float) -> np.ndarray:
    w = np.empty(n_ranks, dtype=np.float64)

    def part(a, b):
        w[a:b] = np.arange(a + 1, b + 1, dtype=np.float64) ** (-s)

    _chunked(n_ranks, part)
    c = np.cumsum(w)
    return c / c[-1]


def zipf_ranks(cdf: np.ndarray, u: np.ndarray) -> np.ndarray:
    """Inverse-CDF Zipf ranks in [1, len(cdf)] for uniforms u in [0, 1)."""
    r = np.searchsorted(cdf, u, side="right") + 1
    return np.minimum(r, len(cdf)).astype(np.int64)


def pair_of_rank(ranks: np.ndarray, seed: int):
    with np.errstate(over="ignore"):
        h = splitmix64(ranks.astype(np.uint64) ^ np.uint64(seed * 0x2545F4914F6CDD1D & 0xFFFFFFFFFFFFFFFF))
    a = (h >> np.uint64(32)).astype(np.uint32).view(np.int32)
    b = (h & np.uint64(0xFFFFFFFF)).astype(np.uint32).view(np.int32)
    return a, b


def groupby_filtered(n: int, seed: int = 2, n_pairs: int = 10_000_000, s: float = 1.1, cdf=None,
                     ranks: np.ndarray | None = None):
    """Columns a, b (int32 keys), f (int32 U[0,100)), vd (f64 N(0,1e3)),
    vi (int64 uniform over the full range)."""
    if ranks is None:
        cdf = zipf_cdf(n_pairs, s) if cdf is None else cdf
    out = {"a": np.empty(n, np.int32), "b": np.empty(n, np.int32), "f": np.empty(n, np.int32),
           "vd": np.empty(n, np.float64), "vi": np.empty(n, np.int64)}

    def part(s0, s1):
        m = s1 - s0
        rk = ranks[s0:s1] if ranks is not None else zipf_ranks(cdf, unit_f64(uniform_u64(seed, 10, m, s0)))
        out["a"][s0:s1], out["b"][s0:s1] = pair_of_rank(rk, seed)
        out["f"][s0:s1] = ((uniform_u64(seed, 11, m, s0) >> np.uint64(32)) % np.uint64(100)).astype(np.int32)
        out["vd"][s0:s1] = normal_f64(seed, 12, m, 1e3, s0)
        out["vi"][s0:s1] = uniform_u64(seed, 14, m, s0).view(np.int64)

    _chunked(n, part)
    return out


def zipf_ranks_torch(cdf: np.ndarray, seed: int, n: int, device: str, chunk: int = 1 << 25):
    """GPU inverse-CDF sampling with the same uniforms as zipf_ranks (used
    for the large benchmark inputs; identical results to the numpy path)."""
    import torch

    c = torch.from_numpy(cdf).to(device)
    uh = np.empty(n, np.float64)

    def part(a, b):
        uh[a:b] = unit_f64(uniform_u64(seed, 10, b - a, a))

    _chunked(n, part)
    out = torch.empty(n, dtype=torch.int64)
    for s0 in range(0, n, chunk):
        m = min(chunk, n - s0)
        u = torch.from_numpy(uh[s0:s0 + m]).to(device)
        r = torch.searchsorted(c, u, right=True) + 1
        out[s0:s0 + m] = torch.clamp(r, max=len(cdf)).cpu()
    return out.numpy()


# ---------------------------------------------------------------------------
# Join then aggregate: unique shuffled int64 build keys + int32 group attr;
# probe keys 90 % matching, Decimal128(15,2) amounts
# ---------------------------------------------------------------------------
def join_build(n_build: int, seed: int = 3, n_groups: int = 100):
    k = splitmix64(np.arange(n_build, dtype=np.uint64) + np.uint64(seed << 40)).view(np.int64)
    g = ((uniform_u64(seed, 21, n_build) >> np.uint64(32)) % np.uint64(n_groups)).astype(np.int32)
    return {"k": k, "g": g}


def join_probe(n_probe: int, n_build: int, seed: int = 3, match: float = 0.9, start: int = 0):
    u = uniform_u64(seed, 22, n_probe, start)
    hit = unit_f64(uniform_u64(seed, 23, n_probe, start)) < match
    idx = (u % np.uint64(n_build)).astype(np.uint64)
    miss = np.uint64(n_build) + (u >> np.uint64(8))
    src = np.where(hit, idx, miss) + np.uint64(seed << 40)
    fk = splitmix64(src).view(np.int64)
    amt = (uniform_u64(seed, 24, n_probe, start) % np.uint64(10_000_000)).astype(np.int64)
    amount = np.stack([amt, np.zeros_like(amt)], axis=1)
    return {"fk": fk, "amount": amount}


# ---------------------------------------------------------------------------
# ORDER BY: int64 keys over the full range; float32 keys with specials
# ---------------------------------------------------------------------------
def sort_i64(n: int, seed: int = 4) -> np.ndarray:
    return uniform_u64(seed, 31, n).view(np.int64)


def sort_f32(n: int, seed: int = 5, nan_frac: float = 0.001) -> np.ndarray:
    u = uniform_u64(seed, 41, n)
    mag = 10.0 ** (unit_f64(uniform_u64(seed, 42, n)) * 60.0 - 30.0)
    sign = np.where((u & np.uint64(1)) == 1, -1.0, 1.0)
    x = (sign * mag).astype(np.float32)
    sel = unit_f64(uniform_u64(seed, 43, n))
    x[sel < 0.001] = np.float32(0.0)
    x[(sel >= 0.001) & (sel < 0.002)] = np.float32(-0.0)
    x[(sel >= 0.002) & (sel < 0.003)] = np.float32(np.inf)
    x[(sel >= 0.003) & (sel < 0.004)] = np.float32(-np.inf)
    nan_sel = (sel >= 0.5) & (sel < 0.5 + nan_frac)
    payload = ((u >> np.uint64(40)) & np.uint64(0x3FFFFF)).astype(np.uint32) | np.uint32(1)
    nan_bits = np.uint32(0x7F800000) | payload | (((u >> np.uint64(63)).astype(np.uint32)) << np.uint32(31))
    xb = x.view(np.uint32)
    xb[nan_sel] = nan_bits[nan_sel]
    return xb.view(np.float32)
