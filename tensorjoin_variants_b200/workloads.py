"""Seeded synthetic workloads for the five join configurations, and epsilon calibration.

Every generator is deterministic (NumPy ``default_rng``), so the same arrays
and thresholds are produced on any host.  The reference measured on public
embedding sets that are not available here; these generators stand in for
them with the shapes, sizes and value distributions of the five configs:

* ``uniform16``   -- plain exact self-join, N=20,000, d=16, U[0,1)^16, ~32 neighbours
* ``mixture64``   -- R-S join, 1M x 1M, d=64, 64-cluster Gaussian mixture (std 0.05), ~16 neighbours
* ``factor512``   -- R-S join, 500k x 500k, d=512, rank-32 factor model + N(0, 0.1^2), rows L2-normalised, ~8 neighbours
* ``int14x128``   -- self-join, N=2M, d=128, int14 uniform, 10% near-duplicates (+-1 jitter), ~24 neighbours
* ``ragged4096``  -- 4,096 independent R-S joins, sizes log-uniform in [256, 65536], d in {8, 32, 128}

Epsilon calibration follows the reference's sampled-pair quantile method
(tensorjoin_20260902_certified_exact_join/precision_routing_20260908_threshold_sweep/src/select_thresholds.py:15-27):
draw random non-self pairs, compute FP64 direct-difference squared distances,
and take the quantile that gives the target expected degree.  ``T = eps*eps``
in FP64 is the threshold every path compares against (``d2 <= T``).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Workload:
    name: str
    R: np.ndarray
    S: np.ndarray | None          # None for self-joins
    eps: float
    T: float | int                # threshold on squared distance (FP64, or int for int14)
    mode: str                     # "rs" | "upper" | "directed"
    screen: str                   # "plain" | "bf16" | "fp16" | "int8limb"
    target_degree: float
    meta: dict = field(default_factory=dict)

    @property
    def n_rows(self) -> int:
        return self.R.shape[0]

    @property
    def n_cols(self) -> int:
        return (self.R if self.S is None else self.S).shape[0]

    @property
    def candidate_pairs_all(self) -> int:
        """Pairs in the full pair space: |R||S| for R-S, N(N-1)/2 for self-joins."""
        if self.S is None:
            n = self.R.shape[0]
            return n * (n - 1) // 2
        return self.R.shape[0] * self.S.shape[0]


def _sample_pairs(rng, n_r, n_s, count, self_join):
    i = rng.integers(0, n_r, count, dtype=np.int64)
    if self_join:
        j = rng.integers(0, n_r - 1, count, dtype=np.int64)
        j += j >= i
    else:
        j = rng.integers(0, n_s, count, dtype=np.int64)
    return i, j


def sampled_d2(R, S, i, j, chunk=1 << 16):
    """FP64 direct-difference squared distances of sampled pairs (float inputs widened to FP64)."""
    out = np.empty(len(i), dtype=np.float64)
    for o in range(0, len(i), chunk):
        a = R[i[o:o + chunk]].astype(np.float64)
        b = S[j[o:o + chunk]].astype(np.float64)
        diff = a - b
        out[o:o + chunk] = np.einsum("ij,ij->i", diff, diff)
    return out


def calibrate_eps(R, S, degree, samples, seed, self_join):
    """eps such that a point has ~``degree`` neighbours: the (degree / n_other) quantile of sampled distances."""
    rng = np.random.default_rng(seed)
    S_ = R if S is None else S
    n_other = (R.shape[0] - 1) if self_join else S_.shape[0]
    i, j = _sample_pairs(rng, R.shape[0], S_.shape[0], samples, self_join)
    d2 = sampled_d2(R, S_, i, j)
    q = min(1.0, degree / n_other)
    eps2 = float(np.quantile(d2, q))
    eps = math.sqrt(eps2)
    return eps, eps * eps


def uniform16(n=20_000, d=16, degree=32, seed=0, samples=10_000):
    """Config 1: N=20,000, d=16, FP32 U[0,1)^d from seed 0; eps from 10,000 seeded random pairs."""
    rng = np.random.default_rng(seed)
    X = rng.random((n, d), dtype=np.float32)
    eps, T = calibrate_eps(X, None, degree, samples, seed + 1, True)
    return Workload("uniform16", X, None, eps, T, "upper", "plain", degree,
                    dict(n=n, d=d, seed=seed, calib_samples=samples))


def _mixture(rng, n, centres, std):
    k, d = centres.shape
    counts = rng.multinomial(n, np.full(k, 1.0 / k))
    labels = np.repeat(np.arange(k), counts)
    rng.shuffle(labels)
    X = centres[labels].astype(np.float32)
    X += rng.standard_normal((n, d), dtype=np.float32) * np.float32(std)
    return X


def mixture64(n=1_000_000, d=64, clusters=64, std=0.05, degree=16, seed=2, samples=1 << 22,
              screen="bf16"):
    """Config 2: R-S, |R|=|S|=n, d=64 Gaussian mixture of 64 clusters (centres U[0,1)^d, std 0.05)."""
    rng = np.random.default_rng(seed)
    centres = rng.random((clusters, d))
    R = _mixture(rng, n, centres, std)
    S = _mixture(rng, n, centres, std)
    eps, T = calibrate_eps(R, S, degree, samples, seed + 1, False)
    return Workload("mixture64", R, S, eps, T, "rs", screen, degree,
                    dict(n=n, d=d, clusters=clusters, std=std, seed=seed, calib_samples=samples))


def _factor_rows(rng, n, W, noise):
    r, d = W.shape
    out = np.empty((n, d), dtype=np.float32)
    step = 1 << 16
    for o in range(0, n, step):
        m = min(step, n - o)
        f = rng.standard_normal((m, r), dtype=np.float32)
        x = f @ W
        x += rng.standard_normal((m, d), dtype=np.float32) * np.float32(noise)
        x /= np.linalg.norm(x.astype(np.float64), axis=1, keepdims=True).astype(np.float32)
        out[o:o + m] = x
    return out


def factor512(n=500_000, d=512, rank=32, noise=0.1, degree=8, seed=3, samples=1 << 22, screen="fp16"):
    """Config 3: R-S, n x n, d=512 rank-32 factor model (loadings N(0,1/32)) + N(0,0.1^2), rows L2-normalised."""
    rng = np.random.default_rng(seed)
    W = (rng.standard_normal((rank, d)) / math.sqrt(rank)).astype(np.float32)
    R = _factor_rows(rng, n, W, noise)
    S = _factor_rows(rng, n, W, noise)
    eps, T = calibrate_eps(R, S, degree, samples, seed + 1, False)
    return Workload("factor512", R, S, eps, T, "rs", screen, degree,
                    dict(n=n, d=d, rank=rank, noise=noise, seed=seed, calib_samples=samples))


def int14x128(n=2_000_000, d=128, dup_frac=0.10, degree=24, seed=4, samples=1 << 22):
    """Config 4: self-join, n x 128 int14 U{-8192..8191}; 10% of rows are copies of other rows with +-1 jitter."""
    rng = np.random.default_rng(seed)
    X = rng.integers(-8192, 8192, size=(n, d), dtype=np.int16)
    ndup = int(round(dup_frac * n))
    dst = rng.choice(n, size=ndup, replace=False)
    src = rng.integers(0, n, size=ndup)
    jitter = rng.integers(-1, 2, size=(ndup, d)).astype(np.int16)
    X[dst] = np.clip(X[src].astype(np.int32) + jitter, -8192, 8191).astype(np.int16)
    # integer eps^2 from the sampled exact integer distances
    rs = np.random.default_rng(seed + 1)
    i, j = _sample_pairs(rs, n, n, samples, True)
    d2 = np.empty(samples, dtype=np.int64)
    for o in range(0, samples, 1 << 16):
        diff = X[i[o:o + (1 << 16)]].astype(np.int64) - X[j[o:o + (1 << 16)]].astype(np.int64)
        d2[o:o + (1 << 16)] = np.einsum("ij,ij->i", diff, diff)
    q = min(1.0, degree / (n - 1))
    T = int(np.quantile(d2, q, method="lower"))
    return Workload("int14x128", X, None, math.sqrt(T), T, "upper", "int8limb", degree,
                    dict(n=n, d=d, dup_frac=dup_frac, seed=seed, calib_samples=samples))


@dataclass
class RaggedJoin:
    R: np.ndarray
    S: np.ndarray
    eps: float
    T: float


def ragged_eps2(n_s, d, clusters, std, degree):
    """Per-join threshold for ~``degree`` neighbours in a well-separated mixture.

    Within one cluster the squared distance of two points is 2 std^2 chi2_d, and a
    point sees about n_s / clusters same-cluster partners, so
    T = 2 std^2 * chi2_d.ppf(degree * clusters / n_s).  Analytic (seeded sampling
    of 4,096 joins would dominate set-up time); the realised degree is reported.
    """
    from scipy.stats import chi2

    q = min(0.999, degree * clusters / n_s)
    return float(2.0 * std * std * chi2.ppf(q, d))


def ragged4096(joins=4096, lo=256, hi=65536, dims=(8, 32, 128), clusters=8, std=0.05, degree=16, seed=5,
               size_scale=1.0):
    """Config 5: thousands of independent R-S joins with log-uniform sizes and d drawn from ``dims``.

    Each join is an 8-cluster mixture (centres U[0,1)^d, isotropic std 0.05) on both sides.  Data are
    drawn per dimension class in bulk and every join's R and S are contiguous slices of its class
    arrays (``RaggedJoin.R`` / ``.S`` are views), so the whole batch also exists as a few large arrays
    (``ragged_classes``) that can be moved to the device in one copy per class.
    """
    rng = np.random.default_rng(seed)
    nr = np.maximum(1, np.round(np.exp(rng.uniform(math.log(lo), math.log(hi), joins)) * size_scale)).astype(np.int64)
    ns = np.maximum(1, np.round(np.exp(rng.uniform(math.log(lo), math.log(hi), joins)) * size_scale)).astype(np.int64)
    dj = rng.choice(np.asarray(dims), joins)
    out = [None] * joins
    for d in dims:
        ks = np.flatnonzero(dj == d)
        if len(ks) == 0:
            continue
        centres = rng.random((len(ks), clusters, d)).astype(np.float32)
        for side, counts in (("R", nr[ks]), ("S", ns[ks])):
            total = int(counts.sum())
            owner = np.repeat(np.arange(len(ks)), counts)
            label = rng.integers(0, clusters, total)
            X = rng.standard_normal((total, d), dtype=np.float32)
            X *= np.float32(std)
            X += centres[owner, label]
            offs = np.concatenate([[0], np.cumsum(counts)])
            for q, k in enumerate(ks):
                part = X[offs[q]:offs[q + 1]]
                if out[k] is None:
                    out[k] = {}
                out[k][side] = part
    res = []
    for k in range(joins):
        T = ragged_eps2(int(ns[k]), int(dj[k]), clusters, std, degree)
        res.append(RaggedJoin(out[k]["R"], out[k]["S"], math.sqrt(T), T))
    return res


CONFIGS = {
    "uniform16": uniform16,
    "mixture64": mixture64,
    "factor512": factor512,
    "int14x128": int14x128,
    "ragged4096": ragged4096,
}


def ragged4096_device(joins=4096, lo=256, hi=65536, dims=(8, 32, 128), clusters=8, std=0.05, degree=16, seed=5,
                      size_scale=1.0):
    """Config 5 drawn on the GPU (seeded torch CUDA generator): the shapes and distributions of
    ``ragged4096``, one bulk draw per dimension class and side, every join a contiguous slice (views).
    Returns ``([(R, S, eps), ...], class_arrays)`` with device tensors."""
    import torch

    rng = np.random.default_rng(seed)
    nr = np.maximum(1, np.round(np.exp(rng.uniform(math.log(lo), math.log(hi), joins)) * size_scale)).astype(np.int64)
    ns = np.maximum(1, np.round(np.exp(rng.uniform(math.log(lo), math.log(hi), joins)) * size_scale)).astype(np.int64)
    dj = rng.choice(np.asarray(dims), joins)
    g = torch.Generator(device="cuda").manual_seed(seed)
    out = [dict() for _ in range(joins)]
    classes = []
    for d in dims:
        ks = np.flatnonzero(dj == d)
        if len(ks) == 0:
            continue
        centres = torch.from_numpy(rng.random((len(ks), clusters, d)).astype(np.float32)).cuda()
        for side, counts in (("R", nr[ks]), ("S", ns[ks])):
            total = int(counts.sum())
            owner = torch.from_numpy(np.repeat(np.arange(len(ks)), counts)).cuda()
            label = torch.randint(0, clusters, (total,), generator=g, device="cuda")
            X = torch.randn((total, d), generator=g, device="cuda") * std + centres[owner, label]
            classes.append(X)
            offs = np.concatenate([[0], np.cumsum(counts)])
            for q, k in enumerate(ks):
                out[k][side] = X[int(offs[q]):int(offs[q + 1])]
    eps = [math.sqrt(ragged_eps2(int(ns[k]), int(dj[k]), clusters, std, degree)) for k in range(joins)]
    return [(out[k]["R"], out[k]["S"], eps[k]) for k in range(joins)], classes
