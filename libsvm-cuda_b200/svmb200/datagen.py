"""Seeded synthetic problems with the shapes of the engine's five workloads.

All feature values are float32 numbers (stored here as float64 holding the
exact float32 value) so that the device's float32 copy of X is bit-identical
to the double values the reference solver reads.  Rows are kept in CSR form
with 1-based feature indices, the libsvm convention (reference
svm-train/svm-train.c:288-389 reads "label idx:val ..." with idx >= 1).

Workloads (sizes are the defaults; every generator takes smaller sizes for
tests):
  dense_gauss      two Gaussian classes, means +-0.5, std 1, 5% flips  (n=4000, d=64)
  sparse_text      Poisson(40) nnz/row over d=20000, lognormal values,
                   rows L2-normalised, sparse-hyperplane labels, 10% flips
  dense_pixels     d=784, values k/255 with 70% zeros, tanh-teacher labels,
                   10% flips  (n=100000)
  multiclass_geo   10 classes, sizes 12000*0.8^k, d=256, centres N(0,4)
  serving_mix      a seeded stream of mixed training jobs
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional

import numpy as np


@dataclasses.dataclass
class CSR:
    """Rows of a problem: libsvm-style sparse rows in CSR arrays."""
    indptr: np.ndarray      # int64 [n+1]
    indices: np.ndarray     # int32 [nnz], 1-based, strictly ascending per row
    values: np.ndarray      # float64 [nnz], each an exact float32 value
    y: np.ndarray           # float64 [n]
    d: int                  # max feature index

    @property
    def n(self) -> int:
        return int(self.indptr.shape[0] - 1)

    @property
    def nnz(self) -> int:
        return int(self.indptr[-1])

    def take(self, rows: np.ndarray) -> "CSR":
        rows = np.asarray(rows, dtype=np.int64)
        lens = self.indptr[rows + 1] - self.indptr[rows]
        indptr = np.zeros(rows.shape[0] + 1, dtype=np.int64)
        np.cumsum(lens, out=indptr[1:])
        idx = np.concatenate([np.arange(self.indptr[r], self.indptr[r + 1]) for r in rows]) if rows.size else np.zeros(0, np.int64)
        return CSR(indptr, self.indices[idx].copy(), self.values[idx].copy(), self.y[rows].copy(), self.d)

    def to_dense(self) -> np.ndarray:
        out = np.zeros((self.n, self.d), dtype=np.float32)
        rows = np.repeat(np.arange(self.n), np.diff(self.indptr))
        out[rows, self.indices - 1] = self.values.astype(np.float32)
        return out


def from_dense(X: np.ndarray, y: np.ndarray) -> CSR:
    """Dense float32 matrix -> CSR without explicit zeros (libsvm text skips them)."""
    X = np.asarray(X, dtype=np.float32)
    n, d = X.shape
    mask = X != 0
    lens = mask.sum(axis=1)
    indptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lens, out=indptr[1:])
    r, c = np.nonzero(mask)
    return CSR(indptr, (c + 1).astype(np.int32), X[r, c].astype(np.float64),
               np.asarray(y, dtype=np.float64), d)


def write_libsvm(path: str, p: CSR) -> None:
    """libsvm text; repr() of the float64 value round-trips it exactly."""
    with open(path, "w") as f:
        for i in range(p.n):
            a, b = p.indptr[i], p.indptr[i + 1]
            lab = p.y[i]
            labs = str(int(lab)) if float(lab).is_integer() else repr(float(lab))
            feats = " ".join(f"{int(k)}:{float(v)!r}" for k, v in zip(p.indices[a:b], p.values[a:b]))
            f.write(f"{labs} {feats}\n" if feats else f"{labs}\n")


def _flip(rng, y, frac):
    m = rng.random(y.shape[0]) < frac
    y = y.copy()
    y[m] = -y[m]
    return y


def from_dense64(X: np.ndarray, y: np.ndarray) -> CSR:
    """Dense float64 matrix -> CSR keeping the full double values (rows a
    caller passes through svm.h need not be float32 numbers)."""
    X = np.asarray(X, dtype=np.float64)
    n, d = X.shape
    mask = X != 0
    indptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(mask.sum(axis=1), out=indptr[1:])
    r, c = np.nonzero(mask)
    return CSR(indptr, (c + 1).astype(np.int32), X[r, c].copy(), np.asarray(y, dtype=np.float64), d)


def dense_gauss_f64(n: int, n_test: int, d: int, seed: int, flip: float = 0.05):
    """dense_gauss with full-precision double features (not float32 numbers)."""
    rng = np.random.default_rng(seed)
    tot = n + n_test
    y = np.where(np.arange(tot) % 2 == 0, 1.0, -1.0)
    rng.shuffle(y)
    X = rng.standard_normal((tot, d)) + 0.5 * y[:, None]
    y = _flip(rng, y, flip)
    return from_dense64(X[:n], y[:n]), from_dense64(X[n:], y[n:])


def regression(n: int, n_test: int, d: int, seed: int, noise: float = 0.1):
    """Regression targets y = sin(x.w) + 0.5 (x.v)^2 / d + noise over Gaussian
    float32 features (epsilon-SVR / nu-SVR workloads)."""
    rng = np.random.default_rng(seed)
    tot = n + n_test
    X = rng.standard_normal((tot, d)).astype(np.float32)
    w = rng.standard_normal(d) / math.sqrt(d)
    v = rng.standard_normal(d)
    Xd = X.astype(np.float64)
    y = np.sin(Xd @ w) + 0.5 * (Xd @ v) ** 2 / d + noise * rng.standard_normal(tot)
    return from_dense(X[:n], y[:n]), from_dense(X[n:], y[n:])


def dense_gauss(n: int = 4000, n_test: int = 1000, d: int = 64, seed: int = 1, flip: float = 0.05):
    """Two Gaussian classes with per-dimension means +0.5 / -0.5, std 1, balanced labels."""
    rng = np.random.default_rng(seed)
    tot = n + n_test
    y = np.where(np.arange(tot) % 2 == 0, 1.0, -1.0)
    rng.shuffle(y)
    X = (rng.standard_normal((tot, d)) + 0.5 * y[:, None]).astype(np.float32)
    y = _flip(rng, y, flip)
    return from_dense(X[:n], y[:n]), from_dense(X[n:], y[n:])


def sparse_text(n: int = 50000, n_test: int = 10000, d: int = 20000, nnz_mean: float = 40.0,
                seed: int = 2, flip: float = 0.10, n_weights: int = 200):
    """Sparse high-dimensional rows: nnz ~ Poisson(nnz_mean) (>=1), uniform indices
    without replacement, lognormal(0,1) values, each row L2-normalised."""
    rng = np.random.default_rng(seed)
    tot = n + n_test
    lens = np.maximum(rng.poisson(nnz_mean, tot), 1).astype(np.int64)
    lens = np.minimum(lens, d)
    indptr = np.zeros(tot + 1, dtype=np.int64)
    np.cumsum(lens, out=indptr[1:])
    indices = np.empty(indptr[-1], dtype=np.int32)
    for i in range(tot):
        indices[indptr[i]:indptr[i + 1]] = np.sort(rng.choice(d, size=lens[i], replace=False)) + 1
    vals = rng.lognormal(0.0, 1.0, indptr[-1])
    rows = np.repeat(np.arange(tot), lens)
    norms = np.sqrt(np.bincount(rows, weights=vals * vals, minlength=tot))
    vals = (vals / norms[rows]).astype(np.float32).astype(np.float64)
    w_idx = rng.choice(d, size=min(n_weights, d), replace=False)
    w = np.zeros(d)
    w[w_idx] = rng.standard_normal(w_idx.shape[0])
    score = np.bincount(rows, weights=vals * w[indices - 1], minlength=tot)
    y = np.where(score >= 0, 1.0, -1.0)
    y = _flip(rng, y, flip)
    full = CSR(indptr, indices, vals, y, d)
    return full.take(np.arange(n)), full.take(np.arange(n, tot))


def dense_pixels(n: int = 100000, n_test: int = 20000, d: int = 784, seed: int = 3,
                 zero_frac: float = 0.70, flip: float = 0.10, hidden: int = 64):
    """Pixel-like rows: values k/255 (k uniform in 0..255) with 70% zeros; labels
    from a random 2-layer tanh teacher network."""
    rng = np.random.default_rng(seed)
    tot = n + n_test
    k = rng.integers(0, 256, size=(tot, d), dtype=np.int32)
    k[rng.random((tot, d)) < zero_frac] = 0
    X = (k.astype(np.float32) / np.float32(255.0)).astype(np.float32)
    W1 = rng.standard_normal((d, hidden)) / math.sqrt(d * 0.1)
    b1 = rng.standard_normal(hidden) * 0.1
    w2 = rng.standard_normal(hidden)
    Xc = X.astype(np.float64) - X.astype(np.float64).mean(axis=0)
    s = np.tanh(Xc @ W1 + b1) @ w2
    y = np.where(s >= np.median(s), 1.0, -1.0)
    y = _flip(rng, y, flip)
    return from_dense(X[:n], y[:n]), from_dense(X[n:], y[n:])


def multiclass_geo(n_classes: int = 10, largest: int = 12000, ratio: float = 0.8, d: int = 256,
                   seed: int = 4, n_test_frac: float = 0.0, scale: float = 1.0):
    """Classes with geometric sizes largest*ratio^k, isotropic unit-std Gaussians at
    N(0,4) centres.  Labels are 1..n_classes; rows are shuffled."""
    rng = np.random.default_rng(seed)
    sizes = [max(2, int(round(largest * scale * ratio ** k))) for k in range(n_classes)]
    centres = rng.normal(0.0, 2.0, size=(n_classes, d))
    Xs, ys = [], []
    for c, m in enumerate(sizes):
        Xs.append(centres[c] + rng.standard_normal((m, d)))
        ys.append(np.full(m, float(c + 1)))
    X = np.concatenate(Xs).astype(np.float32)
    y = np.concatenate(ys)
    perm = rng.permutation(X.shape[0])
    X, y = X[perm], y[perm]
    if n_test_frac > 0:
        nt = int(X.shape[0] * n_test_frac)
        return from_dense(X[nt:], y[nt:]), from_dense(X[:nt], y[:nt]), sizes
    return from_dense(X, y), None, sizes


@dataclasses.dataclass
class Job:
    arrival: float
    problem: CSR
    svm_type: int        # 0 C-SVC, 1 nu-SVC
    kernel_type: int     # 1 poly, 2 rbf
    C: float
    nu: float
    gamma: float
    degree: int


def serving_specs(n_jobs: int = 64, rate: float = 200.0, n_lo: int = 500, n_hi: int = 50000,
                  seed: int = 5, dims=(16, 64, 256, 512)) -> List[dict]:
    """The job stream of serving_mix without the rows: arrival time, size,
    width, data seed and kind, formulation, kernel and C of every job, drawn in
    the same order, so that serving_job(spec) rebuilds job k alone."""
    rng = np.random.default_rng(seed)
    t = 0.0
    specs = []
    for j in range(n_jobs):
        t += rng.exponential(1.0 / rate)
        n = int(round(math.exp(rng.uniform(math.log(n_lo), math.log(n_hi)))))
        d = int(rng.choice(dims))
        js = int(rng.integers(0, 2**31 - 1))
        dense = bool(rng.random() < 0.6)
        svm_type = 1 if rng.random() < 0.3 else 0
        kernel = 2 if rng.random() < 0.5 else 1
        C = float(rng.choice([1.0, 10.0]))
        specs.append(dict(arrival=t, n=n, d=d, seed=js, dense=dense, svm_type=svm_type, kernel=kernel, C=C))
    return specs


def serving_job(spec: dict) -> Job:
    """One job of the serving stream, with its rows."""
    n, d, js = spec["n"], spec["d"], spec["seed"]
    if spec["dense"]:
        p, _ = dense_gauss(n=n, n_test=0, d=d, seed=js, flip=0.05)
    else:
        p, _ = sparse_text(n=n, n_test=0, d=max(d, 64), nnz_mean=min(40.0, max(d, 64) / 2), seed=js)
    return Job(spec["arrival"], p, spec["svm_type"], spec["kernel"], spec["C"], 0.3, 1.0 / p.d, 3)


def serving_mix(n_jobs: int = 64, rate: float = 200.0, n_lo: int = 500, n_hi: int = 50000,
                seed: int = 5, dims=(16, 64, 256, 512)) -> List[Job]:
    """Poisson arrivals of mixed jobs: 60% dense Gaussian mixtures / 40% sparse CSR
    (nnz mean 40), 70% C-SVC / 30% nu-SVC (nu=0.3), RBF or degree-3 poly, C in {1,10}."""
    return [serving_job(s) for s in serving_specs(n_jobs, rate, n_lo, n_hi, seed, dims)]
