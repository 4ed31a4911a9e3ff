"""Seeded synthetic inputs for the benchmark workloads (no public dataset is used).

All arrays are FP64.  Each array has its own PCG64 stream:
    1001 source points, 1002 target points, 1003 a / A, 1004 b,
    1005 barycentric weights w, 1006 b_ext / document data.
Histograms are Dirichlet(alpha) draws (normalised Gamma(alpha, 1)).  Costs are
squared Euclidean distances summed over coordinates in ascending order, then
divided by their maximum.  Matrices are returned column-major (Fortran order).
"""
from __future__ import annotations

import numpy as np

SEED_X, SEED_Y, SEED_A, SEED_B, SEED_W, SEED_DOC = 1001, 1002, 1003, 1004, 1005, 1006


def rng(seed: int, salt: int = 0) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64([seed, salt]))


def dirichlet(g: np.random.Generator, alpha: float, n: int, cols: int | None = None) -> np.ndarray:
    shape = (n,) if cols is None else (n, cols)
    x = g.gamma(alpha, 1.0, size=shape)
    return np.asfortranarray(x / x.sum(axis=0, keepdims=True))


def sq_euclid_cost(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """C_ij = sum_k (x_ik - y_jk)^2 accumulated in ascending k, divided by max C."""
    C = np.zeros((x.shape[0], y.shape[0]), order="F")
    for k in range(x.shape[1]):
        d = x[:, k, None] - y[None, :, k]
        C += d * d
    C /= C.max()
    return C


def sinkhorn_problem(m: int, n: int, alpha: float, dim: int = 2, salt: int = 0):
    """Histograms a (m), b (n) ~ Dirichlet(alpha); points uniform in [0,1]^dim."""
    x = rng(SEED_X, salt).random((m, dim))
    y = rng(SEED_Y, salt).random((n, dim))
    a = dirichlet(rng(SEED_A, salt), alpha, m)
    b = dirichlet(rng(SEED_B, salt), alpha, n)
    return a, b, sq_euclid_cost(x, y)


def vanilla_config(m=256, n=256):
    """Plain vanilla Sinkhorn: Dirichlet(1) histograms, uniform points in [0,1]^2."""
    return sinkhorn_problem(m, n, 1.0, 2)


def log_config(m=4096, n=4096):
    """Plain log Sinkhorn: Dirichlet(0.5) histograms, uniform points in [0,1]^2."""
    return sinkhorn_problem(m, n, 0.5, 2)


def barycenter_config(n=2048, S=32, dim=50, salt: int = 0):
    """Log barycenter: n support points ~ N(0, I_dim), S Dirichlet(0.3) histograms,
    w ~ Dirichlet(1), b_ext ~ Dirichlet(0.3)."""
    x = rng(SEED_X, salt).standard_normal((n, dim))
    C = sq_euclid_cost(x, x)
    A = dirichlet(rng(SEED_A, salt), 0.3, n, S)
    w = dirichlet(rng(SEED_W, salt), 1.0, S)
    b_ext = dirichlet(rng(SEED_DOC, salt), 0.3, n)
    return A, C, w, b_ext


def wdl_config(V=5000, M=2048, S=16, dim=64, salt: int = 0):
    """WDL corpus: V embeddings ~ N(0, I_dim) with squared-Euclidean cost / max;
    M documents of U{20..200} tokens whose ids follow Zipf(1.1) truncated to V
    (redrawn until in range), as normalised count columns (V x M); initial
    logits Alpha0 (V x S), Lambda0 (S x M) ~ N(0, 0.01) (variance 0.01,
    standard deviation 0.1)."""
    x = rng(SEED_X, salt).standard_normal((V, dim))
    C = sq_euclid_cost(x, x)
    g = rng(SEED_DOC, salt)
    Y = np.zeros((V, M), order="F")
    lengths = g.integers(20, 201, size=M)
    for m in range(M):
        ids = np.empty(0, dtype=np.int64)
        while ids.size < lengths[m]:
            z = g.zipf(1.1, size=2 * int(lengths[m]))
            ids = np.concatenate([ids, z[z <= V] - 1])
        np.add.at(Y[:, m], ids[:lengths[m]], 1.0)
        Y[:, m] /= Y[:, m].sum()
    gl = rng(SEED_W, salt)
    Alpha0 = np.asfortranarray(0.1 * gl.standard_normal((V, S)))
    Lambda0 = np.asfortranarray(0.1 * gl.standard_normal((S, M)))
    return Y, C, Alpha0, Lambda0


SEED_STREAM = 1007


def stream_requests(R=200, salt: int = 0):
    """Mixed-size log-Sinkhorn request stream: n and m independently
    log-uniform in [64, 8192] (rounded), eps uniform from {0.01, 0.05, 0.1},
    point dimension d uniform from {2, 3, 64}; unit-rate exponential
    inter-arrival gaps (Poisson arrivals, scaled by the caller).  Returns a
    list of dicts (m, n, eps, d, salt, gap); request i's data come from
    stream_request_data(m, n, d, salt)."""
    g = rng(SEED_STREAM, salt)
    lo, hi = np.log(64.0), np.log(8192.0)
    ms = np.clip(np.rint(np.exp(g.uniform(lo, hi, R))), 64, 8192).astype(int)
    ns = np.clip(np.rint(np.exp(g.uniform(lo, hi, R))), 64, 8192).astype(int)
    eps = g.choice([0.01, 0.05, 0.1], size=R)
    dims = g.choice([2, 3, 64], size=R)
    gaps = g.exponential(1.0, size=R)
    return [{"m": int(ms[i]), "n": int(ns[i]), "eps": float(eps[i]), "d": int(dims[i]), "salt": 10000 * salt + i,
             "gap": float(gaps[i])} for i in range(R)]


def stream_request_data(m, n, d, salt):
    """Histograms a (m), b (n) ~ Dirichlet(1) and points x (m x d), y (n x d)
    uniform in [0,1]^d; the cost is sq_euclid_cost(x, y)."""
    x = rng(SEED_X, salt).random((m, d))
    y = rng(SEED_Y, salt).random((n, d))
    a = dirichlet(rng(SEED_A, salt), 1.0, m)
    b = dirichlet(rng(SEED_B, salt), 1.0, n)
    return a, b, x, y
