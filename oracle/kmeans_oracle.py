"""CPU oracle for the engine's k-means centroid initialisation -- TEST INFRASTRUCTURE ONLY.

Only ``tests/`` may import this module; the shipped engine never calls it.

The reference fits cuML ``KMeans(init="k-means||", n_init=1, max_iter=25,
random_state)`` on the L2-normalised embedding and L2-normalises the centres
(src/rapids_singlecell/preprocessing/_harmony/__init__.py:290-323).  cuML is a
third-party dependency (cuml-cu12/13>=25.10, pyproject.toml) that is not in the
reference tree, and its random streams cannot be reproduced, so this oracle does
not restate cuML: it restates the engine's own seeded k-means (``hb_kmeans_init``,
``rapids_singlecell_b200/csrc/hb_kmeans.cu``), which plays the same role.  Its
parity against cuML is unpinned; its parity against the engine is:

* seeding, bit for bit: k-means++ (Arthur & Vassilvitskii, 2007) over a sample of
  m = min(n, 64 K, 16384) cells, draws from splitmix64 (Steele, Lea & Flood, 2014)
  of (seed, counter), float64 with the same operation order as the device code
  (sequential sums over columns, over each of 1024 contiguous chunks of the sample,
  and over the chunks);
* Lloyd iterations, within tolerance: float64 assignment to the nearest centre
  (the device uses bf16 operands on the tensor core, so cells near a tie may move
  differently) and float64 means; empty centres keep their position; stop when
  |Y_new - Y_old|_F <= tol |Y_new|_F.
"""

from __future__ import annotations

import numpy as np

M64 = (1 << 64) - 1
SAMPLE_BASE = 1 << 40
SEED_THREADS = 1024


def splitmix64(x: int) -> int:
    x = (x + 0x9E3779B97F4A7C15) & M64
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & M64
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & M64
    return x ^ (x >> 31)


def draw(seed: int, ctr: int) -> int:
    return splitmix64(splitmix64(seed & M64) ^ ctr)


def u01(h: int) -> float:
    return float(h >> 11) * (1.0 / 9007199254740992.0)


def sample_size(n: int, K: int) -> int:
    return min(n, min(64 * K, 16384))


def seed_centres(X: np.ndarray, K: int, seed: int) -> np.ndarray:
    """k-means++ seeding as the device performs it; returns float32 [K, d] centres."""
    X = np.asarray(X, dtype=np.float32)
    n, d = X.shape
    m = sample_size(n, K)
    if m == n:
        cells = np.arange(n)
    else:
        cells = np.array([draw(seed, SAMPLE_BASE + j) % n for j in range(m)], dtype=np.int64)
    x = X[cells].astype(np.float64)
    ss = np.zeros(m)
    for c in range(d):
        ss = ss + x[:, c] * x[:, c]
    inv = 1.0 / np.sqrt(ss)
    inv = np.where(inv <= 1e12, inv, 1e12)
    S = x * inv[:, None]
    ch = (m + SEED_THREADS - 1) // SEED_THREADS
    bounds = [(min(m, t * ch), min(m, (t + 1) * ch)) for t in range(SEED_THREADS)]
    Y = np.zeros((K, d), dtype=np.float32)
    pick = draw(seed, 0) % m
    D2 = np.zeros(m)
    for r in range(K):
        cen = S[pick]
        Y[r] = cen.astype(np.float32)
        if r == K - 1:
            break
        acc = np.zeros(m)
        for c in range(d):
            df = S[:, c] - cen[c]
            acc = acc + df * df
        D2 = acc if r == 0 else np.minimum(D2, acc)
        local = np.zeros(SEED_THREADS)
        for t, (j0, j1) in enumerate(bounds):
            s = 0.0
            for v in D2[j0:j1]:
                s = s + v
            local[t] = s
        part = np.zeros(SEED_THREADS)
        run = 0.0
        for t in range(SEED_THREADS):
            part[t] = run
            run = run + local[t]
        total = run
        h = draw(seed, 1 + (r + 1))
        if not total > 0.0:
            pick = h % m
            continue
        target = u01(h) * total
        pick = -1
        for t, (j0, j1) in enumerate(bounds):
            lo = part[t]
            hi = part[t + 1] if t + 1 < SEED_THREADS else total
            if lo <= target < hi:
                a, got, last = lo, -1, -1
                for j in range(j0, j1):
                    if D2[j] > 0.0:
                        last = j
                    a = a + D2[j]
                    if target < a:
                        got = j
                        break
                pick = got if got >= 0 else last
                break
        if pick < 0:
            nz = np.nonzero(D2 > 0.0)[0]
            pick = int(nz[-1]) if nz.size else 0
    return Y


def normalise_rows(X: np.ndarray) -> np.ndarray:
    X = np.asarray(X, dtype=np.float64)
    inv = 1.0 / np.sqrt((X * X).sum(axis=1))
    return X * np.minimum(inv, 1e12)[:, None]


def lloyd(X: np.ndarray, Y0: np.ndarray, max_iter: int, tol: float):
    """Float64 Lloyd iterations on the normalised rows from centres Y0; returns (Y, iterations)."""
    Z = normalise_rows(X)
    Y = np.asarray(Y0, dtype=np.float64).copy()
    K = Y.shape[0]
    it = 0
    for _ in range(max_iter):
        lab = np.argmax(Z @ Y.T - 0.5 * (Y * Y).sum(axis=1)[None, :], axis=1)
        cnt = np.bincount(lab, minlength=K).astype(np.float64)
        sums = np.zeros_like(Y)
        np.add.at(sums, lab, Z)
        Ynew = np.where(cnt[:, None] > 0, sums / np.maximum(cnt, 1.0)[:, None], Y)
        shift = ((Ynew - Y) ** 2).sum()
        Y = Ynew
        it += 1
        if shift <= tol * tol * (Y * Y).sum():
            break
    return Y.astype(np.float32), it


def inertia(X: np.ndarray, Y: np.ndarray) -> float:
    """Sum over cells of the squared distance of the normalised row to its nearest centre."""
    Z = normalise_rows(X)
    Y = np.asarray(Y, dtype=np.float64)
    d2 = 1.0 - 2.0 * Z @ Y.T + (Y * Y).sum(axis=1)[None, :]
    return float(np.maximum(d2.min(axis=1), 0.0).sum())


def kmeans_init(X: np.ndarray, K: int, seed: int, max_iter: int = 25, tol: float = 1e-4):
    Y0 = seed_centres(X, K, seed)
    return lloyd(X, Y0, max_iter, tol)
