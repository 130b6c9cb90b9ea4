"""Writes the golden fixtures ``tests/golden/ref_*.npz`` from the reference itself.

Each case runs rapids_singlecell's Harmony with the reference's own CUDA kernels
(``oracle/ref_harmony.py`` driving ``oracle/_ref/libharmony_ref.so``, compiled from the
reference tree by ``oracle/Makefile``) on a GPU, with injected initial centroids, and
stores the inputs, the parameters and the outputs.  ``tests/test_oracle_vs_reference.py``
then checks the NumPy oracle against these outputs on any machine (no GPU).

    make -C oracle && python tests/golden/make_ref_golden.py [--out DIR]

Inputs are seeded draws of the repository's mixture generator at small sizes, so the
fixtures stay small (about 2 MB together).  The PCA cases (``ref_pca_*.npz``) run the
reference's covariance PCA kernels on a seeded sparse matrix (``oracle/ref_pca.py``).
"""

from __future__ import annotations

import argparse
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from rapids_singlecell_b200.synthetic import MixtureSpec, initial_centroids, make_mixture  # noqa: E402

# name -> (mixture, K, centroid seed, run parameters, dtype, keep R/O/E)
CASES = {
    # reference defaults (harmony2), default tolerances: early stops of both loops are exercised
    "h2_f64": (MixtureSpec(2000, 16, 6, 3, "given", (0.5, 0.3, 0.2), 0.5), 20, 1,
               dict(max_iter_harmony=4, max_iter_clustering=15), "float64", False),
    "h2_f32": (MixtureSpec(2000, 16, 6, 3, "given", (0.5, 0.3, 0.2), 0.5), 20, 1,
               dict(max_iter_harmony=4, max_iter_clustering=15), "float32", False),
    # harmony1 flavour (plain penalty, fixed ridge lambda, no pruning), theta per batch, tau
    # discount, one batch of only 9 cells
    "h1_tau_f64": (MixtureSpec(1800, 12, 5, 4, "given", (0.5, 0.3, 0.195, 0.005), 0.6), 16, 2,
                   dict(max_iter_harmony=3, max_iter_clustering=10, stabilized_penalty=False,
                        dynamic_lambda=False, batch_prune_threshold=None, ridge_lambda=1.0,
                        theta=[1.0, 2.0, 0.5, 3.0], tau=5), "float64", False),
    # one outer x two k-means iterations at fixed counts, with the state R, O, E: the
    # component-level pin of the clustering loop
    "k2_state_f64": (MixtureSpec(2400, 24, 8, 5, "dirichlet", (), 0.5, (0.8, 1.2)), 30, 3,
                     dict(max_iter_harmony=1, max_iter_clustering=2, tol_clustering=float("-inf"),
                          tol_harmony=float("-inf"), block_proportion=0.1, random_state=7),
                     "float64", True),
}


def pca_input(seed=5, n=3000, g=240, rank=8):
    """A sparse, log-normalised-looking cells x genes matrix with a low-rank structure: Poisson
    counts of a rank-`rank` factor model at low depth (about a quarter of the entries nonzero),
    log1p; every gene expressed in at least one cell."""
    import scipy.sparse as sp

    rng = np.random.default_rng(seed)
    F = rng.gamma(2.0, 1.0, (n, rank))
    L = rng.gamma(0.6, 1.0, (rank, g)) * rng.uniform(0.2, 3.0, g)
    lam = F @ L / rank
    counts = rng.poisson(lam * rng.uniform(0.05, 0.3, (n, 1)))
    counts[rng.integers(0, n, g), np.arange(g)] += 1  # no all-zero gene
    X = sp.csr_matrix(np.log1p(counts).astype(np.float32))
    X.sort_indices()
    return X


PCA_CASES = {"pca_center": dict(zero_center=True, n_comps=20), "pca_gram": dict(zero_center=False, n_comps=12)}


def run_pca_case(name, out_dir: Path) -> Path:
    from oracle import ref_pca

    X = pca_input()
    kw = PCA_CASES[name]
    X_pca, comps, var, ratio, mean = ref_pca.pca_csr(X.indptr, X.indices, X.data, X.shape, kw["n_comps"],
                                                      zero_center=kw["zero_center"])
    arrays = dict(indptr=X.indptr.astype(np.int64), indices=X.indices.astype(np.int32), data=X.data,
                  shape=np.asarray(X.shape), params=np.array(json.dumps(kw)), X_pca=X_pca, components=comps,
                  variance=var, variance_ratio=ratio)
    if mean is not None:
        arrays["mean"] = mean
    path = out_dir / f"ref_{name}.npz"
    np.savez_compressed(path, **arrays)
    return path


def run_case(name, out_dir: Path) -> Path:
    from oracle import ref_harmony as rh

    spec, K, cseed, params, dtype, keep_state = CASES[name]
    Z, cats, _ = make_mixture(spec, seed=17)
    Y0 = initial_centroids(Z, K, cseed)
    res = rh.harmonize(Z, cats, spec.n_batches, Y0, n_clusters=K, dtype=np.dtype(dtype), **params)
    km = res.kmeans_objectives
    arrays = dict(
        Z=Z, cats=cats, Y0=Y0,
        params=np.array(json.dumps(dict(params, n_clusters=K, n_batches=spec.n_batches, dtype=dtype))),
        Z_hat=res.Z_hat,
        objectives=np.asarray(res.objectives_harmony, dtype=np.float64),
        kmeans_objectives=np.asarray([v for row in km for v in row], dtype=np.float64),
        kmeans_iters=np.asarray([len(row) for row in km], dtype=np.int32),
        converged=np.asarray(res.converged),
        n_outer=np.asarray(res.n_outer),
    )
    if keep_state:
        arrays.update(R=res.R, O=res.O, E=res.E)
    path = out_dir / f"ref_{name}.npz"
    np.savez_compressed(path, **arrays)
    return path


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--out", default=str(Path(__file__).resolve().parent))
    ap.add_argument("--cases", nargs="*", default=list(CASES) + list(PCA_CASES))
    args = ap.parse_args()
    out = Path(args.out)
    out.mkdir(parents=True, exist_ok=True)
    for name in args.cases:
        if name in PCA_CASES:
            path = run_pca_case(name, out)
            with np.load(path) as f:
                print(f"{path.name}: variance={np.round(f['variance'][:6], 4).tolist()}")
            continue
        path = run_case(name, out)
        with np.load(path) as f:
            print(f"{path.name}: n_outer={int(f['n_outer'])} kmeans_iters={f['kmeans_iters'].tolist()} "
                  f"objectives={np.round(f['objectives'], 6).tolist()}")


if __name__ == "__main__":
    main()
