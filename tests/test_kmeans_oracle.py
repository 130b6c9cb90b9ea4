"""CPU checks of the k-means initialisation oracle (the restatement of the engine's
seeded k-means that the GPU tests compare against)."""

import numpy as np

from oracle import kmeans_oracle as ko
from rapids_singlecell_b200.synthetic import MixtureSpec, make_mixture


def _data(n=3000, d=20, seed=1):
    Z, _, _ = make_mixture(MixtureSpec(n, d, 6, 3, "given", (0.5, 0.3, 0.2), 0.5), seed)
    return Z


def test_draws_are_a_function_of_seed_and_counter():
    assert ko.draw(7, 3) == ko.draw(7, 3)
    assert ko.draw(7, 3) != ko.draw(8, 3) and ko.draw(7, 3) != ko.draw(7, 4)
    u = [ko.u01(ko.draw(1, i)) for i in range(2000)]
    assert 0.0 <= min(u) and max(u) < 1.0 and abs(np.mean(u) - 0.5) < 0.03


def test_seeds_are_distinct_normalised_sample_rows():
    Z = _data()
    Y = ko.seed_centres(Z, 40, 5)
    Zn = ko.normalise_rows(Z).astype(np.float32)
    for y in Y:  # every centre is a normalised input row
        assert np.min(np.abs(Zn - y).max(axis=1)) == 0.0
    assert len({tuple(y) for y in Y}) == 40
    assert np.array_equal(Y, ko.seed_centres(Z, 40, 5))
    assert not np.array_equal(Y, ko.seed_centres(Z, 40, 6))


def test_seeding_samples_with_replacement_beyond_the_sample_size():
    Z = _data(n=5000, d=8)
    assert ko.sample_size(5000, 10) == 640
    Y = ko.seed_centres(Z, 10, 3)
    assert Y.shape == (10, 8) and np.isfinite(Y).all()


def test_lloyd_lowers_the_inertia_of_the_seeds():
    Z = _data()
    Y0 = ko.seed_centres(Z, 30, 2)
    Y, it = ko.lloyd(Z, Y0, 25, 1e-4)
    assert 1 <= it <= 25
    assert ko.inertia(Z, Y) < ko.inertia(Z, Y0)
