"""CPU: the mutation-site sampler of the product's draw layout (tests/draws.py,
restated from the oracle's Philox stream) gives every variable an
independent mutation chance of limit = pm_prob / D, like the per-variable test
of the reference (polynomial_mutation.cu:34)."""
import numpy as np

import draws


def _site_matrix(oracle, n, D, pm_prob, seed=11, gen=3):
    um = draws.mutation_draws_np(oracle, seed, gen, n, D, pm_prob)
    return (um[:, 0] == 0.0).reshape(n, D), um


def test_site_frequency_matches_the_limit(oracle):
    n, D, pm_prob = 4000, 50, 1.0
    sites, um = _site_matrix(oracle, n, D, pm_prob)
    p = pm_prob / D
    freq = sites.mean()
    assert abs(freq - p) < 4 * np.sqrt(p * (1 - p) / (n * D))
    # every position alike: chi-square of the per-position counts
    per_pos = sites.sum(0)
    expected = n * p
    chi2 = ((per_pos - expected) ** 2 / expected).sum()
    assert chi2 < D + 6 * np.sqrt(2 * D)
    # sites per child: binomial(D, p)
    per_child = sites.sum(1)
    assert abs(per_child.mean() - D * p) < 4 * np.sqrt(D * p * (1 - p) / n)
    assert abs(per_child.var() - D * p * (1 - p)) < 0.15 * D * p
    # amplitudes are uniform draws in [0, 1)
    amp = um[sites.reshape(-1), 1]
    assert amp.min() >= 0.0 and amp.max() < 1.0 and abs(amp.mean() - 0.5) < 0.05


def test_every_variable_mutates_at_limit_one(oracle):
    sites, _ = _site_matrix(oracle, 40, 8, 8.0)
    assert sites.all()


def test_no_site_without_mutation_probability(oracle):
    sites, _ = _site_matrix(oracle, 40, 8, 0.0)
    assert not sites.any()


def test_crossover_draws_layout(oracle):
    # one block per four variables of a pair; words in variable order
    n, D = 10, 6
    u, sign, copy = draws.crossover_draws_np(oracle, 5, 1, n, D, 0.5, 0.25)
    blocks = oracle.philox_stream(5, 1, draws.TAG_CROSSOVER, (n // 2) * 2)
    w = blocks.reshape(n // 2, 8)[:, :D].reshape(-1)
    np.testing.assert_array_equal(sign, (w & 1).astype(np.int32))
    np.testing.assert_array_equal(u[:, 0], (w >> 8).astype(np.float32) / np.float32(16777216.0))
    assert (u[:, 1] > 0).any() and (copy > 0).any()
    u1, _, c1 = draws.crossover_draws_np(oracle, 5, 1, n, D, 1.0, 0.0)
    assert not u1[:, 1].any() and not c1.any()
