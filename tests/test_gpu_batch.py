"""GPU: batched instances (cuda_moea.Batch) against the same instances run
one at a time through the plain algorithm: variables, objectives, violations
and front indices must be identical after every checked generation."""
import numpy as np
import pytest
import torch

import cuda_moea as cm

pytestmark = pytest.mark.gpu

KINDS = ["DTLZ1", "DTLZ2", "DTLZ3", "DTLZ4", "DTLZ5", "DTLZ6", "DTLZ7"]


def _specs(count, seed, n_lo=92, n_hi=700):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        kind = KINDS[i % len(KINDS)]
        M = int(rng.choice([3, 5, 8]))
        N = int(rng.integers(n_lo // 2, n_hi // 2 + 1)) * 2
        D = M + (19 if kind == "DTLZ7" else 9)
        out.append((kind, M, N, D, 1000 + i))
    return out


def _make(spec, T):
    kind, M, N, D, seed = spec
    prob = getattr(cm, kind)(D, M)
    return cm.NSGA3(population_size=N, max_generations=T, problem=prob, seed=seed, print_progress=False)


def _same(a, b):
    torch.testing.assert_close(a.variables.cpu(), b.variables.cpu(), rtol=0, atol=0, equal_nan=True)
    torch.testing.assert_close(a.objectives.cpu(), b.objectives.cpu(), rtol=0, atol=0, equal_nan=True)
    torch.testing.assert_close(a.constraints.cpu(), b.constraints.cpu(), rtol=0, atol=0, equal_nan=True)


def test_batch_equals_instances_run_alone():
    T = 6
    specs = _specs(12, 7)
    batch = cm.Batch([_make(s, T) for s in specs])
    assert len(batch) == 12
    assert batch.fused  # NSGA-III on DTLZ1-7 with 2N <= 8192: one launch per stage
    batch.run(3)
    mid = [batch.result(i) for i in range(len(specs))]
    batch.run()
    assert batch.generation == T
    assert batch.graph_kernels > 0
    for i, s in enumerate(specs):
        alone = _make(s, T)
        alone.initialize()
        for _ in range(3):
            alone.step()
        r3 = alone.result()
        _same(mid[i], r3)
        np.testing.assert_array_equal(mid[i].auxiliary_indices.cpu().numpy(), r3.auxiliary_indices.cpu().numpy())
        r = alone.run()
        got = batch.result(i)
        _same(got, r)
        np.testing.assert_array_equal(got.auxiliary_indices.cpu().numpy(), r.auxiliary_indices.cpu().numpy())


def test_batch_rvea_and_constrained_instances():
    T = 5
    algos = [cm.RVEA(population_size=120, max_generations=T, problem=cm.DTLZ2(12, 3), seed=3,
                     print_progress=False),
             cm.NSGA3(population_size=200, max_generations=T, problem=cm.C1DTLZ1(12, 3), seed=4,
                      print_progress=False),
             cm.NSGA3(population_size=92, max_generations=T, problem=cm.DTLZ4(14, 5), seed=5,
                      print_progress=False)]
    batch = cm.Batch(algos)
    batch.run()
    alone = [cm.RVEA(population_size=120, max_generations=T, problem=cm.DTLZ2(12, 3), seed=3,
                     print_progress=False),
             cm.NSGA3(population_size=200, max_generations=T, problem=cm.C1DTLZ1(12, 3), seed=4,
                      print_progress=False),
             cm.NSGA3(population_size=92, max_generations=T, problem=cm.DTLZ4(14, 5), seed=5,
                      print_progress=False)]
    for i, a in enumerate(alone):
        r = a.run()
        got = batch.result(i)
        _same(got, r)
        assert got.active_count == r.active_count


def test_batch_rejects_callbacks_and_mismatched_generations():
    from cuda_moea._lib import MoeaError

    class Sphere(cm.PythonProblem):
        def __init__(self):
            super().__init__(4, 2)

        def evaluate(self, x, context):
            return torch.stack((x.square().sum(1), (x - 1).square().sum(1)), 1)

    with pytest.raises((MoeaError, ValueError)):
        cm.Batch([cm.NSGA3(population_size=32, max_generations=3, problem=Sphere(), print_progress=False)])
    with pytest.raises(MoeaError):
        cm.Batch([cm.NSGA3(population_size=32, max_generations=3, problem=cm.DTLZ2(12, 3), print_progress=False),
                  cm.NSGA3(population_size=32, max_generations=4, problem=cm.DTLZ2(12, 3), print_progress=False)])


@pytest.mark.parametrize("seed,n_hi", [(21, 4096), (22, 200)])
def test_fused_batch_equals_branch_batch(seed, n_hi):
    """The fused batch (one launch per stage) against the graph-branch batch on
    the same instances, including the largest fused size (N = 4096) and tiny
    populations."""
    T = 4
    specs = _specs(9, seed, n_lo=92, n_hi=n_hi)
    if n_hi == 4096:
        specs[0] = ("DTLZ1", 3, 4096, 12, 7)
        specs[1] = ("DTLZ7", 8, 4096, 27, 8)
    fused = cm.Batch([_make(s, T) for s in specs])
    branch = cm.Batch([_make(s, T) for s in specs], fuse=False)
    assert fused.fused and not branch.fused
    for _ in range(T):
        fused.step()
        branch.step()
        for i in range(len(specs)):
            a, b = fused.result(i), branch.result(i)
            _same(a, b)
            np.testing.assert_array_equal(a.auxiliary_indices.cpu().numpy(), b.auxiliary_indices.cpu().numpy())


def test_half_width_tiles_equal_full_width_tiles():
    """The half-width dominance tiles (twice the tile CTAs, each staging half
    the word tables) write the same dominance rows as the full-width ones, for
    every objective count that selects its own tile width."""
    T = 4
    rng = np.random.default_rng(5)
    specs = []
    for i, M in enumerate([2, 3, 4, 5, 6, 8, 9, 10, 12]):
        kind = KINDS[i % len(KINDS)]
        N = int(rng.integers(46, 1200)) * 2
        specs.append((kind, M, N, M + (19 if kind == "DTLZ7" else 9), 300 + i))
    specs.append(("DTLZ2", 5, 4096, 14, 9))
    full = cm.Batch([_make(s, T) for s in specs])
    half = cm.Batch([_make(s, T) for s in specs], half_tiles=True)
    assert full.fused and half.fused
    assert full.schedule["half_tiles"] == []
    assert half.schedule["half_tiles"] == sorted({s[1] for s in specs})
    for _ in range(T):
        full.step()
        half.step()
        for i in range(len(specs)):
            a, b = full.result(i), half.result(i)
            _same(a, b)
            np.testing.assert_array_equal(a.auxiliary_indices.cpu().numpy(), b.auxiliary_indices.cpu().numpy())


def test_autotuned_batch_equals_instances_and_caches_its_schedule():
    """The autotuned schedule (tuned on a scratch copy of the batch) changes
    how the generation is launched, never what it computes; a second batch of
    the same mix takes the cached schedule."""
    T = 12
    specs = _specs(40, 11)
    batch = cm.Batch([_make(s, T) for s in specs], autotune=True)
    sched = batch.schedule
    assert batch.fused and sched["source"] == "autotuned"
    assert sched["groups"] >= 1 and sched["tuned_ms"] > 0 and sched["default_ms"] > 0
    assert sched["tuned_ms"] <= sched["default_ms"] * 1.0001
    assert sorted(set(sched["group_of"])) == list(range(sched["groups"]))
    batch.run()
    again = cm.Batch([_make(s, T) for s in specs], autotune=True)
    assert again.schedule["source"] == "autotuned (cached)"
    assert again.schedule["group_of"] == sched["group_of"]
    assert again.schedule["half_tiles"] == sched["half_tiles"]
    assert set(sched["half_tiles"]) <= {s[1] for s in specs}
    again.close()
    for i in (0, 7, 19, 39):
        r = _make(specs[i], T).run()
        got = batch.result(i)
        _same(got, r)
        np.testing.assert_array_equal(got.auxiliary_indices.cpu().numpy(), r.auxiliary_indices.cpu().numpy())
