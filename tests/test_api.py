"""Construction of every problem and strategy through the Python API, as the
reference's CPU tests do (tests/python/test_api.py:45-104 of CUDA-MOEA)."""
import pytest
import torch

import cuda_moea as cm


class Sphere(cm.PythonProblem):
    def __init__(self):
        super().__init__(4, 2)

    def evaluate(self, variables, context):
        return torch.stack((variables.square().sum(1), (variables - 1).square().sum(1)), 1)


class Mating(cm.PythonMating):
    def select(self, parents, state, context):
        return torch.arange(parents["variables"].shape[0], device=parents["variables"].device,
                            dtype=torch.int32)


class Crossover(cm.PythonCrossover):
    def apply(self, parents, parent_indices, context):
        return parents["variables"][parent_indices.long()]


class Mutation(cm.PythonMutation):
    def mutate(self, offspring, context):
        return offspring["variables"]


class References(cm.PythonReferenceDirections):
    def initialize(self, requested_count, objective_count, context):
        return torch.eye(objective_count)


class Selector(cm.PythonEnvironmentSelector):
    def select(self, parents, offspring, context):
        size = parents["variables"].shape[0]
        return {"indices": torch.arange(size, device=parents["variables"].device)}


def test_sbx_variable_copy_probability():
    crossover = cm.SBX(variable_copy_probability=0.5)
    assert crossover._spec()["variable_copy_probability"] == 0.5
    algorithm = cm.NSGA3(population_size=16, max_generations=1, crossover=crossover, enable_warmup=False)
    assert not algorithm.initialized


def test_initial_population_construct():
    initial = torch.zeros((16, 4), dtype=torch.float32)
    algorithm = cm.NSGA3(population_size=16, max_generations=1, problem=Sphere(),
                         initial_population=initial, enable_warmup=False)
    assert not algorithm.initialized
    with pytest.raises(ValueError):
        cm.NSGA3(population_size=16, problem=Sphere(), initial_population=torch.zeros(8, 4))


def test_all_builtin_problems_construct():
    names = ["DTLZ1", "DTLZ2", "DTLZ3", "DTLZ4", "DTLZ5", "DTLZ6", "DTLZ7", "ConvexDTLZ2",
             "C1DTLZ1", "C1DTLZ3", "C2DTLZ2", "C2ConvexDTLZ2", "C3DTLZ1", "C3DTLZ4", "CSDP"]
    for name in names:
        algorithm = cm.NSGA3(population_size=16, max_generations=1, problem=getattr(cm, name)(8, 3),
                             enable_warmup=False)
        assert not algorithm.initialized


def test_all_builtin_strategies_construct():
    combinations = [
        dict(mating=cm.RandomMating(), crossover=cm.SBX(), mutation=cm.NoMutation(),
             reference_directions=cm.DasDennisDirections(2),
             environment_selector=cm.NSGA3EnvironmentSelector()),
        dict(mating=cm.TournamentMating(), mutation=cm.PolynomialMutation(),
             reference_directions=cm.AdaptiveRVEADirections(),
             environment_selector=cm.RVEAEnvironmentSelector()),
        dict(reference_directions=cm.UserDefinedDirections(torch.eye(3))),
    ]
    for options in combinations:
        assert not cm.Algorithm("NSGA3", population_size=16, max_generations=1,
                                enable_warmup=False, **options).initialized


def test_custom_strategies_construct():
    algorithm = cm.NSGA3(population_size=16, max_generations=1, problem=Sphere(), mating=Mating(),
                         crossover=Crossover(), mutation=Mutation(), reference_directions=References(),
                         environment_selector=Selector(), enable_warmup=False)
    assert not algorithm.initialized


def test_builder():
    algorithm = (cm.AlgorithmBuilder("RVEA").population_size(16).max_generations(2)
                 .problem(cm.DTLZ2()).build())
    assert algorithm.generation == 0


def test_invalid_algorithm_and_device():
    with pytest.raises(ValueError):
        cm.Algorithm("MOEAD")
    with pytest.raises(ValueError):
        cm.NSGA3(device="cpu")


def test_two_layer_directions():
    """Explicit two-layer Das-Dennis sets for UserDefinedDirections: the
    outer layer's compositions of h1, then the inner layer's compositions of
    h2 moved halfway to the centroid; rows on the simplex."""
    from math import comb

    import cuda_moea as cm
    d = cm.two_layer_directions(10, 3, 2)
    assert tuple(d.shape) == (comb(12, 9) + comb(11, 9), 10) == (275, 10)
    assert float((d.sum(1) - 1).abs().max()) < 1e-6
    outer, inner = d[:220], d[220:]
    assert float(((outer * 3) - (outer * 3).round()).abs().max()) < 1e-6  # multiples of 1/3
    assert float(inner.min()) >= 0.5 / 10 - 1e-7                           # shifted off the boundary
    assert len({tuple(r.tolist()) for r in d}) == 275                     # no repeated direction
    d3 = cm.two_layer_directions(3, 2, 0)
    assert tuple(d3.shape) == (6, 3)
    with pytest.raises(ValueError):
        cm.two_layer_directions(0, 3, 2)
