"""GPU: runs composed from strategy objects (cuda_moea/composed.py), the form
the Python crossover, mutation and environmental-selection strategies run in.

- With only built-in strategies (forced through the composed step) every
  generation equals the algorithm object's, bit for bit: NSGA-III (fused and
  staged sizes), constrained NSGA-III with a constraint-activation schedule,
  and RVEA with adaptive directions.
- A PythonCrossover that copies the mated parents plus a PythonMutation that
  returns None reproduce the algorithm object with SBX probability 0 and no
  mutation; a PythonEnvironmentSelector is called with the documented views
  and its indices / state (rank for tournament mating, active count, result
  indices) are honoured; a PythonReferenceDirections' update runs after every
  selection.
- The reference's own custom-strategy smoke case (tests/python/test_api.py
  of CUDA-MOEA) runs end to end.
"""
import pytest
import torch

import cuda_moea as cm

pytestmark = pytest.mark.gpu


def _bits(t):
    return t.contiguous().view(torch.int32)


def _lockstep(make, generations):
    a, b = make(), make()
    b._compose = True
    a.initialize()
    b.initialize()
    for g in range(generations):
        a.step()
        b.step()
        ra, rb = a.result(), b.result()
        assert torch.equal(_bits(ra.variables), _bits(rb.variables)), f"variables, generation {g}"
        assert torch.equal(_bits(ra.objectives), _bits(rb.objectives)), f"objectives, generation {g}"
        assert torch.equal(_bits(ra.constraints), _bits(rb.constraints)), f"violations, generation {g}"
        assert ra.active_count == rb.active_count
        assert torch.equal(ra.auxiliary_indices, rb.auxiliary_indices), f"result indices, generation {g}"
    assert torch.equal(_bits(a.reference_directions), _bits(b.reference_directions))


@pytest.mark.parametrize("N", [256, 6000])
def test_composed_builtins_equal_algorithm_nsga3(N):
    _lockstep(lambda: cm.NSGA3(population_size=N, max_generations=12, problem=cm.DTLZ1(7, 3), seed=4,
                               crossover=cm.SBX(eta_initial=30.0, eta_final=5.0, variable_copy_probability=0.3),
                               print_progress=False), 6)


def test_composed_builtins_equal_algorithm_constrained_schedule():
    _lockstep(lambda: cm.NSGA3(population_size=400, max_generations=8, problem=cm.C1DTLZ1(12, 3, 0.5), seed=9,
                               environment_selector=cm.NSGA3EnvironmentSelector(cv_bins=8, cv_clip_upper=4.0),
                               print_progress=False), 8)


def test_composed_builtins_equal_algorithm_rvea():
    _lockstep(lambda: cm.RVEA(population_size=300, max_generations=10, problem=cm.DTLZ2(17, 8), seed=6,
                              reference_directions=cm.AdaptiveRVEADirections(frequency=0.2),
                              print_progress=False), 7)


class CopyCrossover(cm.PythonCrossover):
    def __init__(self):
        self.calls = 0

    def initialize(self, info):
        self.info = info

    def apply(self, parents, parent_indices, context):
        self.calls += 1
        assert parent_indices.dtype == torch.int32 and parent_indices.is_cuda
        assert context["generation"] == self.calls - 1
        return parents["variables"][parent_indices.long()]


class KeepMutation(cm.PythonMutation):
    def __init__(self):
        self.calls = 0

    def mutate(self, offspring, context):
        self.calls += 1
        assert tuple(offspring["bounds"].shape) == (offspring["variables"].shape[1], 2)
        return None


def test_python_crossover_and_mutation_reproduce_builtin_equivalents():
    N, T = 200, 6
    ref = cm.NSGA3(population_size=N, max_generations=T, problem=cm.DTLZ2(12, 3), seed=3, print_progress=False,
                   crossover=cm.SBX(probability=0.0), mutation=cm.NoMutation()).run()
    cx, mu = CopyCrossover(), KeepMutation()
    algo = cm.NSGA3(population_size=N, max_generations=T, problem=cm.DTLZ2(12, 3), seed=3, print_progress=False,
                    crossover=cx, mutation=mu)
    got = algo.run()
    assert cx.calls == T and mu.calls == T
    assert cx.info["population_size"] == N and cx.info["dimension"] == 12
    assert torch.equal(_bits(ref.variables), _bits(got.variables))
    assert torch.equal(_bits(ref.objectives), _bits(got.objectives))
    assert torch.equal(ref.auxiliary_indices, got.auxiliary_indices)


class SumSelector(cm.PythonEnvironmentSelector):
    """Keeps the N members with the smallest objective sum; reports ranks for
    tournament mating and its result indices."""

    def initialize(self, info, references, context):
        self.info, self.references = info, references
        self.prepared = 0

    def prepare(self, population, context):
        self.prepared += 1
        n = population["variables"].shape[0]
        return {"rank": torch.zeros(n, dtype=torch.int32, device=population["variables"].device)}

    def select(self, parents, offspring, context):
        f = torch.cat([parents["objectives"], offspring["objectives"]])
        order = torch.argsort(f.sum(1), stable=True)[: parents["variables"].shape[0]]
        self.last = order
        rank = torch.arange(order.numel(), dtype=torch.int32, device=order.device) // 10
        return {"indices": order, "rank": rank, "active_count": order.numel(),
                "result_indices": torch.arange(5, dtype=torch.int32, device=order.device)}


def test_python_environment_selector():
    N, M = 120, 3
    sel = SumSelector()
    algo = cm.NSGA3(population_size=N, max_generations=4, problem=cm.DTLZ1(7, M), seed=8, print_progress=False,
                    environment_selector=sel)
    algo.initialize()
    assert sel.prepared == 1 and sel.info["population_size"] == N
    assert sel.references is not None and sel.references.shape[1] == M
    before = algo.population
    px, pf = before.variables.clone(), before.objectives.clone()
    algo.step()
    after = algo.result()
    # the next population is the selected rows of parents + offspring, in the selector's order
    assert tuple(after.objectives.shape) == (N, M)
    assert torch.equal(after.objectives[sel.last < N], pf[sel.last[sel.last < N].long()])
    s = after.objectives.sum(1)
    assert bool((s[1:] >= s[:-1]).all()), "rows in the selector's order"
    assert torch.equal(after.auxiliary_indices, torch.arange(5, dtype=torch.int32, device="cuda"))
    assert after.active_count == N
    assert not torch.equal(px, after.variables)
    algo.run()
    assert algo.generation == 4


class UpdatingReferences(cm.PythonReferenceDirections):
    def __init__(self):
        self.updates = 0

    def initialize(self, requested_count, objective_count, context):
        return torch.eye(objective_count, device=f"cuda:{context['device']}") + 0.1

    def update(self, population, directions, active_count, context):
        self.updates += 1
        assert directions.shape[1] == population["objectives"].shape[1]
        return directions * 1.0


def test_python_reference_directions_update():
    refs = UpdatingReferences()
    algo = cm.NSGA3(population_size=64, max_generations=5, problem=cm.DTLZ2(12, 3), seed=2, print_progress=False,
                    reference_directions=refs)
    r = algo.run()
    assert refs.updates == 5
    assert torch.isfinite(r.objectives).all()


class Sphere(cm.PythonProblem):
    def __init__(self):
        super().__init__(4, 2)

    def evaluate(self, variables, context):
        return torch.stack((variables.square().sum(1), (variables - 1).square().sum(1)), 1)


class Mating(cm.PythonMating):
    def select(self, parents, state, context):
        return torch.arange(parents["variables"].shape[0], device=parents["variables"].device, dtype=torch.int32)


class Crossover(cm.PythonCrossover):
    def apply(self, parents, parent_indices, context):
        return parents["variables"][parent_indices.long()]


class Mutation(cm.PythonMutation):
    def mutate(self, offspring, context):
        return offspring["variables"]


class References(cm.PythonReferenceDirections):
    def initialize(self, requested_count, objective_count, context):
        return torch.eye(objective_count, device=f"cuda:{context['device']}")


class Selector(cm.PythonEnvironmentSelector):
    def select(self, parents, offspring, context):
        size = parents["variables"].shape[0]
        return {"indices": torch.arange(size, device=parents["variables"].device)}


def test_reference_custom_strategy_smoke():
    algorithm = cm.NSGA3(population_size=32, max_generations=2, problem=Sphere(), mating=Mating(),
                         crossover=Crossover(), mutation=Mutation(), reference_directions=References(),
                         environment_selector=Selector(), enable_warmup=False, print_progress=False)
    result = algorithm.run()
    assert tuple(result.variables.shape) == (32, 4)
    assert tuple(result.objectives.shape) == (32, 2)
    assert result.variables.is_cuda
    # selecting the parents again: the population never changes
    x = result.variables
    torch.testing.assert_close(result.objectives, torch.stack((x.square().sum(1), (x - 1).square().sum(1)), 1))


def test_composed_builtins_equal_algorithm_rvea_more_directions_than_points():
    # 91 directions for 30 points: more winners than survivors, the truncation
    # by (flag, metric, index) of the elitism
    _lockstep(lambda: cm.RVEA(population_size=30, max_generations=10, problem=cm.DTLZ2(12, 3), seed=3,
                              reference_directions=cm.DasDennisDirections(12), print_progress=False), 8)
