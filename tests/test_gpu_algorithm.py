"""End-to-end runs of NSGA3 / RVEA through the Python API on the GPU: API
behaviour of the reference (shapes, CUDA tensors, reset, streams), a
generation-by-generation trajectory check of NSGA-III against the oracle's
selection, graph replay against direct launches, and solution quality (IGD on
the analytic DTLZ2 front)."""
import numpy as np
import pytest
import torch

import cuda_moea as cm

pytestmark = pytest.mark.gpu


class Sphere(cm.PythonProblem):
    def __init__(self):
        super().__init__(4, 2)

    def evaluate(self, variables, context):
        return torch.stack((variables.square().sum(1), (variables - 1).square().sum(1)), 1)


class BiSphere(cm.PythonProblem):
    """Two shifted spheres with a radius constraint (the reference's BiSphere plugin)."""

    def __init__(self, dimension, offset=1.5, radius=2.0):
        super().__init__(dimension, 2, -5.0, 5.0, constraints=1)
        self.offset, self.radius = offset, radius

    def evaluate(self, x, context):
        f = torch.stack((x.square().sum(1), (x - self.offset).square().sum(1)), 1)
        return f, (f[:, 0] - self.radius ** 2).clamp_min(0)


def igd_dtlz2(objs: torch.Tensor) -> float:
    ref = torch.from_numpy(__import__("oracle.oracle", fromlist=["x"]).reference_directions(1, 30, 3).T.copy())
    ref = ref.to(objs.device, torch.float64)  # unit directions lie on the DTLZ2 front
    d = torch.cdist(ref, objs.to(torch.float64))
    return float(d.min(1).values.mean())


def test_cuda_smoke_python_problem():
    algorithm = cm.NSGA3(population_size=32, max_generations=2, problem=Sphere(),
                         enable_warmup=False, print_progress=False)
    result = algorithm.run()
    assert tuple(result.variables.shape) == (32, 4)
    assert tuple(result.objectives.shape) == (32, 2)
    assert result.variables.is_cuda
    x = result.variables
    torch.testing.assert_close(result.objectives,
                               torch.stack((x.square().sum(1), (x - 1).square().sum(1)), 1))


@pytest.mark.parametrize("algorithm", [cm.NSGA3, cm.RVEA])
@pytest.mark.parametrize("dimension", [7, 129])
def test_python_problem_streams_reset_lifetime(algorithm, dimension):
    p = BiSphere(dimension)
    with torch.cuda.stream(torch.cuda.Stream()):
        algo = algorithm(problem=p, population_size=32, max_generations=2, enable_warmup=False,
                         print_progress=False)
        algo.initialize()
        for action in (lambda: None, algo.step, algo.reset):
            action()
            pop = algo.population
            valid = torch.isfinite(pop.variables).all(1)
            assert valid.any()
            x = pop.variables[valid]
            f = torch.stack((x.square().sum(1), (x - 1.5).square().sum(1)), 1)
            torch.testing.assert_close(pop.objectives[valid], f, rtol=2e-5, atol=2e-4)
            torch.testing.assert_close(pop.constraints[valid], (f[:, 0] - 4).clamp_min(0),
                                       rtol=2e-5, atol=2e-4)
        result = algo.run(copy=False)
        del algo, p
        assert result.active_count > 0
        assert torch.isfinite(result.objectives[:result.active_count]).all()


TRAJECTORIES = [
    # (problem, D, M, N, generations, seed, two-layer directions or None)
    ("DTLZ1", 7, 3, 200, 6, 77, None),
    # the constrained ten-objective configuration, two-layer (3, 2) = 275
    # user-defined directions; beyond the reference's eight objectives, so the
    # oracle alone is the check
    ("C1DTLZ1", 14, 10, 400, 5, 5, (3, 2)),
    ("C3DTLZ4", 14, 10, 400, 5, 6, (3, 2)),
]


@pytest.mark.parametrize("kind,D,M,N,T,seed,layers", TRAJECTORIES)
def test_nsga3_trajectory_matches_oracle_selection(oracle, kind, D, M, N, T, seed, layers):
    """Each generation: offspring from the fused reproduction kernel (same
    Philox streams as the algorithm), objectives from the problem kernel, then
    the oracle's NSGA-III selection must reproduce the algorithm's next
    parents exactly (survivor set, fronts, objectives, niching RNG offset)."""
    from cuda_moea import stages
    from cuda_moea.problem import PROBLEM_KINDS
    kw = {}
    if layers is not None:
        kw["reference_directions"] = cm.UserDefinedDirections(cm.two_layer_directions(M, *layers))
    algo = cm.NSGA3(population_size=N, max_generations=T, problem=getattr(cm, kind)(D, M), seed=seed,
                    print_progress=False, use_graphs=False, **kw)
    algo.initialize()
    if layers is None:
        refs = oracle.reference_directions(0, N, M)
    else:
        refs = algo.reference_directions.cpu().numpy().copy()
        assert refs.shape == (M, 275)
    pop = algo.population
    par_x = pop.variables.clone()
    par_f = pop.objectives.t().contiguous().cpu().numpy()
    par_cv = pop.constraints.cpu().numpy().copy()
    ideal = par_f.min(1).astype(np.float32)
    fronts0, _ = oracle.ndsort(par_cv, par_f, N)
    rank = torch.from_numpy(fronts0).cuda()
    bounds = torch.tile(torch.tensor([0.0, 1.0]), (D,)).cuda()
    dseed = oracle.derive_seed(seed)
    offset = 0
    constrained = False
    for g in range(T):
        off_x, _ = stages.reproduce(par_x, torch.from_numpy(par_cv).cuda(), rank, N, bounds, N,
                                    seed=dseed, generation=g)
        off_f, off_cv = stages.problem_evaluate(PROBLEM_KINDS[kind], off_x, M)
        mix_f = np.concatenate([par_f, off_f.cpu().numpy()], 1)
        mix_cv = np.concatenate([par_cv, off_cv.cpu().numpy()])
        constrained |= bool((mix_cv > 0).any())
        want = oracle.nsga3_select(mix_cv, mix_f, refs, dseed, offset, ideal)
        offset, ideal = want["offset"], want["ideal"]
        algo.step()
        pop = algo.population
        surv = want["survivors"]
        mix_x = torch.cat([par_x, off_x]).cpu().numpy()
        np.testing.assert_array_equal(pop.variables.cpu().numpy(), mix_x[surv])
        np.testing.assert_array_equal(pop.objectives.t().cpu().numpy(), mix_f[:, surv])
        np.testing.assert_array_equal(pop.constraints.cpu().numpy(), mix_cv[surv])
        par_x = pop.variables.clone()
        par_f = pop.objectives.t().contiguous().cpu().numpy()
        par_cv = pop.constraints.cpu().numpy().copy()
        rank = torch.from_numpy(want["fronts"]).cuda()
    if kind.startswith("C"):
        assert constrained  # the violation-first dominance was exercised


@pytest.mark.parametrize("kind", ["NSGA3", "RVEA"])
def test_graph_replay_equals_direct_launches(kind):
    runs = []
    for graphs in (True, False):
        a = cm.Algorithm(kind, population_size=256, max_generations=8, problem=cm.DTLZ2(12, 3),
                         seed=5, print_progress=False, use_graphs=graphs)
        r = a.run()
        runs.append((r.variables.cpu(), r.objectives.cpu(), r.active_count))
    torch.testing.assert_close(runs[0][0], runs[1][0], rtol=0, atol=0, equal_nan=True)
    torch.testing.assert_close(runs[0][1], runs[1][1], rtol=0, atol=0, equal_nan=True)
    assert runs[0][2] == runs[1][2]


@pytest.mark.parametrize("problem,dirs", [("DTLZ1", None), ("DTLZ2", "user_unnormalised")])
def test_association_modes_give_identical_runs(problem, dirs):
    runs = []
    for mode in (0, 1, 2):
        kw = {}
        if dirs == "user_unnormalised":
            d = torch.rand(150, 3, generator=torch.Generator().manual_seed(3)) * 2 + 0.05
            kw["reference_directions"] = cm.UserDefinedDirections(d, normalize=False)
        prob = cm.DTLZ1(7, 3) if problem == "DTLZ1" else cm.DTLZ2(12, 3)
        a = cm.NSGA3(population_size=1000, max_generations=12, problem=prob, seed=11,
                     environment_selector=cm.NSGA3EnvironmentSelector(association_mode=mode),
                     print_progress=False, **kw)
        r = a.run()
        runs.append((r.variables.cpu(), r.objectives.cpu()))
    for other in runs[1:]:
        torch.testing.assert_close(runs[0][0], other[0], rtol=0, atol=0)
        torch.testing.assert_close(runs[0][1], other[1], rtol=0, atol=0)


def test_many_objective_default_search_equals_scan():
    """Eight objectives, 6435 directions, 8400 merged points: the default mode
    takes the tensor-core search there (the cone tree covers M <= 5); every
    generation equals the full scan's and the explicit tensor mode's."""
    runs = []
    for mode in (0, 1, 2):
        a = cm.NSGA3(population_size=4200, max_generations=6, problem=cm.DTLZ2(17, 8), seed=23,
                     reference_directions=cm.DasDennisDirections(8), print_progress=False,
                     environment_selector=cm.NSGA3EnvironmentSelector(association_mode=mode))
        a.initialize()
        gens = []
        for _ in range(6):
            a.step()
            r = a.result()
            gens.append((r.variables.cpu(), r.auxiliary_indices.cpu()))
        runs.append(gens)
    for other in runs[1:]:
        for g, (x, y) in enumerate(zip(runs[0], other)):
            torch.testing.assert_close(x[0], y[0], rtol=0, atol=0, msg=f"variables, generation {g}")
            torch.testing.assert_close(x[1], y[1], rtol=0, atol=0, msg=f"fronts, generation {g}")


def test_nsga3_dtlz2_quality():
    algo = cm.NSGA3(population_size=92, max_generations=100, problem=cm.DTLZ2(12, 3), seed=2887,
                    print_progress=False)
    r = algo.run()
    assert r.total_ms > 0
    assert igd_dtlz2(r.objectives) < 0.08
    # NSGA-III keeps the survivor fronts as result indices
    assert r.auxiliary_indices.shape == (92,) and int(r.auxiliary_indices.min()) >= 0


def test_rvea_dtlz2_quality_and_front_zero():
    algo = cm.RVEA(population_size=92, max_generations=100, problem=cm.DTLZ2(12, 3), seed=2887,
                   print_progress=False)
    r = algo.run()
    act = r.active_count
    assert 0 < act <= 92
    assert igd_dtlz2(r.objectives[:act]) < 0.1
    aux = r.auxiliary_indices.cpu().numpy()
    assert len(aux) > 0 and aux.max() < act


def test_constrained_and_quantized_and_user_directions():
    algo = cm.NSGA3(population_size=200, max_generations=20, problem=cm.C1DTLZ1(12, 3),
                    environment_selector=cm.NSGA3EnvironmentSelector(cv_bins=16, cv_clip_upper=10.0),
                    print_progress=False)
    r = algo.run()
    assert torch.isfinite(r.objectives).all()
    algo = cm.NSGA3(population_size=100, max_generations=5, problem=cm.DTLZ2(12, 3),
                    reference_directions=cm.UserDefinedDirections(torch.eye(3) + 0.1),
                    print_progress=False)
    r = algo.run()
    assert tuple(r.objectives.shape) == (100, 3)
    # RVEA with fixed two-layer directions (gamma computed for any provider)
    algo = cm.RVEA(population_size=64, max_generations=5, problem=cm.DTLZ2(17, 8),
                   reference_directions=cm.DasDennisDirections(3), print_progress=False)
    assert algo.run().active_count > 0


def test_errors_raise():
    with pytest.raises(Exception):
        cm.NSGA3(population_size=33, max_generations=2, print_progress=False).run()
    with pytest.raises(Exception):
        cm.RVEA(population_size=32, max_generations=2, mating=cm.TournamentMating(),
                print_progress=False).run()


@pytest.mark.parametrize("problem,D,M,N", [("DTLZ2", 12, 3, 92), ("DTLZ7", 24, 5, 500), ("DTLZ1", 12, 8, 1000),
                                           ("DTLZ4", 12, 3, 4096)])
@pytest.mark.parametrize("graphs", [True, False])
def test_small_population_fused_equals_staged(problem, D, M, N, graphs):
    """Populations with 2N <= 8192 run as the fused generation by default;
    every generation equals the staged path's."""
    runs = []
    for fuse in (True, False):
        a = cm.NSGA3(population_size=N, max_generations=8, problem=getattr(cm, problem)(D, M), seed=17,
                     print_progress=False, use_graphs=graphs, fuse_small=fuse)
        a.initialize()
        gens = []
        for _ in range(8):
            a.step()
            r = a.result()
            gens.append((r.variables.cpu(), r.objectives.cpu(), r.auxiliary_indices.cpu()))
        runs.append(gens)
    for g, (x, y) in enumerate(zip(runs[0], runs[1])):
        torch.testing.assert_close(x[0], y[0], rtol=0, atol=0, msg=f"variables, generation {g}")
        torch.testing.assert_close(x[1], y[1], rtol=0, atol=0, msg=f"objectives, generation {g}")
        torch.testing.assert_close(x[2], y[2], rtol=0, atol=0, msg=f"fronts, generation {g}")


@pytest.mark.parametrize("D", [12, 20001])
def test_rvea_dead_rows_without_views_equal_rows_with_views(D):
    """The RVEA update skips dead rows that already hold the NaN sentinels
    from an earlier generation of the same slot, and writes them again once a
    population view has been handed out.  A run that takes no view until its
    end must equal, bit for bit and NaN rows included, a run that takes one
    every generation.  D=20001 cuts rows into several update work items and
    leaves no 16-byte row alignment."""
    def run(view_each):
        algo = cm.RVEA(population_size=120, max_generations=12, problem=cm.DTLZ2(D, 3), seed=99,
                       print_progress=False)
        algo.initialize()
        for _ in range(12):
            algo.step()
            if view_each:
                algo.population_view()
        r = algo.result()
        return (r.variables, r.objectives, r.constraints, r.active_count)
    a, b = run(True), run(False)
    for x, y in zip(a[:3], b[:3]):
        assert torch.equal(x.view(torch.int32), y.view(torch.int32))
    assert a[3] == b[3]
    assert a[3] < 120 and torch.isnan(a[0][a[3]:]).all()
