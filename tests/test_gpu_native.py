"""Problem plugins on the GPU: the plugin's objectives and constraints against
a float64 restatement of its formula, whole NSGA3 / RVEA runs through the
plugin hooks (determinism, the constraint that switches on through
prepare_parent, reset), and the evaluation benchmark."""
import ctypes
from pathlib import Path

import pytest
import torch

import cuda_moea as cm
from cuda_moea import native
from cuda_moea._lib import check, lib

pytestmark = pytest.mark.gpu

HERE = Path(__file__).resolve().parent
CACHE = HERE / ".native_cache"
D = 6


@pytest.fixture(scope="module")
def spheres_lib():
    return native.build_problem(HERE / "native" / "weighted_spheres", cache_dir=CACHE)


def _problem(lib_path, **params):
    return cm.NativeProblem(library=lib_path, name="WeightedSpheres", dimension=D, objectives=2,
                            lower_bounds=-1.0, upper_bounds=2.0, parameters=params)


def _formula(x, shift=0.5, weights=(1.0, 1.0), radius=1.0, constrained=False):
    x = x.to(torch.float64)
    a = x.square().sum(1)
    f = torch.stack((weights[0] * a, weights[1] * (x - shift).square().sum(1)), 1)
    cv = (a - radius * radius).clamp_min(0) if constrained else torch.zeros_like(a)
    return f, cv


def test_plugin_evaluation_matches_formula(spheres_lib):
    from cuda_moea.native import NativeInstance
    params = dict(shift=0.25, weights=[2.0, 0.5], radius=1.5, constrained=True)
    inst = NativeInstance(_problem(spheres_lib, **params)._spec())
    g = torch.Generator(device="cuda").manual_seed(5)
    for N in (1, 1000, 70001):
        x = torch.rand((N, D), device="cuda", generator=g) * 3 - 1
        objs = torch.full((2, N), float("nan"), device="cuda")
        cv = torch.full((N,), float("nan"), device="cuda")
        s = torch.cuda.current_stream()
        check(lib().moea_native_evaluate(inst.ptr, x.data_ptr(), objs.data_ptr(), cv.data_ptr(), N, D, 2, 0, 10,
                                         ctypes.c_void_p(s.cuda_stream)))
        torch.cuda.synchronize()
        f, c = _formula(x, 0.25, (2.0, 0.5), 1.5, True)
        torch.testing.assert_close(objs.t().to(torch.float64), f, rtol=1e-5, atol=1e-5)
        torch.testing.assert_close(cv.to(torch.float64), c, rtol=1e-5, atol=1e-5)
        assert (c > 0).any() and (c == 0).any() or N == 1


@pytest.mark.parametrize("algorithm", [cm.NSGA3, cm.RVEA])
def test_plugin_runs_are_deterministic_and_evaluated_by_the_plugin(spheres_lib, algorithm):
    results = []
    for _ in range(2):
        a = algorithm(problem=_problem(spheres_lib, shift=0.75, weights=[1.0, 3.0]), population_size=256,
                      max_generations=15, seed=41, enable_warmup=False, print_progress=False)
        results.append(a.run())
    r0, r1 = results
    assert r0.active_count == r1.active_count > 0
    # RVEA leaves NaN rows in inactive slots: bitwise equality with NaN == NaN
    torch.testing.assert_close(r0.variables, r1.variables, rtol=0, atol=0, equal_nan=True)
    torch.testing.assert_close(r0.objectives, r1.objectives, rtol=0, atol=0, equal_nan=True)
    valid = torch.isfinite(r0.variables).all(1)
    f, _ = _formula(r0.variables[valid], 0.75, (1.0, 3.0))
    torch.testing.assert_close(r0.objectives[valid].to(torch.float64), f, rtol=1e-5, atol=1e-5)


def test_constraint_switches_on_through_prepare_parent(spheres_lib):
    switch = 3
    a = cm.NSGA3(problem=_problem(spheres_lib, constrained=True, switch_at=switch), population_size=200,
                 max_generations=12, seed=7, enable_warmup=False, print_progress=False)
    a.initialize()
    while a.generation < switch - 1:
        a.step()
    pop = a.population
    valid = torch.isfinite(pop.variables).all(1)
    assert (pop.constraints[valid] == 0).all()
    while a.generation < switch + 2:
        a.step()
    pop = a.population
    valid = torch.isfinite(pop.variables).all(1)
    _, cv = _formula(pop.variables[valid], constrained=True)
    torch.testing.assert_close(pop.constraints[valid].to(torch.float64), cv, rtol=1e-5, atol=1e-5)
    a.reset()
    assert a.generation == 0
    pop = a.population
    valid = torch.isfinite(pop.variables).all(1)
    assert valid.any()
    r = a.run()
    assert r.active_count > 0


def test_plugin_benchmark(spheres_lib):
    x = torch.rand((4096, D), device="cuda") * 3 - 1
    out = native.benchmark(_problem(spheres_lib), x, repeats=20, warmup=3)
    assert out["size"] == 4096 and out["repeats"] == 20
    assert out["cuda_ms_per_eval"] > 0 and out["wall_ms_per_eval"] > 0


# The reference's example plugin (examples/native/bi_sphere) compiled unchanged
# against this SDK by oracle/ref/Makefile; the two cases follow the reference's
# GPU plugin tests (tests/python/test_native_problem.py:234-270).
BI_SPHERE = HERE.parent / "oracle" / "_ref" / "bi_sphere" / "problem.so"
needs_bi_sphere = pytest.mark.skipif(not BI_SPHERE.is_file(), reason="reference example plugin not built")


def _bi_sphere(**kwargs):
    options = dict(library=BI_SPHERE, name="BiSphere", dimension=7, objectives=2,
                   lower_bounds=-5.0, upper_bounds=5.0)
    options.update(kwargs)
    return cm.NativeProblem(**options)


@needs_bi_sphere
def test_reference_plugin_unconstrained_and_benchmark():
    p = _bi_sphere(parameters={"offset": 2.0})
    algo = cm.NSGA3(problem=p, population_size=32, max_generations=1, enable_warmup=False, print_progress=False)
    result = algo.run()
    torch.testing.assert_close(result.constraints, torch.zeros_like(result.constraints))
    timing = native.benchmark(p, result.variables, repeats=3, warmup=1)
    assert timing["wall_ms_per_eval"] > 0
    assert timing["cuda_ms_per_eval"] > 0


@needs_bi_sphere
@pytest.mark.parametrize("algorithm", [cm.NSGA3, cm.RVEA])
@pytest.mark.parametrize("dimension", [7, 129])
def test_reference_plugin_objectives_constraints_streams_reset_and_lifetime(algorithm, dimension):
    import gc
    p = _bi_sphere(dimension=dimension, parameters={"offset": 1.5, "radius": 2.0, "constrained": True})
    with torch.cuda.stream(torch.cuda.Stream()):
        algo = algorithm(problem=p, population_size=32, max_generations=2, enable_warmup=False,
                         print_progress=False)
        algo.initialize()
        for action in (lambda: None, algo.step, algo.reset):
            action()
            population = algo.population
            valid = torch.isfinite(population.variables).all(1)
            assert valid.any()
            x = population.variables[valid]
            expected = torch.stack((x.square().sum(1), (x - 1.5).square().sum(1)), 1)
            torch.testing.assert_close(population.objectives[valid], expected, rtol=2e-5, atol=2e-4)
            torch.testing.assert_close(population.constraints[valid], (expected[:, 0] - 4).clamp_min(0),
                                       rtol=2e-5, atol=2e-4)
        del population, x, expected, valid
        result = algo.run(copy=False)
        del algo, p
        gc.collect()
        assert result.active_count > 0
        assert torch.isfinite(result.objectives[:result.active_count]).all()
