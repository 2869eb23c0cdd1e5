"""GPU: snapshots in the reference's data-recorder layout
(nat/src/algorithm/data_recorder.cu:128-292) and resumption from them.

The format is checked file by file against the reference's text and binary
layout, the saved populations against a twin run stepped by hand, and a
resumed run against the uninterrupted one (bit for bit)."""
import json

import numpy as np
import pytest
import torch

import cuda_moea as cm
from cuda_moea._lib import MoeaError

pytestmark = pytest.mark.gpu


def _metadata_text(algorithm, problem, N, D, M, C, T, seed, interval, K):
    """metadata.json as data_recorder.cu:162-194 writes it."""
    name = "null" if problem is None else json.dumps(problem)
    return ("{\n"
            '  "format_version": 1,\n'
            '  "scalar_type": "float32",\n'
            '  "index_type": "int32",\n'
            f'  "algorithm_name": "{algorithm}",\n'
            f'  "problem_name": {name},\n'
            f'  "population_size": {N},\n'
            f'  "dimension": {D},\n'
            f'  "objective_count": {M},\n'
            f'  "constraint_count": {C},\n'
            f'  "max_generations": {T},\n'
            f'  "random_seed": {seed},\n'
            f'  "generation_interval": {interval},\n'
            f'  "reference_direction_count": {K},\n'
            '  "layouts": {\n'
            '    "variables": "row-major (N,D)",\n'
            '    "objectives": "objective-major (M,N)",\n'
            '    "constraints": "(N)",\n'
            '    "reference_directions": "objective-major (M,K)",\n'
            '    "bounds": "separate lower/upper arrays (D)"\n'
            "  }\n"
            "}\n")


def _snapshot_text(g, N, D, M, active, K, aux):
    """snapshot.json as data_recorder.cu:272-289 writes it."""
    return ("{\n"
            f'  "generation": {g},\n'
            f'  "population_size": {N},\n'
            f'  "dimension": {D},\n'
            f'  "objective_count": {M},\n'
            f'  "active_count": {active},\n'
            f'  "reference_direction_count": {K},\n'
            f'  "auxiliary_index_count": {aux}\n'
            "}\n")


def _f32(path, shape):
    a = np.fromfile(path, dtype=np.float32)
    assert a.size == int(np.prod(shape)), path
    return a.reshape(shape)


def test_snapshot_files_match_the_reference_layout(tmp_path):
    N, D, M, T, seed, every = 92, 12, 3, 5, 7, 2
    kw = dict(population_size=N, max_generations=T, problem=cm.DTLZ2(D, M), seed=seed, print_progress=False)
    algo = cm.NSGA3(save_data=tmp_path, save_interval=every, **kw)
    twin = cm.NSGA3(**kw)
    twin.initialize()
    states = {0: twin.result()}
    for g in range(1, T + 1):
        twin.step()
        states[g] = twin.result()
    algo.run()
    K = 91  # Das-Dennis directions of 12 partitions in 3 objectives
    assert (tmp_path / "metadata.json").read_text() == _metadata_text("NSGA-III", "DTLZ2", N, D, M, 0, T, seed,
                                                                    every, K)
    np.testing.assert_array_equal(np.fromfile(tmp_path / "lower_bounds.bin", np.float32), np.zeros(D, np.float32))
    np.testing.assert_array_equal(np.fromfile(tmp_path / "upper_bounds.bin", np.float32), np.ones(D, np.float32))
    dirs0 = _f32(tmp_path / "initial_reference_directions.bin", (M, K))
    saved = sorted(p.name for p in tmp_path.iterdir() if p.is_dir())
    assert saved == ["generation_000000", "generation_000002", "generation_000004", "generation_000005"]
    for g in (0, 2, 4, 5):
        d = tmp_path / f"generation_{g:06d}"
        want = states[g]
        np.testing.assert_array_equal(_f32(d / "variables.bin", (N, D)), want.variables.cpu().numpy())
        np.testing.assert_array_equal(_f32(d / "objectives.bin", (M, N)), want.objectives.t().cpu().numpy())
        np.testing.assert_array_equal(_f32(d / "constraints.bin", (N,)), want.constraints.cpu().numpy())
        np.testing.assert_array_equal(_f32(d / "reference_directions.bin", (M, K)), dirs0)
        np.testing.assert_array_equal(np.fromfile(d / "selector_auxiliary_indices.bin", np.int32),
                                      want.auxiliary_indices.cpu().numpy())
        assert (d / "snapshot.json").read_text() == _snapshot_text(g, N, D, M, N, K, N)


def _resume_case(kind, tmp_path):
    if kind == "nsga3_fused":
        return cm.NSGA3, dict(population_size=92, max_generations=10, problem=cm.DTLZ2(12, 3), seed=11)
    if kind == "nsga3_staged":
        return cm.NSGA3, dict(population_size=1000, max_generations=10, problem=cm.DTLZ1(7, 3), seed=12)
    if kind == "rvea_adaptive":
        return cm.RVEA, dict(population_size=120, max_generations=10, problem=cm.DTLZ2(12, 3), seed=13)
    if kind == "constrained_switch":
        # the constraint switch falls after the snapshot (generation 6 of 10)
        return cm.NSGA3, dict(population_size=200, max_generations=10, seed=14,
                              problem=cm.C1DTLZ1(12, 3, constraint_activation_ratio=0.6))
    raise ValueError(kind)


@pytest.mark.parametrize("kind", ["nsga3_fused", "nsga3_staged", "rvea_adaptive", "constrained_switch"])
def test_resume_equals_the_uninterrupted_run(tmp_path, kind):
    make, kw = _resume_case(kind, tmp_path)
    full = make(save_data=tmp_path / "run", save_interval=5, print_progress=False, **kw)
    want = full.run()
    resumed = make(print_progress=False, **kw)
    resumed.load_snapshot(tmp_path / "run" / "generation_000005")
    assert resumed.generation == 5
    got = resumed.run()
    for a, b in ((got.variables, want.variables), (got.objectives, want.objectives),
                 (got.constraints, want.constraints)):
        torch.testing.assert_close(a.cpu(), b.cpu(), rtol=0, atol=0, equal_nan=True)
    assert got.active_count == want.active_count
    np.testing.assert_array_equal(got.auxiliary_indices.cpu().numpy(), want.auxiliary_indices.cpu().numpy())


def test_named_python_problem_and_load_errors(tmp_path):
    class Sphere(cm.PythonProblem):
        def __init__(self):
            super().__init__(4, 2, constraints=0, name="Sphere \"2\"")

        def evaluate(self, x, context):
            return torch.stack((x.square().sum(1), (x - 1).square().sum(1)), 1)

    algo = cm.NSGA3(population_size=32, max_generations=3, problem=Sphere(), save_data=tmp_path / "py",
                    save_interval=3, print_progress=False)
    algo.run()
    meta = (tmp_path / "py" / "metadata.json").read_text()
    assert '"problem_name": "Sphere \\"2\\"",' in meta
    assert json.loads(meta)["problem_name"] == 'Sphere "2"'
    # a snapshot of another population size is rejected, and so is a missing one
    other = cm.NSGA3(population_size=34, max_generations=3, problem=Sphere(), print_progress=False)
    with pytest.raises(MoeaError):
        other.load_snapshot(tmp_path / "py" / "generation_000003")
    with pytest.raises(MoeaError):
        other.load_snapshot(tmp_path / "nothing_here")
    with pytest.raises(ValueError):
        cm.NSGA3(population_size=32, max_generations=3, save_data=tmp_path / "x", save_interval=0)
    with pytest.raises((MoeaError, ValueError)):
        cm.Batch([cm.NSGA3(population_size=32, max_generations=3, problem=cm.DTLZ2(12, 3),
                           save_data=tmp_path / "b", print_progress=False)])
