"""GPU: whole-run quality against the reference's own algorithm on the same
GPU, with the reference's published quality protocol (tests/benchmark/DTLZ/
plan.py quality_jobs and adapters/dtlz.py _run_cuda of CUDA-MOEA): DTLZ2,
M=3, D=12, N=1024 (RVEA: 990), 500 generations, initial populations uniform
from torch's CPU generator seeded with the run's seed, SBX eta 30 pc 1 with
copy probability 0.5, PM eta 20; NSGA-III on 990 Das-Dennis directions with
sparse ratio 1, RVEA on adaptive directions (frequency 0.1, alpha 2).

Whole trajectories are not portable between the two random streams, so the
check is statistical: the final IGD of every run (FP64, moea_igd, itself
pinned to the reference's metric) against 20000 seeded sphere samples, and
Welch's t of the mean difference between the product's runs and the
reference's runs over the same seeds, |t| < 4.  MOEA_QUALITY_SEEDS sets the
number of seeds (10 by default, 30 for the published protocol); run with -s to
print the summary.
"""
import os
import statistics

import pytest
import torch

import cuda_moea as cm
from oracle.ref import ref as R

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not R.algo_available(), reason="oracle/_ref not built (needs the reference sources)")]


def _runs(name, seeds):
    from cuda_moea import metrics, stages
    front = metrics.pareto_front_points("DTLZ2", 3, 20000, 2887).to(torch.float64).cuda()
    dirs = stages.reference_directions(2, 1024, 3)  # 990 directions, (M, count)
    alg = 0 if name == "NSGA3" else 1
    N = 1024 if alg == 0 else 990
    ours, ref, ms_ours, ms_ref = [], [], [], []
    for seed in range(seeds):
        gen = torch.Generator(device="cpu").manual_seed(seed)
        x0 = torch.empty((N, 12), dtype=torch.float32).uniform_(0.0, 1.0, generator=gen)
        objs, act, ms = R.algo_run(alg, 2, 12, 3, N, 500, seed, 30.0, 0.5, x0.numpy(),
                                   dirs.numpy() if alg == 0 else None, 0.1)
        ref.append(metrics.igd(torch.from_numpy(objs.T[:act].copy()).cuda(), front))
        ms_ref.append(ms / 500)
        kw = dict(population_size=N, max_generations=500, problem=cm.DTLZ2(12, 3), seed=seed, print_progress=False,
                  initial_population=x0,
                  crossover=cm.SBX(probability=1.0, eta_initial=30.0, eta_final=30.0, variable_copy_probability=0.5),
                  mutation=cm.PolynomialMutation(probability=1.0, eta_initial=20.0, eta_final=20.0))
        if alg == 0:
            kw["environment_selector"] = cm.NSGA3EnvironmentSelector(sparse_ratio=1.0)
            kw["reference_directions"] = cm.UserDefinedDirections(dirs.t().contiguous())
        else:
            kw["environment_selector"] = cm.RVEAEnvironmentSelector(alpha=2.0)
            kw["reference_directions"] = cm.AdaptiveRVEADirections(frequency=0.1)
        r = cm.Algorithm(name, **kw).run()
        ours.append(metrics.igd(r.objectives[: r.active_count], front))
        ms_ours.append(r.total_ms / 500)
    return ours, ref, ms_ours, ms_ref


@pytest.mark.parametrize("name", ["NSGA3", "RVEA"])
def test_final_igd_matches_reference_runs(name):
    seeds = int(os.environ.get("MOEA_QUALITY_SEEDS", "10"))
    ours, ref, ms_ours, ms_ref = _runs(name, seeds)
    mo, mr = statistics.mean(ours), statistics.mean(ref)
    so, sr = statistics.stdev(ours), statistics.stdev(ref)
    t = (mo - mr) / ((so ** 2 + sr ** 2) / seeds) ** 0.5
    print(f"\n{name}: {seeds} seeds  IGD product {mo:.6f} +- {so:.2e}  reference {mr:.6f} +- {sr:.2e}  "
          f"Welch t {t:+.2f}  ms/gen product {statistics.mean(ms_ours):.3f} reference {statistics.mean(ms_ref):.3f}")
    assert abs(t) < 4.0
