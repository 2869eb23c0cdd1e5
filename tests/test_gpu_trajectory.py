"""GPU: whole generations of the timed configurations, through the public API
and the captured CUDA graphs, against an independent composition of the same
generation.

- NSGA-III at the headline size (DTLZ1, M=3, D=7, N=32768, 32640 directions,
  graphs on, default association): each generation's offspring come from the
  product's reproduction kernel and the reference's DTLZ kernel, and the
  oracle's complete NSGA-III selection must reproduce the algorithm's next
  parents exactly (nsga3_environment_selector.cu:289-538).
- RVEA (DTLZ2, M=8, N=1024, adaptive directions) at D=17 and at D=131072: the
  whole generation is composed from the reference's own kernels (compiled from
  its sources into oracle/_ref): tournament-free random mating draws, SBX and
  polynomial mutation on the product's Philox draws, DTLZ2, translation,
  partition, APD, elitism, merge and survivor update with dead-slot sentinels,
  and the direction adaptation on the schedule of
  AdaptiveRVEADirections::update (reference_directions.cu:132-162).  Every
  value of the next population must be bit-identical.
"""
import math

import numpy as np
import pytest
import torch

import cuda_moea as cm
from oracle.ref import ref as R

import draws

pytestmark = pytest.mark.gpu
need_ref = pytest.mark.skipif(not R.available(), reason="oracle/_ref not built (needs the reference sources)")


def _bits(t: torch.Tensor) -> torch.Tensor:
    return t.contiguous().view(torch.int32)


@need_ref
def test_nsga3_headline_generations_with_graphs_match_oracle(oracle):
    from cuda_moea import stages
    N, D, M, seed = 32768, 7, 3, 2887
    algo = cm.NSGA3(population_size=N, max_generations=50, problem=cm.DTLZ1(D, M), seed=seed,
                    print_progress=False, use_graphs=True)
    algo.initialize()
    refs = algo.reference_directions.cpu().numpy().copy()
    assert refs.shape == (M, 32640)
    np.testing.assert_array_equal(refs, oracle.reference_directions(0, N, M))
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
    for g in range(3):
        off_x, _ = stages.reproduce(par_x, torch.from_numpy(par_cv).cuda(), rank, N, bounds, N,
                                    seed=dseed, generation=g)
        off_f, off_cv = R.problem_t(1, off_x, M)
        mix_f = np.concatenate([par_f, off_f.cpu().numpy()], 1)
        mix_cv = np.concatenate([par_cv, off_cv.cpu().numpy()])
        want = oracle.nsga3_select(mix_cv, mix_f, refs, dseed, offset, ideal)
        offset, ideal = want["offset"], want["ideal"]
        algo.step()
        assert algo.graph_info[0], "the headline generation must replay a CUDA graph"
        stats = algo.selection_stats()
        assert stats["max_front"] == want["max_front"]
        assert [stats[k] for k in ("N_prior", "N_last", "N_rem", "N_nds")] == list(want["sizes"])
        pop = algo.population
        surv = want["survivors"]
        mix_x = torch.cat([par_x, off_x])
        assert torch.equal(_bits(pop.variables), _bits(mix_x[torch.from_numpy(surv).cuda().long()]))
        np.testing.assert_array_equal(pop.objectives.t().cpu().numpy(), mix_f[:, surv])
        np.testing.assert_array_equal(pop.constraints.cpu().numpy(), mix_cv[surv])
        np.testing.assert_array_equal(algo.result().auxiliary_indices.cpu().numpy(), want["fronts"])
        par_x = pop.variables.clone()
        par_f = pop.objectives.t().contiguous().cpu().numpy()
        par_cv = pop.constraints.cpu().numpy().copy()
        rank = torch.from_numpy(want["fronts"]).cuda()


@need_ref
@pytest.mark.parametrize("D", [17, 131072])
def test_rvea_generations_match_reference_kernels(oracle, D):
    from cuda_moea import stages as st
    N, M, T, seed, freq, alpha = 1024, 8, 10, 31, 0.2, 2.0
    interval = max(1, int(math.floor(freq * T + 0.5)))  # std::lround of a positive value
    algo = cm.RVEA(population_size=N, max_generations=T, problem=cm.DTLZ2(D, M), seed=seed,
                   reference_directions=cm.AdaptiveRVEADirections(frequency=freq),
                   crossover=cm.SBX(30.0, 30.0, 1.0, 0.0), mutation=cm.PolynomialMutation(20.0, 20.0, 1.0),
                   print_progress=False)
    algo.initialize()
    refs0 = algo.reference_directions.cpu().numpy().copy()
    np.testing.assert_array_equal(refs0, R.directions(2, N, M))
    K = refs0.shape[1]
    refs = refs0.copy()
    gamma = R.rvea_gamma(refs)
    pop = algo.population
    par_x, par_f, par_cv = pop.variables.clone(), pop.objectives.t().contiguous(), pop.constraints.clone()
    active = N
    bounds = torch.tile(torch.tensor([0.0, 1.0]), (D,)).cuda()
    dseed = oracle.derive_seed(seed)
    adapted = 0
    for g in range(4):
        off_x, _ = draws.reference_reproduce(st, R, par_x, par_cv, None, active, bounds, N, mating=0,
                                             seed=dseed, generation=g, sbx_eta=30.0, sbx_prob=1.0,
                                             sbx_copy_prob=0.0, pm_eta=20.0, pm_prob=1.0)
        off_f, off_cv = R.problem_t(2, off_x, M)
        mix_f = torch.cat([par_f, off_f], 1).cpu().numpy()
        mix_cv = torch.cat([par_cv, off_cv]).cpu().numpy()
        t, _ = R.rvea_translate(mix_f)
        theta, idx = R.rvea_partition(t, refs, active, N)
        apd = R.rvea_apd(t, theta, gamma, idx, g + 1, T, alpha)
        sel, act = R.rvea_elitism(idx, mix_cv, apd, N, K)
        nx, nf, ncv = R.rvea_update_t(par_x, off_x, par_f, off_f, par_cv, off_cv,
                                      torch.from_numpy(sel).cuda(), act)
        del off_x
        if (g + 1) % interval == 0:
            refs = R.rvea_adapt(refs0, nf.cpu().numpy(), act)
            gamma = R.rvea_gamma(refs)
            adapted += 1
        algo.step()
        pop = algo.population
        assert algo.result().active_count == act
        assert torch.equal(_bits(pop.variables), _bits(nx)), f"variables differ at generation {g}"
        assert torch.equal(_bits(pop.objectives.t()), _bits(nf)), f"objectives differ at generation {g}"
        assert torch.equal(_bits(pop.constraints), _bits(ncv)), f"violations differ at generation {g}"
        np.testing.assert_array_equal(algo.reference_directions.cpu().numpy().view(np.uint32),
                                      refs.view(np.uint32))
        par_x, par_f, par_cv, active = nx, nf, ncv, act
        del nx
    assert adapted == 2
