"""GPU: IGD in FP64 against a numpy FP64 restatement of the reference metric
(tests/evaluation/metrics/igd.py: finite rows, optional non-dominated filter,
mean nearest distance), with NaN/inf rows, duplicates and dominated rows."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def igd_numpy(approx, ref, filter_nondominated=True):
    a = approx[np.isfinite(approx).all(1)].astype(np.float64)
    if filter_nondominated:
        no_worse = (a[:, None, :] <= a[None, :, :]).all(2)   # [p, q]: p no worse than q
        better = (a[:, None, :] < a[None, :, :]).any(2)
        dominated = (no_worse & better).any(0)
        a = a[~dominated]
    d = np.sqrt(((ref[:, None, :] - a[None, :, :]) ** 2).sum(2))
    return d.min(1).mean()


@pytest.mark.parametrize("M,n,r", [(2, 300, 101), (3, 1000, 496), (5, 700, 210), (8, 400, 120)])
@pytest.mark.parametrize("filt", [True, False])
def test_igd_fp64_matches_restatement(M, n, r, filt):
    from cuda_moea import metrics
    rng = np.random.default_rng(M * n)
    approx = (rng.random((n, M)) * 2).astype(np.float32)
    approx[:20] = approx[20:40]            # duplicates
    approx[40, 0] = np.nan
    approx[41, 1 % M] = np.inf
    ref = rng.random((r, M))
    got = metrics.igd(torch.from_numpy(approx), torch.from_numpy(ref), filter_nondominated=filt)
    want = igd_numpy(approx, ref, filt)
    assert abs(got - want) <= 1e-12 * max(1.0, abs(want))


def test_igd_of_converged_dtlz2_run():
    import cuda_moea as cm
    front = cm.metrics.dtlz_reference_front("DTLZ2", 3, 30)
    r = cm.NSGA3(population_size=92, max_generations=100, problem=cm.DTLZ2(12, 3), seed=2887,
                 print_progress=False).run()
    v = cm.metrics.igd(r.objectives, front)
    assert 0.0 < v < 0.08
    assert abs(v - igd_numpy(r.objectives.cpu().numpy(), front.numpy())) <= 1e-12


def test_igd_rejects_all_nonfinite():
    from cuda_moea import metrics
    from cuda_moea._lib import MoeaError
    with pytest.raises(MoeaError):
        metrics.igd(torch.full((5, 3), float("nan")), torch.rand(4, 3, dtype=torch.float64))


def test_igd_equals_reference_metric_on_golden_cases():
    """moea_igd against the reference's own igd() (tests/evaluation/metrics/
    igd.py:23-47), whose values on seeded approximations are recorded in
    tests/golden/quality_reference.json: non-finite rows dropped, with and
    without the non-dominated filter, FP64 (relative tolerance 1e-12)."""
    import json
    import sys
    from pathlib import Path
    from cuda_moea import metrics
    golden_dir = Path(__file__).resolve().parent / "golden"
    sys.path.insert(0, str(golden_dir))
    from quality_inputs import approximation
    cases = json.loads((golden_dir / "quality_reference.json").read_text())["igd"]
    for c in cases:
        x = torch.from_numpy(approximation(c["seed"], c["n"], c["objectives"])).cuda()
        ref = metrics.pareto_front_points("DTLZ2", c["objectives"], c["front_count"], 2887).to(torch.float64)
        got = metrics.igd(x, ref, filter_nondominated=c["filter_nondominated"])
        assert abs(got - c["igd"]) <= 1e-12 * abs(c["igd"]), (c, got)
