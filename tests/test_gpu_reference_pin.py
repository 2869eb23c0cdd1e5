"""GPU: the product's stages against CUDA-MOEA's own stage code
(oracle/_ref/libmoea_ref.so, built from the reference sources) on identical
inputs, and the oracle against the same outputs.

Both sides run on the same B200 with the same CUDA math library, so stages
that share a formula agree bit for bit: fronts, association, niching, every
DTLZ objective and constraint violation, the RVEA translation, partition,
gamma, APD and elitism.  The intercepts differ by the reference's FP32 SVD
against the product's FP64 solve (tolerance stated in the test).
"""
import numpy as np
import pytest
import torch

from oracle.ref import ref as R

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not R.available(), reason="oracle/_ref not built (needs the reference sources)")]


@pytest.fixture(scope="module")
def st():
    from cuda_moea import stages
    return stages


@pytest.fixture(scope="module")
def ws(st):
    w = st.Workspace(max_points=16384, max_objectives=16, max_directions=40000)
    yield w
    w.close()


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("M,N,kind", [(3, 2048, "dtlz1"), (3, 4096, "uniform"), (2, 1000, "ties"),
                                      (5, 1500, "uniform"), (8, 800, "ties")])
def test_ndsort_vs_reference(st, ws, oracle, M, N, kind):
    rng = np.random.default_rng(M * N)
    n = 2 * N
    if kind == "dtlz1":
        objs, _ = oracle.evaluate("DTLZ1", rng.random((n, M + 4)).astype(np.float32), M)
    elif kind == "ties":
        objs = rng.integers(0, 7, (M, n)).astype(np.float32)
    else:
        objs = rng.random((M, n)).astype(np.float32)
    cv = np.where(rng.random(n) < 0.25, rng.integers(1, 5, n) * 0.25, 0).astype(np.float32)
    ref_fr, ref_mf = R.ndsort(cv, objs, N)
    got, gmf = st.ndsort(ws, _t(cv), _t(objs), N)
    np.testing.assert_array_equal(got.cpu().numpy(), ref_fr)
    assert gmf == ref_mf
    o_fr, o_mf = oracle.ndsort(cv, objs, N)
    np.testing.assert_array_equal(o_fr, ref_fr)


# the reference supports at most 8 objectives (MAX_M, cuda_globals.cuh)
@pytest.mark.parametrize("M,n,N", [(3, 6000, 4096), (5, 3000, 2000), (8, 2000, 8000)])
def test_normalize_associate_vs_reference(st, ws, oracle, M, n, N):
    rng = np.random.default_rng(n + M)
    f = (rng.random((M, n)) * rng.random(n) * 5 + 0.05).astype(np.float32)
    ideal = f.min(1).astype(np.float32)
    ref_f, ref_rcp = R.normalize(f, ideal)
    got_f, got_rcp, _ = st.normalize(ws, _t(f), _t(ideal))
    np.testing.assert_allclose(got_rcp.cpu().numpy(), ref_rcp, rtol=2e-5)
    np.testing.assert_allclose(got_f.cpu().numpy(), ref_f, rtol=2e-5, atol=1e-7)
    refs = oracle.reference_directions(0, N, M)
    # association on the reference's normalised values: identical formula
    ri, rd = R.associate(ref_f, refs)
    gi, gd = st.associate(ws, _t(ref_f), _t(refs))
    np.testing.assert_array_equal(gi.cpu().numpy(), ri)
    np.testing.assert_array_equal(gd.cpu().numpy(), rd)


def test_niching_vs_reference(st, ws):
    rng = np.random.default_rng(99)
    N, H = 2000, 500
    for np_, nl in [(1200, 1500), (0, 4000), (1999, 3)]:
        nds = np_ + nl
        gidx = rng.permutation(2 * N)[:nds].astype(np.int32)
        idx = rng.integers(0, H, nds).astype(np.int32)
        dist = (rng.integers(0, 60, nds) / 11.0).astype(np.float32)
        sizes = np.array([np_, nl, N - np_, nds], np.int32)
        rs, ro = R.niching(555, 1000, gidx, dist, idx, sizes, H, N)
        gs, go = st.niching(ws, 555, 1000, _t(gidx), _t(dist), _t(idx), _t(sizes), H, N)
        assert go == ro
        np.testing.assert_array_equal(gs.cpu().numpy(), rs)


PROBLEMS = [(1, 7, 3), (2, 12, 3), (3, 12, 3), (4, 12, 3), (5, 12, 3), (6, 12, 3), (7, 22, 3),
            (8, 12, 3), (2, 17, 8), (9, 14, 8), (10, 12, 3), (11, 12, 3), (12, 12, 3), (13, 12, 3),
            (14, 14, 8), (15, 7, 3), (2, 1000, 3), (1, 3000, 5), (7, 700, 4)]


@pytest.mark.parametrize("kind,D,M", PROBLEMS)
def test_problem_bit_exact_vs_reference(st, kind, D, M):
    rng = np.random.default_rng(kind * 100 + D)
    N = 257
    if kind == 15:
        lo = np.array([0.5, 0.45, 0.5, 0.5, 0.875, 0.4, 0.4], np.float32)
        hi = np.array([1.5, 1.35, 1.5, 1.5, 2.625, 1.2, 1.2], np.float32)
        x = (lo + rng.random((N, D)) * (hi - lo)).astype(np.float32)
    else:
        x = rng.random((N, D)).astype(np.float32)
        x[:4] = 0.5
    rf, rcv = R.problem(kind, x, M)
    gf, gcv = st.problem_evaluate(kind, _t(x), M)
    np.testing.assert_array_equal(gf.cpu().numpy(), rf)
    np.testing.assert_array_equal(gcv.cpu().numpy(), rcv)


def test_rvea_vs_reference(st, ws, oracle):
    rng = np.random.default_rng(3)
    M, N = 8, 1024
    n = 2 * N
    objs = (rng.random((M, n)) + 0.1).astype(np.float32)
    objs[:, 900:N] = 1e15
    cv = np.where(rng.random(n) < 0.1, rng.random(n), 0).astype(np.float32)
    refs = oracle.reference_directions(2, N, M)
    rt, rz = R.rvea_translate(objs)
    gt, gz = st.rvea_translate(ws, _t(objs))
    np.testing.assert_array_equal(gt.cpu().numpy(), rt)
    rth, ridx = R.rvea_partition(rt, refs, 900, N)
    gth, gidx = st.rvea_partition(ws, _t(rt), _t(refs), 900, N)
    np.testing.assert_array_equal(gidx.cpu().numpy(), ridx)
    np.testing.assert_array_equal(gth.cpu().numpy(), rth)
    rg = R.rvea_gamma(refs)
    np.testing.assert_array_equal(st.rvea_gamma(ws, _t(refs)).cpu().numpy(), rg)
    for gen in (1, 37, 100):
        ra = R.rvea_apd(rt, rth, rg, ridx, gen, 100, 2.0)
        ga = st.rvea_apd(ws, _t(rt), _t(rth), _t(rg), _t(ridx), gen, 100, 2.0)
        np.testing.assert_array_equal(ga.cpu().numpy(), ra)
    rs, ra_ = R.rvea_elitism(ridx, cv, ra, N, refs.shape[1])
    gs, ga_ = st.rvea_elitism(ws, _t(ridx), _t(cv), _t(ra), N, refs.shape[1])
    assert ga_ == ra_
    np.testing.assert_array_equal(gs.cpu().numpy(), rs)


# ---------------------------------------------------------------- reproduction
def test_tournament_sbx_pm_bit_exact_vs_reference(st):
    """The explicit-draw stages against the reference's own kernels
    (mating_selection.cu:11-35, sbx_crossover.cu:20-70,
    polynomial_mutation.cu:20-60) on identical draws: same formula, same
    CUDA powf, so every bit agrees."""
    rng = np.random.default_rng(81)
    for n, D, lo, hi in [(257, 33, 0.0, 1.0), (1000, 7, -5.0, 5.0), (64, 1025, -1.0, 3.0)]:
        parents = (lo + rng.random((n, D)) * (hi - lo)).astype(np.float32)
        bounds = np.tile([lo, hi], D).astype(np.float32)
        cv = np.where(rng.random(n) < 0.3, rng.integers(0, 4, n) * 0.5, 0).astype(np.float32)
        rank = rng.integers(0, 5, n).astype(np.int32)
        cand = rng.integers(0, n, (n, 2)).astype(np.int32)
        w_r = R.tournament(cand, rank, cv)
        np.testing.assert_array_equal(st.tournament(_t(cand), _t(rank), _t(cv)).cpu().numpy(), w_r)
        pairs = n // 2
        u = rng.random((pairs * D, 2)).astype(np.float32)
        u[:7, 0] = [0.0, 0.5, 0.49999997, 0.99999994, 0.25, 0.75, 1e-7]
        sign = rng.integers(0, 2, pairs * D).astype(np.int32)
        copy = rng.random(pairs * D).astype(np.float32)
        for eta, prob, cp in [(30.0, 1.0, 0.0), (30.0, 0.9, 0.5), (2.0, 0.7, 0.2), (100.0, 1.0, 1.0)]:
            o_r = R.sbx(parents, w_r, bounds, u, sign, copy, eta, prob, cp, n)
            o_g = st.sbx(_t(parents), _t(w_r), _t(bounds), _t(u), _t(sign), _t(copy), eta, prob, cp, n)
            np.testing.assert_array_equal(o_g.cpu().numpy().view(np.uint32), o_r.view(np.uint32))
        um = rng.random((n * D, 2)).astype(np.float32)
        um[:, 0] *= 0.2 / D * rng.integers(0, 2, n * D)  # about half the values mutate
        um[:5, 1] = [0.0, 0.5, 0.50000006, 0.99999994, 0.25]
        for eta, prob in [(20.0, 1.0), (5.0, 0.5)]:
            m_r = R.pm(o_r, bounds, um, eta, prob)
            m_g = st.pm(_t(o_r), _t(bounds), _t(um), eta, prob)
            np.testing.assert_array_equal(m_g.cpu().numpy().view(np.uint32), m_r.view(np.uint32))


def test_annealed_index_vs_reference(oracle):
    """The host-side annealing of the SBX/PM distribution index
    (sbx_crossover.cu:12-18): the oracle's restatement against the
    reference's function."""
    for b, e, g, t in [(30.0, 30.0, 0, 100), (5.0, 40.0, 37, 100), (40.0, 5.0, 99, 100),
                       (20.0, 3.0, 150, 100), (10.0, 20.0, 3, 0), (7.5, 1.25, 1, 3)]:
        assert np.float32(oracle.annealed(b, e, g, t)) == np.float32(R.annealed(b, e, g, t))


def test_quantize_cv_bit_exact_vs_reference(st, oracle):
    """Optional CV quantisation (cv_quantization.cu:11-95): product and
    oracle against the reference's kernel, linear and log mappings."""
    rng = np.random.default_rng(4)
    cv = (rng.random(5000) * 3).astype(np.float32)
    cv[:500] = 0.0
    cv[500:505] = -0.0
    cv[505:510] = np.nan
    cv[510:515] = [1e-4, 2.5, 3.0, 1e30, -1.0]
    for eps, clip, la, bins in [(0.0, 2.0, 0.0, 16), (1e-3, 2.5, 3.0, 64), (0.0, 10.0, 0.5, 1000)]:
        want = R.quantize_cv(cv, eps, clip, la, bins)
        got = st.quantize_cv(_t(cv), eps, clip, la, bins).cpu().numpy()
        np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))
        o = oracle.quantize_cv(cv, eps, clip, la, bins)
        if la == 0.0:
            np.testing.assert_array_equal(o.view(np.uint32), want.view(np.uint32))
        else:  # the host log1pf differs from CUDA's by an ulp near bin edges
            assert (o != want).mean() < 1e-3


def test_rvea_adapt_bit_exact_vs_reference(st, ws, oracle):
    """Direction adaptation (rvea_reference_adaptation.cu:279-317), called as
    AdaptiveRVEADirections::update calls it, on populations with dead slots,
    a degenerate (zero-range) objective and non-finite rows."""
    rng = np.random.default_rng(17)
    for M, N, active in [(8, 1024, 900), (3, 92, 92), (5, 500, 1)]:
        v0 = oracle.reference_directions(2, N, M)
        objs = (rng.random((M, N)) * rng.random(M)[:, None] * 4).astype(np.float32)
        objs[:, active:] = 1e15
        objs[M - 1, :] = 0.25  # zero range in the last objective
        want = R.rvea_adapt(v0, objs, active)
        got = st.rvea_adapt(ws, _t(v0), _t(objs), active).cpu().numpy()
        np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))
        np.testing.assert_allclose(oracle.rvea_adapt(v0, objs, active), want, rtol=3e-6, atol=3e-7)


def test_fused_reproduction_bit_exact_vs_reference_kernels(st):
    """The product's fused Philox reproduction (mating, SBX, PM in one pass)
    against the reference's kernels fed with the same draws, regenerated from
    the product's Philox stream: tournament and random mating, odd
    populations, copy probability, every value bit for bit."""
    import draws
    rng = np.random.default_rng(5)
    for n, D, mating, cp, seed, gen in [(300, 13, 1, 0.0, 2024, 5), (301, 7, 1, 0.5, 7, 0),
                                        (128, 4099, 0, 0.5, 99, 41)]:
        parents = _t(rng.random((n, D)).astype(np.float32))
        bounds = _t(np.tile([0.0, 1.0], D).astype(np.float32))
        cv = _t(np.where(rng.random(n) < 0.2, rng.random(n), 0).astype(np.float32))
        rank = _t(rng.integers(0, 4, n).astype(np.int32))
        active = n - 3 if mating == 0 else n
        off_g, pidx_g = st.reproduce(parents, cv, rank, active, bounds, n, mating=mating, seed=seed,
                                     generation=gen, sbx_prob=0.9, sbx_copy_prob=cp)
        off_r, pidx_r = draws.reference_reproduce(st, R, parents, cv, rank, active, bounds, n, mating=mating,
                                                  seed=seed, generation=gen, sbx_eta=30.0, sbx_prob=0.9,
                                                  sbx_copy_prob=cp, pm_eta=20.0, pm_prob=1.0)
        assert torch.equal(pidx_g, pidx_r)
        assert torch.equal(off_g.view(torch.int32), off_r.view(torch.int32))
