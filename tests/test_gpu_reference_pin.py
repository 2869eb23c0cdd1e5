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
