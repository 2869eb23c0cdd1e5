"""Parity of the CUDA stages (called through libmoea_b200's C ABI) with the
oracle on identical seeded inputs.

Integer work (fronts, sizes, compaction, association indices, niching and
elitism selections, tournament winners, random draws) must match bit for bit.
FP32 values match bit for bit where both sides use the same formula and
correctly rounded operations (association distances, normalised objectives);
where the GPU calls CUDA's transcendental functions (powf in SBX/PM, cosf/sinf
in DTLZ, rsqrtf/acosf in RVEA) the tolerance is stated per test.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


@pytest.fixture(scope="module")
def st():
    from cuda_moea import stages
    return stages


@pytest.fixture(scope="module")
def ws(st):
    w = st.Workspace(max_points=16384, max_objectives=16, max_directions=40000)
    yield w
    w.close()


def _t(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.to(DEV)


def _population(rng, M, n, kind):
    """Synthetic objective matrices with the edge cases of the domain."""
    if kind == "uniform":
        objs = rng.random((M, n)).astype(np.float32)
    elif kind == "ties":
        objs = rng.integers(0, 5, size=(M, n)).astype(np.float32)
    elif kind == "dtlz1":
        x = rng.random((n, M + 4)).astype(np.float32)
        from oracle import oracle as O
        objs, _ = O.evaluate("DTLZ1", x, M)
    elif kind == "correlated":
        base = rng.random(n).astype(np.float32)
        objs = (base[None, :] + 0.05 * rng.random((M, n))).astype(np.float32)
    else:
        raise ValueError(kind)
    return objs


def _cv(rng, n, mode):
    if mode == "feasible":
        return np.zeros(n, np.float32)
    cv = np.where(rng.random(n) < 0.35, rng.integers(1, 4, n).astype(np.float32) * 0.5, 0.0)
    cv = cv.astype(np.float32)
    if mode == "nan":
        cv[rng.integers(0, n, 3)] = np.nan
    if mode == "negzero":
        cv[rng.integers(0, n, 5)] = -0.0
    if mode in ("mostly_infeasible", "all_infeasible"):
        # distinct and repeated violations: one front per violation value
        share = 0.9 if mode == "mostly_infeasible" else 1.0
        cv = np.where(rng.random(n) < share, rng.integers(1, n // 3 + 2, n).astype(np.float32) * 0.125, 0.0)
        cv = cv.astype(np.float32)
        cv[rng.integers(0, n, 4)] = np.nan
    return cv


CASES = [(1, 64, "uniform", "feasible"), (2, 184, "ties", "mixed"), (3, 184, "uniform", "feasible"),
         (3, 2048, "dtlz1", "feasible"), (3, 2048, "ties", "mixed"), (3, 4097, "correlated", "feasible"),
         (5, 1500, "ties", "nan"), (8, 1024, "uniform", "mixed"), (10, 3000, "uniform", "negzero"),
         (16, 700, "ties", "feasible"), (3, 8, "uniform", "feasible"), (3, 33, "ties", "mixed"),
         (3, 4096, "uniform", "mostly_infeasible"), (10, 3000, "ties", "all_infeasible"),
         (3, 16000, "dtlz1", "mostly_infeasible"), (2, 97, "uniform", "all_infeasible")]


@pytest.mark.parametrize("M,n,kind,cvmode", CASES)
def test_ndsort_fronts_bit_exact(st, ws, oracle, M, n, kind, cvmode):
    rng = np.random.default_rng(M * 1000 + n)
    objs = _population(rng, M, n, kind)
    if cvmode == "nan" or kind == "ties":
        objs[rng.integers(0, M), rng.integers(0, n, 2)] = np.nan
    cv = _cv(rng, n, cvmode)
    for target in (max(1, n // 2), n):
        want, wmf = oracle.ndsort(cv, objs, target)
        got, gmf = st.ndsort(ws, _t(cv), _t(objs), target)
        np.testing.assert_array_equal(got.cpu().numpy(), want)
        assert gmf == wmf


@pytest.mark.parametrize("M,n,feasible_share", [(3, 65536, 1.0), (5, 40000, 0.7)])
def test_ndsort_full_size_many_fronts(st, oracle, M, n, feasible_share):
    """Full-size sorts with dozens of thin fronts: points near the DTLZ1 front
    (g small), so rows are thousands of words long and every peel front
    queues hundreds of row scans per CTA.  Three GPU runs against the oracle:
    the peel's CTAs race only in timing, never in the result."""
    rng = np.random.default_rng(n + M)
    x = rng.random((n, M + 4)).astype(np.float32)
    x[:, M - 1:] = (0.5 + 0.02 * rng.standard_normal((n, 5))).astype(np.float32)
    objs, _ = oracle.evaluate("DTLZ1", x, M)
    cv = np.where(rng.random(n) < feasible_share, 0.0, rng.random(n) * 2.0).astype(np.float32)
    target = n // 2
    want, wmf = oracle.ndsort(cv, objs, target)
    assert wmf >= 10  # many fronts, or the test exercises nothing
    w = st.Workspace(max_points=n, max_objectives=M, max_directions=1)
    try:
        for _ in range(3):
            got, gmf = st.ndsort(w, _t(cv), _t(objs), target)
            np.testing.assert_array_equal(got.cpu().numpy(), want)
            assert gmf == wmf
    finally:
        w.close()


@pytest.mark.parametrize("M,n,kind,cvmode", [(3, 65536, "dtlz1-thin", "feasible"), (5, 40000, "dtlz1-thin", "mixed"),
                                            (3, 16000, "dtlz1", "mostly_infeasible"), (8, 1024, "uniform", "mixed"),
                                            (3, 900, "ties", "nan"), (2, 97, "uniform", "all_infeasible")])
def test_ndsort_general_and_lane_owned_peels_agree(st, oracle, M, n, kind, cvmode):
    """The two peel kernels (the lane-owned one, default up to 151,552 points,
    and the general one beyond) give the same fronts as the oracle on the same
    inputs, from thin-front full-size sorts down to single-CTA grids."""
    rng = np.random.default_rng(n * 7 + M)
    if kind == "dtlz1-thin":
        x = rng.random((n, M + 4)).astype(np.float32)
        x[:, M - 1:] = (0.5 + 0.02 * rng.standard_normal((n, 5))).astype(np.float32)
        objs, _ = oracle.evaluate("DTLZ1", x, M)
    else:
        objs = _population(rng, M, n, kind)
    if cvmode == "nan":
        objs[rng.integers(0, M), rng.integers(0, n, 2)] = np.nan
    cv = _cv(rng, n, cvmode)
    target = max(1, n // 2)
    want, wmf = oracle.ndsort(cv, objs, target)
    w = st.Workspace(max_points=n, max_objectives=M, max_directions=1)
    try:
        for general in (False, True, False):
            w.set_peel(general)
            got, gmf = st.ndsort(w, _t(cv), _t(objs), target)
            np.testing.assert_array_equal(got.cpu().numpy(), want)
            assert gmf == wmf
    finally:
        w.close()


@pytest.mark.parametrize("M,n,kind,cvmode", [(2, 97, "uniform", "feasible"), (3, 65536, "dtlz1-thin", "feasible"),
                                            (3, 5000, "ties", "nan"), (4, 3001, "correlated", "mixed"),
                                            (5, 40000, "dtlz1-thin", "mixed"), (8, 10000, "uniform", "negzero"),
                                            (9, 4099, "uniform", "mixed"), (10, 16384, "dtlz1", "mostly_infeasible"),
                                            (12, 257, "ties", "feasible"), (16, 2000, "correlated", "feasible"),
                                            (3, 3, "uniform", "feasible"), (3, 1, "uniform", "feasible"),
                                            (4, 2, "ties", "feasible"), (7, 129, "ties", "all_infeasible")])
def test_ndsort_block_and_word_tiles_agree(st, oracle, M, n, kind, cvmode):
    """The two dominance-row kernels (block prefix sets with search trees, the
    default, and the per-word tables) give the oracle's fronts on the same
    inputs: block sizes 256 (M <= 4) and 128 (M >= 5), ragged last blocks,
    ties, NaN objectives and violations, infeasible majorities."""
    rng = np.random.default_rng(n * 11 + M)
    if kind == "dtlz1-thin":
        x = rng.random((n, M + 4)).astype(np.float32)
        x[:, M - 1:] = (0.5 + 0.02 * rng.standard_normal((n, 5))).astype(np.float32)
        objs, _ = oracle.evaluate("DTLZ1", x, M)
    else:
        objs = _population(rng, M, n, kind)
    if cvmode == "nan":
        objs[rng.integers(0, M), rng.integers(0, n, 2)] = np.nan
    cv = _cv(rng, n, cvmode)
    target = max(1, n // 2)
    want, wmf = oracle.ndsort(cv, objs, target)
    w = st.Workspace(max_points=max(n, 2), max_objectives=M, max_directions=1)
    try:
        for word in (False, True, False):
            w.set_tiles(word)
            got, gmf = st.ndsort(w, _t(cv), _t(objs), target)
            np.testing.assert_array_equal(got.cpu().numpy(), want)
            assert gmf == wmf
    finally:
        w.close()


def test_ndsort_all_mutually_nondominated(st, ws, oracle):
    # points on a line f1 = 1 - f0: no dominance pair at all (the reference's
    # CSR queue path leaves every front at -1 in this case; the relation gives front 0)
    n = 1000
    f0 = np.linspace(0, 1, n, dtype=np.float32)
    objs = np.stack([f0, 1 - f0]).astype(np.float32)
    cv = np.zeros(n, np.float32)
    got, gmf = st.ndsort(ws, _t(cv), _t(objs), n // 2)
    assert gmf == 0 and (got.cpu().numpy() == 0).all()


def test_extract_ideal_normalize_associate(st, ws, oracle):
    rng = np.random.default_rng(11)
    M, n, N = 3, 4000, 2000
    objs = _population(rng, M, n, "dtlz1")
    cv = np.zeros(n, np.float32)
    fronts, mf = oracle.ndsort(cv, objs, N)
    gidx_w, sizes_w = oracle.nds_extract(fronts, mf, N)
    gidx_g, sizes_g = st.nds_extract(ws, _t(fronts), mf, N)
    np.testing.assert_array_equal(sizes_g.cpu().numpy(), sizes_w)
    np.testing.assert_array_equal(gidx_g.cpu().numpy()[: sizes_w[3]], gidx_w)
    ideal_w = oracle.ideal_point(objs)
    np.testing.assert_array_equal(st.ideal_point(ws, _t(objs)).cpu().numpy(), ideal_w)
    nds = objs[:, gidx_w].copy()
    f_w, rcp_w, ext_w, ill = oracle.normalize(nds, ideal_w)
    f_g, rcp_g, ext_g = st.normalize(ws, _t(nds), _t(ideal_w))
    np.testing.assert_array_equal(ext_g.cpu().numpy(), ext_w)
    # FP64 solve on both sides, different summation order: equal up to 1 ulp
    np.testing.assert_allclose(rcp_g.cpu().numpy(), rcp_w, rtol=2.5e-7)
    if np.array_equal(rcp_g.cpu().numpy(), rcp_w):
        np.testing.assert_array_equal(f_g.cpu().numpy(), f_w)
    refs = oracle.reference_directions(1, 40, 3)
    idx_w, dist_w = oracle.associate(f_w, refs)
    idx_g, dist_g = st.associate(ws, _t(f_w), _t(refs))
    np.testing.assert_array_equal(idx_g.cpu().numpy(), idx_w)
    np.testing.assert_array_equal(dist_g.cpu().numpy(), dist_w)


@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("M,n,H_mode", [(3, 3000, (1, 254)), (3, 500, (1, 12)), (5, 2000, (0, 3000)),
                                        (8, 1500, (0, 900)), (10, 1200, (0, 2000)), (2, 4096, (1, 999))])
def test_association_bit_exact(st, ws, oracle, M, n, H_mode, mode):
    rng = np.random.default_rng(M + n)
    refs = oracle.reference_directions(H_mode[0], H_mode[1], M)
    x = rng.random((M, n)).astype(np.float32) * rng.random(n).astype(np.float32) * 3
    x[:, :10] = refs[:, :10] * 2.0          # exactly on directions
    x[:, 10:14] = 0.0                       # at the ideal point: every distance is 0
    x[0, 14] = np.inf                       # non-finite point: no association
    idx_w, dist_w = oracle.associate(x, refs)
    idx_g, dist_g = st.associate(ws, _t(x), _t(refs), mode)
    np.testing.assert_array_equal(idx_g.cpu().numpy(), idx_w)
    np.testing.assert_array_equal(dist_g.cpu().numpy(), dist_w)


def _dirs(rng, kind, M, H):
    if kind == "random_unit":
        r = np.abs(rng.standard_normal((M, H))).astype(np.float32)
        return (r / np.sqrt((r.astype(np.float64) ** 2).sum(0))).astype(np.float32)
    if kind == "signed_unit":      # directions in every orthant, points too
        r = rng.standard_normal((M, H)).astype(np.float32)
        return (r / np.sqrt((r.astype(np.float64) ** 2).sum(0))).astype(np.float32)
    if kind == "non_unit":         # user directions left unnormalised: full re-score
        return (rng.random((M, H)) * 3 + 0.01).astype(np.float32)
    if kind == "duplicates":       # repeated directions: ties go to the smaller index
        base = rng.random((M, H // 4)).astype(np.float32) + 0.05
        base = (base / np.sqrt((base.astype(np.float64) ** 2).sum(0))).astype(np.float32)
        return np.ascontiguousarray(np.tile(base, 4)[:, rng.permutation(H)])
    raise ValueError(kind)


@pytest.mark.parametrize("M,H,n,kind", [(3, 4000, 3000, "random_unit"), (3, 2000, 2000, "signed_unit"),
                                        (4, 1500, 2000, "non_unit"), (3, 2048, 3000, "duplicates"),
                                        (1, 7, 100, "random_unit"), (2, 31, 500, "signed_unit"),
                                        (16, 600, 800, "random_unit"), (6, 5000, 1500, "duplicates")])
def test_association_tree_adversarial(st, ws, oracle, M, H, n, kind):
    """The cone-tree search against the full scan and the oracle on direction
    sets the Das-Dennis tests do not reach."""
    rng = np.random.default_rng(M * 1000 + H)
    refs = _dirs(rng, kind, M, H)
    if kind == "signed_unit":
        x = rng.standard_normal((M, n)).astype(np.float32)
    else:
        x = (rng.random((M, n)) * rng.random(n) * 2).astype(np.float32)
    k = min(16, H)
    x[:, :k] = refs[:, :k] * 1.5
    x[:, 16:20] = 0.0
    x[:, 20] = 1e-30
    x[:, 21] = 3e18
    x[1 % M, 22] = np.nan
    idx_w, dist_w = oracle.associate(x, refs)
    for mode in (0, 1, 2):
        idx_g, dist_g = st.associate(ws, _t(x), _t(refs), mode)
        np.testing.assert_array_equal(idx_g.cpu().numpy(), idx_w, err_msg=f"mode {mode}")
        np.testing.assert_array_equal(dist_g.cpu().numpy(), dist_w, err_msg=f"mode {mode}")


def test_association_tree_full_size(st, oracle):
    """M=3 with the 32640 Das-Dennis directions of 254 partitions (the bench
    workload's direction set), 16384 points: tree search == tensor-core
    search == full scan, and a sample against the oracle."""
    rng = np.random.default_rng(32640)
    refs = oracle.reference_directions(1, 254, 3)
    n = 16384
    x = (rng.random((3, n)) ** 2 * rng.random(n) * 4).astype(np.float32)
    w = st.Workspace(max_points=n, max_objectives=3, max_directions=refs.shape[1])
    try:
        a_i, a_d = st.associate(w, _t(x), _t(refs), 0)
        b_i, b_d = st.associate(w, _t(x), _t(refs), 1)
        c_i, c_d = st.associate(w, _t(x), _t(refs), 2)
    finally:
        w.close()
    np.testing.assert_array_equal(a_i.cpu().numpy(), b_i.cpu().numpy())
    np.testing.assert_array_equal(a_d.cpu().numpy(), b_d.cpu().numpy())
    np.testing.assert_array_equal(c_i.cpu().numpy(), b_i.cpu().numpy())
    np.testing.assert_array_equal(c_d.cpu().numpy(), b_d.cpu().numpy())
    sample = rng.choice(n, 512, replace=False)
    idx_w, dist_w = oracle.associate(np.ascontiguousarray(x[:, sample]), refs)
    np.testing.assert_array_equal(a_i.cpu().numpy()[sample], idx_w)
    np.testing.assert_array_equal(a_d.cpu().numpy()[sample], dist_w)


@pytest.mark.parametrize("M,n,H_mode,kind", [(3, 65536, (1, 254), "dtlz1"), (8, 16000, (1, 8), "uniform"),
                                             (10, 8192, (1, 6), "uniform"), (5, 20000, (1, 20), "cluster"),
                                             (3, 129, (1, 15), "uniform"), (16, 4000, (1, 3), "uniform")])
def test_association_tensor_equals_scan(st, oracle, M, n, H_mode, kind):
    """The tensor-core association (split TF32 dots, re-score within the error
    bound) against the FP32 full scan: identical indices and distances,
    including points on the bisector of two directions (exact ties) and
    points clustered around one direction; a sample against the oracle."""
    rng = np.random.default_rng(M * 7 + n)
    refs = oracle.reference_directions(H_mode[0], H_mode[1], M)
    H = refs.shape[1]
    if kind == "dtlz1":
        x = (rng.random((M, n)) ** 2 * rng.random(n) * 4).astype(np.float32)
    elif kind == "cluster":
        c = refs[:, H // 3:H // 3 + 1]
        x = (c * (1 + rng.random(n)) + 1e-4 * rng.standard_normal((M, n))).astype(np.float32)
    else:
        x = (rng.random((M, n)) * rng.random(n) * 2).astype(np.float32)
    pairs = min(64, n // 4, H - 1)
    a = rng.integers(0, H - 1, pairs)
    x[:, :pairs] = refs[:, a] + refs[:, a + 1]          # equidistant from two directions
    x[:, pairs:2 * pairs] = refs[:, a] * 3.0             # on a direction
    w = st.Workspace(max_points=n, max_objectives=M, max_directions=H)
    try:
        s_i, s_d = st.associate(w, _t(x), _t(refs), 1)
        t_i, t_d = st.associate(w, _t(x), _t(refs), 2)
        t2_i, t2_d = st.associate(w, _t(x), _t(refs), 2)
    finally:
        w.close()
    np.testing.assert_array_equal(t_i.cpu().numpy(), s_i.cpu().numpy())
    np.testing.assert_array_equal(t_d.cpu().numpy(), s_d.cpu().numpy())
    np.testing.assert_array_equal(t2_i.cpu().numpy(), t_i.cpu().numpy())
    sample = np.concatenate([np.arange(min(n, 2 * pairs)), rng.choice(n, min(n, 256), replace=False)])
    idx_w, dist_w = oracle.associate(np.ascontiguousarray(x[:, sample]), refs)
    np.testing.assert_array_equal(t_i.cpu().numpy()[sample], idx_w)
    np.testing.assert_array_equal(t_d.cpu().numpy()[sample], dist_w)


def test_niching_bit_exact(st, ws, oracle):
    rng = np.random.default_rng(5)
    N, H = 1000, 200
    for np_, nl in [(0, 2000), (600, 900), (999, 5), (400, 600)]:
        nds = np_ + nl
        gidx = rng.permutation(2 * N)[:nds].astype(np.int32)
        idx = rng.integers(0, H, nds).astype(np.int32)
        dist = (rng.integers(0, 50, nds) / 7.0).astype(np.float32)  # many equal distances
        sizes = np.array([np_, nl, N - np_, nds], np.int32)
        sel_w, off_w = oracle.niching(2887, 77, gidx, dist, idx, sizes, H, N)
        sel_g, off_g = st.niching(ws, 2887, 77, _t(gidx), _t(dist), _t(idx), _t(sizes), H, N)
        assert off_g == off_w
        np.testing.assert_array_equal(sel_g.cpu().numpy(), sel_w)


@pytest.mark.parametrize("np_,nl,N,H,ties", [
    (0, 65536, 32768, 32640, False),    # the whole merged population in the last front
    (31000, 1800, 32768, 32640, False),  # a typical headline generation
    (20000, 45536, 32768, 500, True),    # large niches, many equal distances
    (32767, 1, 32768, 91, False),        # one member
    (0, 4097, 2100, 7, True),            # uneven slices, few directions
])
def test_niching_large_last_front(st, oracle, np_, nl, N, H, ties):
    """The last front's three stable sorts at the merged sizes of the
    headline workload (up to 65536 members), against the oracle."""
    rng = np.random.default_rng(nl + H)
    ws_big = st.Workspace(2 * N, 3, H)
    try:
        nds = np_ + nl
        gidx = rng.permutation(2 * N)[:nds].astype(np.int32)
        idx = rng.integers(0, H, nds).astype(np.int32)
        idx[rng.integers(0, nds, 3)] = -1  # members without a direction sort last
        if ties:
            dist = (rng.integers(0, 9, nds) / 3.0).astype(np.float32)
        else:
            dist = rng.random(nds).astype(np.float32)
        sizes = np.array([np_, nl, N - np_, nds], np.int32)
        for offset in (0, 123456789):
            sel_w, off_w = oracle.niching(2887, offset, gidx, dist, idx, sizes, H, N)
            sel_g, off_g = st.niching(ws_big, 2887, offset, _t(gidx), _t(dist), _t(idx), _t(sizes), H, N)
            assert off_g == off_w
            np.testing.assert_array_equal(sel_g.cpu().numpy(), sel_w)
    finally:
        ws_big.close()


@pytest.mark.parametrize("seed,M,N,kind", [(0, 3, 92, "dtlz1"), (1, 3, 1024, "dtlz1"),
                                           (2, 3, 2048, "uniform"), (3, 5, 600, "ties"),
                                           (4, 8, 512, "uniform"), (5, 3, 4096, "correlated")])
@pytest.mark.parametrize("assoc_mode", [0, 1, 2])
def test_nsga3_select_bit_exact(st, ws, oracle, seed, M, N, kind, assoc_mode):
    rng = np.random.default_rng(seed)
    objs = _population(rng, M, 2 * N, kind)
    cv = _cv(rng, 2 * N, "mixed" if seed % 2 else "feasible")
    refs = oracle.reference_directions(0, N, M)
    ideal = np.full(M, np.inf, np.float32)
    ideal = np.minimum(ideal, objs[:, :N].min(1))
    want = oracle.nsga3_select(cv, objs, refs, 12345, 9, ideal)
    got = st.nsga3_select(ws, _t(cv), _t(objs), _t(refs), 12345, 9, _t(ideal), assoc_mode)
    np.testing.assert_array_equal(got["sizes"].cpu().numpy(), want["sizes"])
    np.testing.assert_array_equal(got["survivors"].cpu().numpy(), want["survivors"])
    np.testing.assert_array_equal(got["fronts"].cpu().numpy(), want["fronts"])
    np.testing.assert_array_equal(got["ideal"].cpu().numpy(), want["ideal"])
    assert got["offset"] == want["offset"]


def test_rng_blocks_match_oracle_philox(st, oracle):
    for gen, tag, count in [(0, 1, 1000), (17, 3, 4099), (123456, 4, 77)]:
        got = st.rng_blocks(987654321, gen, tag, count).cpu().numpy().view(np.uint32)
        want = oracle.philox_stream(987654321, gen, tag, count)
        np.testing.assert_array_equal(got, want)


def test_tournament_sbx_pm_explicit_draws(st, oracle):
    rng = np.random.default_rng(8)
    n, D = 257, 33
    parents = rng.random((n, D)).astype(np.float32)
    bounds = np.tile([0.0, 1.0], D).astype(np.float32)
    cv = np.where(rng.random(n) < 0.3, rng.random(n), 0).astype(np.float32)
    rank = rng.integers(0, 5, n).astype(np.int32)
    cand = rng.integers(0, n, (n, 2)).astype(np.int32)
    w_w = oracle.tournament(cand, rank, cv)
    w_g = st.tournament(_t(cand), _t(rank), _t(cv))
    np.testing.assert_array_equal(w_g.cpu().numpy(), w_w)
    pairs = n // 2
    u = rng.random((pairs * D, 2)).astype(np.float32)
    sign = rng.integers(0, 2, pairs * D).astype(np.int32)
    copy = rng.random(pairs * D).astype(np.float32)
    for cp in (0.0, 0.5):
        o_w = oracle.sbx(parents, w_w, bounds, u, sign, copy, 30.0, 0.9, cp, n)
        o_g = st.sbx(_t(parents), _t(w_w), _t(bounds), _t(u), _t(sign), _t(copy), 30.0, 0.9, cp, n)
        # powf differs by a few ulp between CUDA and the host libm
        np.testing.assert_allclose(o_g.cpu().numpy(), o_w, rtol=2e-6, atol=2e-7)
    um = rng.random((n * D, 2)).astype(np.float32)
    um[:, 0] *= 0.05  # mutate often
    m_w = oracle.pm(o_w, bounds, um, 20.0, 1.0)
    m_g = st.pm(_t(o_w), _t(bounds), _t(um), 20.0, 1.0)
    np.testing.assert_allclose(m_g.cpu().numpy(), m_w, rtol=5e-6, atol=5e-7)


def test_fused_reproduce_matches_composed_oracle(st, oracle):
    """The fused Philox reproduction against the oracle's tournament, SBX and
    PM fed with the oracle's own Philox stream in the product's draw layout
    (stated in tests/draws.py); tolerance for the host powf."""
    import draws
    rng = np.random.default_rng(9)
    for n, D, seed, gen, sbx_prob, copy_prob, pm_prob in [(300, 13, 2024, 5, 0.9, 0.0, 1.0),
                                                          (301, 3, 77, 2, 1.0, 0.5, 1.0),
                                                          (64, 8, 5, 1, 1.0, 0.0, 8.0)]:
        parents = rng.random((n, D)).astype(np.float32)
        bounds = np.tile([0.0, 1.0], D).astype(np.float32)
        cv = np.where(rng.random(n) < 0.2, rng.random(n), 0).astype(np.float32)
        rank = rng.integers(0, 4, n).astype(np.int32)
        off_g, pidx_g = st.reproduce(_t(parents), _t(cv), _t(rank), n, _t(bounds), n, seed=seed,
                                     generation=gen, sbx_prob=sbx_prob, sbx_copy_prob=copy_prob, pm_prob=pm_prob)
        cand = draws.mating_candidates_np(oracle, seed, gen, n, n)
        pidx_w = oracle.tournament(cand, rank, cv)
        np.testing.assert_array_equal(pidx_g.cpu().numpy(), pidx_w)
        u, sign, copy = draws.crossover_draws_np(oracle, seed, gen, n, D, sbx_prob, copy_prob)
        off_w = oracle.sbx(parents, pidx_w, bounds, u, sign, copy, 30.0, sbx_prob, copy_prob, n)
        um = draws.mutation_draws_np(oracle, seed, gen, n, D, pm_prob)
        off_w = oracle.pm(off_w, bounds, um, 20.0, pm_prob)
        np.testing.assert_allclose(off_g.cpu().numpy(), off_w, rtol=5e-6, atol=5e-7)


PROBLEMS = [("DTLZ1", 7, 3), ("DTLZ2", 12, 3), ("DTLZ3", 12, 3), ("DTLZ4", 12, 3), ("DTLZ5", 12, 3),
            ("DTLZ6", 12, 3), ("DTLZ7", 22, 3), ("ConvexDTLZ2", 12, 3), ("DTLZ2", 17, 8),
            ("C1DTLZ1", 14, 10), ("C3DTLZ4", 14, 10), ("C1DTLZ3", 12, 3), ("C2DTLZ2", 12, 3),
            ("C2ConvexDTLZ2", 12, 3), ("C3DTLZ1", 12, 3), ("CSDP", 7, 3), ("DTLZ2", 700, 3),
            ("DTLZ1", 600, 5)]


@pytest.mark.parametrize("kind,D,M", PROBLEMS)
def test_problem_objectives(st, oracle, kind, D, M):
    from cuda_moea.problem import PROBLEM_KINDS
    rng = np.random.default_rng(D * 31 + M)
    N = 333
    if kind == "CSDP":
        lo = np.array([0.5, 0.45, 0.5, 0.5, 0.875, 0.4, 0.4], np.float32)
        hi = np.array([1.5, 1.35, 1.5, 1.5, 2.625, 1.2, 1.2], np.float32)
        x = (lo + rng.random((N, D)) * (hi - lo)).astype(np.float32)
    else:
        x = rng.random((N, D)).astype(np.float32)
        x[:5, :] = 0.5   # g == 0 rows (DTLZ1/3 cancellation)
        x[5:8, :M] = 0.0
        x[8:10, :M] = 1.0
    f_g, cv_g = st.problem_evaluate(PROBLEM_KINDS[kind], _t(x), M)
    f_g, cv_g = f_g.cpu().numpy(), cv_g.cpu().numpy()
    f32, c32 = oracle.evaluate(kind, x, M, 0)
    f64, c64 = oracle.evaluate(kind, x, M, 1)
    # same expression shapes and reduction order: agreement limited by CUDA's
    # cosf/sinf/powf (and __cosf/__sinf in DTLZ5) against the host libm
    scale = np.maximum(np.abs(f32), 1.0)
    tol = 2e-5 if kind in ("DTLZ5", "DTLZ6") else 4e-6
    assert (np.abs(f_g - f32) / scale).max() <= tol
    # error against the FP64 evaluation, stated bound
    assert (np.abs(f_g - f64) / np.maximum(np.abs(f64), 1.0)).max() <= (2e-4 if kind == "DTLZ6" else 3e-5)
    np.testing.assert_allclose(cv_g, c32, rtol=1e-5, atol=1e-5)


def test_rvea_stages(st, ws, oracle):
    rng = np.random.default_rng(21)
    M, N = 8, 512
    n = 2 * N
    objs = rng.random((M, n)).astype(np.float32) + 0.1
    active = 450
    objs[:, active:N] = 1e15
    cv = np.where(rng.random(n) < 0.1, rng.random(n), 0).astype(np.float32)
    t_w, z_w = oracle.rvea_translate(objs)
    t_g, z_g = st.rvea_translate(ws, _t(objs))
    np.testing.assert_array_equal(z_g.cpu().numpy(), z_w)
    np.testing.assert_array_equal(t_g.cpu().numpy(), t_w)
    refs = oracle.reference_directions(2, 300, M)
    th_w, idx_w = oracle.rvea_partition(t_w, refs, active, N)
    th_g, idx_g = st.rvea_partition(ws, _t(t_w), _t(refs), active, N)
    idx_g = idx_g.cpu().numpy()
    # rsqrtf/acosf on the GPU vs 1/sqrtf/acosf on the host: identical choice
    # unless two cosines round to the same value after the scaling
    mism = np.nonzero(idx_g != idx_w)[0]
    assert len(mism) <= max(1, n // 500), mism
    np.testing.assert_allclose(th_g.cpu().numpy(), th_w, rtol=3e-6, atol=3e-6)
    g_w = oracle.rvea_gamma(refs)
    g_g = st.rvea_gamma(ws, _t(refs)).cpu().numpy()
    np.testing.assert_allclose(g_g, g_w, rtol=3e-6, atol=3e-7)
    apd_w = oracle.rvea_apd(t_w, th_w, g_w, idx_w, 10, 100, 2.0)
    apd_g = st.rvea_apd(ws, _t(t_w), _t(th_w), _t(g_w), _t(idx_w), 10, 100, 2.0).cpu().numpy()
    np.testing.assert_allclose(apd_g, apd_w, rtol=1e-6)
    # elitism on identical inputs is exact integer work
    sel_w, act_w = oracle.rvea_elitism(idx_w, cv, apd_w, N, refs.shape[1])
    sel_g, act_g = st.rvea_elitism(ws, _t(idx_w), _t(cv), _t(apd_w), N, refs.shape[1])
    assert act_g == act_w
    np.testing.assert_array_equal(sel_g.cpu().numpy(), sel_w)
    v_w = oracle.rvea_adapt(refs, objs[:, :N], active)
    v_g = st.rvea_adapt(ws, _t(refs), _t(objs[:, :N].copy()), active).cpu().numpy()
    np.testing.assert_allclose(v_g, v_w, rtol=3e-6, atol=3e-7)


def test_quantize_cv(st, oracle):
    rng = np.random.default_rng(4)
    cv = (rng.random(5000) * 3).astype(np.float32)
    cv[:500] = 0.0
    cv[500:510] = np.nan
    for eps, clip, la, bins in [(0.0, 2.0, 0.0, 16), (1e-3, 2.5, 3.0, 64)]:
        want = oracle.quantize_cv(cv, eps, clip, la, bins)
        got = st.quantize_cv(_t(cv), eps, clip, la, bins).cpu().numpy()
        if la == 0.0:
            np.testing.assert_array_equal(got, want)
        else:  # log1pf differs by an ulp near bin edges
            assert (got != want).mean() < 1e-3
