"""CPU checks of the oracle itself: published known-answer vectors, hand-made
cases with known fronts / associations / intercepts, and the reference's
documented semantics (tie rules, stop rule, NaN handling)."""
import numpy as np
import pytest


def test_philox_known_answers(oracle):
    # Random123 philox4x32-10 known-answer vectors (Salmon et al., SC'11)
    assert [hex(v) for v in oracle.philox([0, 0, 0, 0], [0, 0])] == \
        ["0x6627e8d5", "0xe169c58d", "0xbc57ac4c", "0x9b00dbd8"]
    assert [hex(v) for v in oracle.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2)] == \
        ["0x408f276d", "0x41c83b0e", "0xa20bc7c6", "0x6d5451fd"]
    assert [hex(v) for v in oracle.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344],
                                          [0xA4093822, 0x299F31D0])] == \
        ["0xd16cfe09", "0x94fdcceb", "0x5001e420", "0x24126ea1"]


def _splitmix64_ref(counter, seed):
    mask = (1 << 64) - 1
    z = (counter ^ seed) & mask
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & mask
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & mask
    return (z ^ (z >> 31)) & 0xFFFFFFFF


def test_splitmix_and_seed(oracle):
    for c, s in [(0, 0), (1, 2887), (123456789, 0xDEADBEEF), (2 ** 40 + 7, 2 ** 63 + 5)]:
        assert oracle.splitmix_u32(c, s) == _splitmix64_ref(c, s)
    # the reference derives the island seed with the same mixing from CudaConfig.seed
    mask = (1 << 64) - 1
    x = 2887
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & mask
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & mask
    assert oracle.derive_seed(2887) == (x ^ (x >> 31))


def test_dominance_chain_and_stop_rule(oracle):
    # 8 points on a chain p0 < p1 < ... < p7 (each dominates the next)
    objs = np.array([[i, i, i] for i in range(8)], np.float32).T.copy()
    cv = np.zeros(8, np.float32)
    fronts, mf = oracle.ndsort(cv, objs, 8)
    assert list(fronts) == list(range(8)) and mf == 7
    # stop rule: fronts peeled until >= target assigned, the rest -1
    fronts, mf = oracle.ndsort(cv, objs, 3)
    assert mf == 2 and list(fronts) == [0, 1, 2] + [-1] * 5


def test_dominance_constraints_ties_duplicates_nan(oracle):
    # feasible beats infeasible; infeasible by strictly smaller cv; duplicates
    # never dominate each other; NaN objectives are incomparable
    objs = np.array([[1, 1], [1, 1], [0, 2], [2, 2], [5, 5], [5, 5], [np.nan, 0], [0, 0]],
                    np.float32).T.copy()
    cv = np.array([0, 0, 0, 0, 1, 1, 0, 2], np.float32)
    fronts, mf = oracle.ndsort(cv, objs, 8)
    # feasible: p0 == p1 (duplicates), p2 incomparable with them, p3 dominated by
    # p0/p1/p2; p6 (NaN) front 0; infeasible p4 == p5 (cv 1) before p7 (cv 2)
    assert fronts[0] == 0 and fronts[1] == 0 and fronts[2] == 0 and fronts[6] == 0
    assert fronts[3] == 1
    assert fronts[4] == 2 and fronts[5] == 2 and fronts[7] == 3
    assert mf == 3
    assert not oracle.dominates(cv, objs, 0, 1)
    assert oracle.dominates(cv, objs, 0, 3)
    assert oracle.dominates(cv, objs, 4, 7)
    assert not oracle.dominates(cv, objs, 7, 4)


def test_ndsort_matches_bruteforce_definition(oracle):
    rng = np.random.default_rng(3)
    for M, n in [(2, 60), (3, 120), (5, 90)]:
        objs = rng.integers(0, 6, size=(M, n)).astype(np.float32)  # many ties
        cv = np.where(rng.random(n) < 0.3, rng.integers(0, 3, n), 0).astype(np.float32)
        fronts, mf = oracle.ndsort(cv, objs, n)
        # front = length of the longest dominance chain ending at the point
        dom = np.zeros((n, n), bool)
        for p in range(n):
            for q in range(n):
                dom[p, q] = oracle.dominates(cv, objs, p, q)
        rank = np.zeros(n, int)
        changed = True
        while changed:
            changed = False
            for q in range(n):
                r = max([rank[p] + 1 for p in range(n) if dom[p, q]], default=0)
                if r != rank[q]:
                    rank[q] = r
                    changed = True
        assert (fronts == rank).all()
        assert mf == rank.max()


def test_extract_order(oracle):
    fronts = np.array([2, 0, -1, 1, 0, 2, 1], np.int32)
    gidx, sizes = oracle.nds_extract(fronts, 2, 4)
    assert list(sizes) == [4, 2, 0, 6]
    assert list(gidx) == [1, 3, 4, 6, 0, 5]


def test_association_tie_goes_to_smaller_index(oracle):
    # a point on the bisector is equidistant from the two axis directions
    refs = np.array([[1, 0, np.sqrt(0.5)], [0, 1, np.sqrt(0.5)]], np.float32)
    x = np.array([[1.0, 0.5, 2.0], [1.0, 0.5, 0.0]], np.float32)
    idx, dist = oracle.associate(x, refs[:, :2].copy())
    assert idx[0] == 0 and idx[1] == 0  # ties -> smaller index
    assert idx[2] == 0 and dist[2] == 0.0
    idx, dist = oracle.associate(x, refs)
    assert idx[0] == 2 and dist[0] < 1e-6


def test_normalize_hyperplane_and_fallback(oracle):
    # points on the plane f0/2 + f1/4 + f2/8 = 1: intercepts (2, 4, 8)
    pts = np.array([[2, 0, 0], [0, 4, 0], [0, 0, 8], [1, 2, 0], [0.5, 1, 2]], np.float32).T.copy()
    f, rcp, ext, ill = oracle.normalize(pts, np.zeros(3, np.float32))
    assert ill == 0
    np.testing.assert_allclose(rcp, [0.5, 0.25, 0.125], rtol=1e-6)
    assert list(ext) == [0, 1, 2]
    np.testing.assert_allclose(f, pts * rcp[:, None], rtol=1e-6)
    # degenerate: every point identical -> singular extreme matrix -> row-maximum fallback
    same = np.ones((3, 4), np.float32) * 3.0
    f, rcp, ext, ill = oracle.normalize(same, np.zeros(3, np.float32))
    assert ill == 1
    np.testing.assert_allclose(rcp, [1 / 3.0] * 3, rtol=1e-6)
    # all at the ideal point -> maxima below 1e-10 -> unit intercepts
    f, rcp, ext, ill = oracle.normalize(np.zeros((3, 4), np.float32), np.zeros(3, np.float32))
    assert ill == 1 and list(rcp) == [1.0, 1.0, 1.0]


@pytest.mark.parametrize("M", [5, 8, 10])
def test_normalize_many_objectives(oracle, M):
    """The Jacobi intercept solve at the many-objective sizes: a non-diagonal
    extreme matrix gives the hyperplane through its columns (FP64 solve of
    E^T a = 1), and a rank-deficient objective set takes the row-maximum
    fallback (normalization.cu:1302-1394)."""
    rng = np.random.default_rng(M)
    b = (1.0 + rng.random(M)).astype(np.float32)
    # extremes: b_j on axis j plus off-axis parts below 0.03, so their
    # achievement scalarising value (<= 3e4 with the 1e6 weights) stays below
    # every interior point's (components >= 0.05, value >= 5e4)
    ext_pts = np.diag(b) + (rng.random((M, M)) * 0.03).astype(np.float32)
    interior = (0.05 + rng.random((M, 300))).astype(np.float32)
    pts = np.concatenate([interior[:, :100], ext_pts, interior[:, 100:]], axis=1)
    ideal = np.zeros(M, np.float32)
    f, rcp, ext, ill = oracle.normalize(pts, ideal)
    assert ill == 0
    assert list(ext) == list(range(100, 100 + M))
    E = pts[:, ext].astype(np.float64)
    want = np.linalg.solve(E.T, np.ones(M))
    np.testing.assert_allclose(rcp, want, rtol=1e-5)
    np.testing.assert_allclose(f, pts * rcp[:, None], rtol=1e-5)
    # two equal objectives make every extreme matrix singular
    dup = interior.copy()
    dup[M - 1] = dup[M - 2]
    f, rcp, ext, ill = oracle.normalize(dup, ideal)
    assert ill == 1
    np.testing.assert_allclose(rcp, 1.0 / dup.max(axis=1), rtol=1e-6)


def test_reference_direction_counts(oracle):
    assert oracle.reference_directions(0, 92, 3).shape == (3, 91)
    assert oracle.reference_directions(0, 32768, 3).shape == (3, 32640)
    assert oracle.reference_directions(1, 254, 3).shape == (3, 32640)
    assert oracle.reference_directions(1, 255, 3).shape == (3, 32896)
    assert oracle.reference_directions(2, 1024, 8).shape == (8, 912)
    r = oracle.reference_directions(1, 2, 3)
    # prev_permutation order of the stars-and-bars mask
    expect = np.array([[0, 0, 1], [0, .5, .5], [0, 1, 0], [.5, 0, .5], [.5, .5, 0], [1, 0, 0]],
                      np.float32)
    expect = expect / np.linalg.norm(expect, axis=1, keepdims=True)
    np.testing.assert_allclose(r.T, expect, rtol=1e-6)


def test_niching_semantics(oracle):
    # 2 prior points on direction 0; last front: 2 on direction 0, 2 on direction 1
    gidx = np.array([10, 11, 20, 21, 22, 23], np.int32)
    idx = np.array([0, 0, 0, 0, 1, 1], np.int32)
    dist = np.array([.1, .2, .3, .05, .4, .2], np.float32)
    sizes = np.array([2, 4, 2, 6], np.int32)
    sel, off = oracle.niching(7, 100, gidx, dist, idx, sizes, 3, 4)
    assert off == 108  # two draws per last-front member
    assert list(sel[:2]) == [10, 11]
    # direction 1 is empty among the prior fronts: its closest member (23) is
    # the deterministic first choice; the second pick is random between the
    # closer direction-0 member (21) and direction 1's second member (22)
    assert sel[2] == 23 and sel[3] in (21, 22)


def test_tournament_rules(oracle):
    cv = np.array([0, 0, 1, 2, 0.5], np.float32)
    rank = np.array([3, 1, 0, 0, 0], np.int32)
    cand = np.array([[0, 2], [2, 0], [2, 3], [3, 2], [0, 1], [1, 0], [3, 3], [4, 4]], np.int32)
    w = oracle.tournament(cand, rank, cv)
    assert list(w) == [0, 0, 2, 2, 1, 1, 3, 4]


def test_sbx_pm_bounds_and_copy(oracle):
    rng = np.random.default_rng(1)
    par = rng.random((6, 5)).astype(np.float32)
    b = np.tile([0.0, 1.0], 5).astype(np.float32)
    pidx = np.array([0, 1, 2, 3, 4, 5], np.int32)
    u = rng.random((15, 2)).astype(np.float32)
    sign = rng.integers(0, 2, 15).astype(np.int32)
    copy = rng.random(15).astype(np.float32)
    off = oracle.sbx(par, pidx, b, u, sign, copy, 30.0, 1.0, 1.0, 6)  # copy prob 1 -> copies
    np.testing.assert_array_equal(off, par)
    off = oracle.sbx(par, pidx, b, u, sign, copy, 30.0, 1.0, 0.0, 6)
    assert (off >= 0).all() and (off <= 1).all()
    # children are symmetric about the parents' midpoint unless clamped
    mid_p = (par[0::2] + par[1::2]) / 2
    mid_c = (off[0::2] + off[1::2]) / 2
    inside = (off > 0) & (off < 1)
    ok = inside[0::2] & inside[1::2]
    np.testing.assert_allclose(mid_c[ok], mid_p[ok], atol=1e-6)
    m = oracle.pm(off, b, rng.random((30, 2)).astype(np.float32), 20.0, 1.0)
    assert (m >= 0).all() and (m <= 1).all()


def test_problem_fp32_against_fp64(oracle):
    rng = np.random.default_rng(5)
    for kind, D, M in [("DTLZ1", 7, 3), ("DTLZ2", 12, 3), ("DTLZ3", 12, 3), ("DTLZ4", 12, 3),
                       ("DTLZ5", 12, 3), ("DTLZ6", 12, 3), ("DTLZ7", 22, 3), ("ConvexDTLZ2", 12, 3),
                       ("DTLZ2", 17, 8), ("C1DTLZ1", 14, 10), ("C3DTLZ4", 14, 10)]:
        x = rng.random((64, D)).astype(np.float32)
        f32, cv32 = oracle.evaluate(kind, x, M, 0)
        f64, cv64 = oracle.evaluate(kind, x, M, 1)
        # FP32 rounding of the angle arguments makes small objectives (cos near
        # pi/2) relatively inaccurate; bound the error against max(|f|, 1)
        scale = np.maximum(np.abs(f64), 1.0)
        assert (np.abs(f32 - f64) / scale).max() < (2e-4 if kind == "DTLZ6" else 2e-5), kind
    # the analytic DTLZ2 front: sum of squares == 1 at g == 0
    x = np.full((4, 12), 0.5, np.float32)
    x[:, :2] = rng.random((4, 2))
    f, _ = oracle.evaluate("DTLZ2", x, 3, 1)
    np.testing.assert_allclose((f ** 2).sum(0), 1.0, rtol=1e-6)


def test_rvea_semantics(oracle):
    """Hand cases for the RVEA stages: translation floor, partition tie and
    dead slots, gamma of orthogonal directions, APD edge values, and elitism
    (objective_translation.cu:125, reference_partition.cu:407,
    angle_penalized_distance.cu:159,387, elitism_selection.cu:194)."""
    out, z = oracle.rvea_translate(np.array([[1, 2, 3], [5, 4, 6]], np.float32))
    np.testing.assert_array_equal(z, [1, 4])
    np.testing.assert_array_equal(out, np.array([[1e-32, 1, 2], [1, 1e-32, 2]], np.float32))

    refs = np.eye(2, dtype=np.float32)  # directions e0, e1 as columns
    t = np.array([[2, 1, 1], [1, 1, 3]], np.float32)
    th, idx = oracle.rvea_partition(t, refs, 2, 3)
    assert list(idx) == [0, 0, 2]  # (1,1) ties -> smaller direction; slot 2 is dead -> K
    np.testing.assert_allclose(th[:2], [np.arccos(2 / np.sqrt(5)), np.pi / 4], rtol=1e-6)

    g = oracle.rvea_gamma(refs)
    np.testing.assert_allclose(g, [np.pi / 2] * 2, rtol=1e-6)
    assert oracle.rvea_gamma(np.ones((2, 1), np.float32))[0] == np.float32(np.pi)

    t = np.array([[3, 0, 1], [4, 0, 1]], np.float32)
    apd = oracle.rvea_apd(t, np.zeros(3, np.float32), g, np.array([0, 0, 5], np.int32), 0, 10, 2.0)
    # generation 0: no angle penalty, APD = |f'|; a zero vector -> 0; a dead direction -> 1e30
    np.testing.assert_allclose(apd, [5, 0, 1e30], rtol=1e-6)

    idx = np.array([0, 0, 1, 1], np.int32)
    cv = np.array([0, 0, 0, 0.5], np.float32)
    apd = np.array([2, 1, 3, 9], np.float32)
    sel, act = oracle.rvea_elitism(idx, cv, apd, 4, 2)
    assert act == 2 and sorted(sel) == [1, 2]  # one winner per direction, feasible first
    sel, act = oracle.rvea_elitism(idx, cv, apd, 1, 2)
    assert act == 1 and list(sel) == [1]  # more winners than N: the smallest metric


def test_rvea_adaptation(oracle):
    """Directions scaled by the objective ranges of the active members only,
    renormalised; a zero range falls back to the unscaled direction
    (rvea_reference_adaptation.cu:279)."""
    s = np.float32(np.sqrt(0.5))
    v0 = np.array([[1, 0, s], [0, 1, s]], np.float32)
    objs = np.array([[0, 2, 1, 100], [3, 4, 3.5, -50]], np.float32)  # the last slot is dead
    v = oracle.rvea_adapt(v0, objs, 3)
    want = np.array([[1, 0, 2 / np.sqrt(5)], [0, 1, 1 / np.sqrt(5)]])
    np.testing.assert_allclose(v, want, rtol=1e-6, atol=1e-7)
    flat = np.ones((2, 4), np.float32)
    np.testing.assert_allclose(oracle.rvea_adapt(v0, flat, 4), v0, rtol=1e-6)
