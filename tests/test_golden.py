"""CPU: the oracle against golden vectors produced by CUDA-MOEA's own stage
code (tests/golden/reference_stages.npz, generated on a B200 by
tests/golden/make_golden.py from oracle/_ref, which is built from the
reference sources).  This pins the oracle to the reference.

Exact: fronts, last-front index, association index and distance on the same
normalised input (this also pins the fused multiply-add form of the
reference's distance), niching selection and RNG offset, RVEA translation,
APD on the same angles, elitism.  Tolerances: intercepts (the reference's
FP32 cuSOLVER SVD against the oracle's FP64 solve), problem objectives and
RVEA angles (CUDA cosf/sinf/powf/rsqrtf/acosf against the host libm), SBX
and PM values (CUDA powf), the log CV mapping (log1pf) and the adapted
directions (rsqrtf).  Exact too: tournament winners, the annealed
distribution index, the linear CV quantisation and the RVEA survivor update
with its dead-slot sentinels.
"""
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden" / "reference_stages.npz"
pytestmark = pytest.mark.skipif(not GOLDEN.exists(), reason="golden vectors not generated yet")


@pytest.fixture(scope="module")
def g():
    return dict(np.load(GOLDEN))


def _cases(g, prefix):
    ids = sorted({k.split("_")[0] for k in g if k.startswith(prefix)})
    return ids


def test_ndsort_golden(g, oracle):
    ids = _cases(g, "nds")
    assert len(ids) >= 5
    for c in ids:
        fr, mf = oracle.ndsort(g[f"{c}_cv"], g[f"{c}_objs"], int(g[f"{c}_N"]))
        np.testing.assert_array_equal(fr, g[f"{c}_fronts"], err_msg=c)
        assert mf == int(g[f"{c}_max_front"]), c


def test_normalize_golden(g, oracle):
    for c in _cases(g, "norm"):
        f, rcp, ext, ill = oracle.normalize(g[f"{c}_f"], g[f"{c}_ideal"])
        # FP32 SVD + pinv in the reference, FP64 Jacobi in the oracle
        np.testing.assert_allclose(rcp, g[f"{c}_rcp"], rtol=2e-5, err_msg=c)
        np.testing.assert_allclose(f, g[f"{c}_out"], rtol=2e-5, atol=1e-7, err_msg=c)


def test_association_golden(g, oracle):
    for c in _cases(g, "assoc"):
        idx, dist = oracle.associate(g[f"{c}_x"], g[f"{c}_refs"])
        np.testing.assert_array_equal(idx, g[f"{c}_idx"], err_msg=c)
        np.testing.assert_array_equal(dist, g[f"{c}_dist"], err_msg=c)


def test_niching_golden(g, oracle):
    for c in _cases(g, "nich"):
        sel, off = oracle.niching(1234567, int(g[f"{c}_offset"]), g[f"{c}_gidx"], g[f"{c}_dist"],
                                  g[f"{c}_idx"], g[f"{c}_sizes"], int(g[f"{c}_H"]), int(g[f"{c}_N"]))
        np.testing.assert_array_equal(sel, g[f"{c}_sel"], err_msg=c)
        assert off == int(g[f"{c}_offset_out"])


def test_problems_golden(g, oracle):
    for c in _cases(g, "prob"):
        kind, M = int(g[f"{c}_kind"]), int(g[f"{c}_M"])
        f, cv = oracle.evaluate(kind, g[f"{c}_x"], M)
        ref = g[f"{c}_objs"]
        tol = 2e-5 if kind in (5, 6) else 4e-6
        assert (np.abs(f - ref) / np.maximum(np.abs(ref), 1.0)).max() <= tol, (c, kind)
        np.testing.assert_allclose(cv, g[f"{c}_cv"], rtol=1e-5, atol=1e-5, err_msg=c)


def test_rvea_golden(g, oracle):
    t, z = oracle.rvea_translate(g["rvea_objs"])
    np.testing.assert_array_equal(z, g["rvea_z"])
    np.testing.assert_array_equal(t, g["rvea_t"])
    th, idx = oracle.rvea_partition(g["rvea_t"], g["rvea_refs"], 130, 150)
    assert (idx != g["rvea_idx"]).sum() <= 1
    # theta = acosf(cos) with the device's rsqrtf/acosf against the host's
    # 1/sqrtf and acosf: a few ulps apart in cos, which acos amplifies by
    # 1/sin(theta) near theta = 0, so the check is on the cosines
    np.testing.assert_allclose(np.cos(th.astype(np.float64)), np.cos(g["rvea_theta"].astype(np.float64)),
                               rtol=0, atol=2e-6)
    np.testing.assert_allclose(oracle.rvea_gamma(g["rvea_refs"]), g["rvea_gamma"], rtol=3e-6, atol=3e-7)
    apd = oracle.rvea_apd(g["rvea_t"], g["rvea_theta"], g["rvea_gamma"], g["rvea_idx"], 10, 100, 2.0)
    np.testing.assert_array_equal(apd, g["rvea_apd"])
    sel, act = oracle.rvea_elitism(g["rvea_idx"], g["rvea_cv"], g["rvea_apd"], 150, g["rvea_refs"].shape[1])
    assert act == int(g["rvea_active"])
    np.testing.assert_array_equal(sel, g["rvea_sel"])


def _has(g, key):
    if key not in g:
        pytest.skip("golden vectors predate this case")


def test_reproduction_golden(g, oracle):
    _has(g, "rep_winners")
    np.testing.assert_array_equal(oracle.tournament(g["rep_cand"], g["rep_rank"], g["rep_cv"]), g["rep_winners"])
    n = g["rep_parents"].shape[0]
    off = oracle.sbx(g["rep_parents"], g["rep_winners"], g["rep_bounds"], g["rep_u"], g["rep_sign"],
                     g["rep_copy"], 15.0, 0.9, 0.3, n)
    np.testing.assert_allclose(off, g["rep_sbx"], rtol=2e-6, atol=2e-7)
    mut = oracle.pm(g["rep_sbx"], g["rep_bounds"], g["rep_um"], 20.0, 1.0)
    np.testing.assert_allclose(mut, g["rep_pm"], rtol=5e-6, atol=5e-7)
    assert np.float32(oracle.annealed(5.0, 40.0, 37, 100)) == g["rep_annealed"][0]
    assert np.float32(oracle.annealed(20.0, 3.0, 150, 100)) == g["rep_annealed"][1]


def test_quantize_golden(g, oracle):
    _has(g, "quant_cv")
    np.testing.assert_array_equal(oracle.quantize_cv(g["quant_cv"], 0.0, 2.0, 0.0, 16), g["quant_lin"])
    assert (oracle.quantize_cv(g["quant_cv"], 1e-3, 2.5, 3.0, 64) != g["quant_log"]).mean() < 1e-2


def test_rvea_adapt_and_update_golden(g, oracle):
    _has(g, "adapt_out")
    np.testing.assert_allclose(oracle.rvea_adapt(g["adapt_v0"], g["adapt_objs"], int(g["adapt_active"])),
                               g["adapt_out"], rtol=3e-6, atol=3e-7)
    # survivor update (rvea_population_update.cu:263-300): the selected rows in
    # ascending order, then NaN variables and 1e15 objectives/violations
    sel = np.sort(g["upd_sel"])
    act, N = len(sel), g["upd_px"].shape[0]
    x = np.concatenate([g["upd_px"], g["upd_ox"]])[sel]
    f = np.concatenate([g["upd_pf"], g["upd_of"]], 1)[:, sel]
    cv = np.concatenate([g["upd_pc"], g["upd_oc"]])[sel]
    np.testing.assert_array_equal(g["upd_x"][:act], x)
    assert np.isnan(g["upd_x"][act:]).all()
    np.testing.assert_array_equal(g["upd_f"][:, :act], f)
    assert (g["upd_f"][:, act:] == np.float32(1e15)).all()
    np.testing.assert_array_equal(g["upd_cv"][:act], cv)
    assert (g["upd_cv"][act:] == np.float32(1e15)).all() and act < N
