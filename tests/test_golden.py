"""CPU: the oracle against golden vectors produced by CUDA-MOEA's own stage
code (tests/golden/reference_stages.npz, generated on a B200 by
tests/golden/make_golden.py from oracle/_ref, which is built from the
reference sources).  This pins the oracle to the reference.

Exact: fronts, last-front index, association index and distance on the same
normalised input (this also pins the fused multiply-add form of the
reference's distance), niching selection and RNG offset, RVEA translation,
APD on the same angles, elitism.  Tolerances: intercepts (the reference's
FP32 cuSOLVER SVD against the oracle's FP64 solve), problem objectives and
RVEA angles (CUDA cosf/sinf/powf/rsqrtf/acosf against the host libm).
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
