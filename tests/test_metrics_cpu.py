"""CPU: the analytic DTLZ reference fronts."""
import numpy as np


def test_dtlz_reference_fronts():
    from cuda_moea.metrics import dtlz_reference_front
    f1 = dtlz_reference_front("DTLZ1", 3, 12).numpy()
    assert f1.shape == (91, 3)
    np.testing.assert_allclose(f1.sum(1), 0.5, rtol=0, atol=1e-15)
    f2 = dtlz_reference_front("DTLZ2", 5, 4).numpy()
    assert f2.shape == (70, 5)
    np.testing.assert_allclose(np.linalg.norm(f2, axis=1), 1.0, rtol=0, atol=1e-15)
    assert (f2 >= 0).all()
