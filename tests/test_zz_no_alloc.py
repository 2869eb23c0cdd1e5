"""GPU: the allocation-free association entry point (moea_associate_static)
against the workspace entry point in full-scan mode, on two consecutive calls
with different inputs, so that a stale scratch value from the first call
would show in the second.  Collected last (file name) so that it also runs
after every other GPU test in the same process."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_associate_static_matches_workspace_scan(oracle):
    from cuda_moea import stages as st
    ws = st.Workspace(max_points=8192, max_objectives=8, max_directions=4000)
    try:
        cases = [(3, 5000, oracle.reference_directions(1, 40, 3)),
                 (5, 1200, oracle.reference_directions(0, 1000, 5))]
        for k, (M, n, refs) in enumerate(cases):
            rng = np.random.default_rng(100 + k)
            x = (rng.random((M, n)) * rng.random(n) * 2).astype(np.float32)
            x[:, :4] = 0.0
            xt = torch.from_numpy(x).cuda()
            rt = torch.from_numpy(np.ascontiguousarray(refs)).cuda()
            i_s, d_s = st.associate_static(xt, rt)
            i_w, d_w = st.associate(ws, xt, rt, st.ASSOC_SCAN)
            torch.cuda.synchronize()
            np.testing.assert_array_equal(i_s.cpu().numpy(), i_w.cpu().numpy())
            np.testing.assert_array_equal(d_s.cpu().numpy(), d_w.cpu().numpy())
    finally:
        ws.close()


def test_associate_static_at_the_size_limit(oracle):
    """The full static scratch (65536 points, the last valid slot included)
    and a point count that is not a multiple of the block size, two calls in
    a row, against the workspace scan."""
    from cuda_moea import stages as st
    ws = st.Workspace(max_points=65536, max_objectives=3, max_directions=1000)
    try:
        refs = torch.from_numpy(np.ascontiguousarray(oracle.reference_directions(1, 30, 3))).cuda()
        for k, n in enumerate((65536, 65531)):
            rng = np.random.default_rng(300 + k)
            x = (rng.random((3, n)) * rng.random(n) * 3).astype(np.float32)
            x[:, -3:] = 0.0
            xt = torch.from_numpy(x).cuda()
            i_s, d_s = st.associate_static(xt, refs)
            i_w, d_w = st.associate(ws, xt, refs, st.ASSOC_SCAN)
            torch.cuda.synchronize()
            np.testing.assert_array_equal(i_s.cpu().numpy(), i_w.cpu().numpy())
            np.testing.assert_array_equal(d_s.cpu().numpy(), d_w.cpu().numpy())
    finally:
        ws.close()


def test_associate_static_rejects_oversize():
    from cuda_moea import stages as st
    from cuda_moea._lib import MoeaError
    x = torch.zeros((3, 65537), dtype=torch.float32, device="cuda")
    r = torch.ones((3, 4), dtype=torch.float32, device="cuda")
    with pytest.raises(MoeaError):
        st.associate_static(x, r)
