"""CPU checks of the C-ABI library: it loads, exports every entry point that
include/moea_b200.h declares, reports errors without a GPU, and the host-only
entry points (reference directions) agree with the oracle."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "moea_b200.h"


def _declared():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(moea_[a-z0-9_]+)\s*\(", text)) - {"moea_evaluate_fn", "moea_mating_fn"})


def test_library_exports_every_declared_symbol():
    from cuda_moea import _lib
    L = _lib.lib()
    declared = _declared()
    assert len(declared) >= 30
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, missing
    # the ctypes table covers the whole header
    assert sorted(_lib.SYMBOLS) == declared
    assert L.moea_abi_version() == 1


def test_ctypes_signatures_match_header_arity():
    """Every declaration's parameter count is the one its ctypes binding passes."""
    from cuda_moea import _lib
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    arity = {}
    for name, args in re.findall(r"\b(moea_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", text, flags=re.S):
        if name.endswith("_fn"):
            continue
        args = args.strip()
        arity[name] = 0 if args in ("", "void") else args.count(",") + 1
    bound = {name: len(argtypes) for name, _, argtypes in _lib._SIGNATURES}
    assert arity == bound


def test_errors_are_status_codes_not_exits():
    from cuda_moea import _lib
    L = _lib.lib()
    h = ctypes.c_void_p()
    st = L.moea_workspace_create(0, 0, 3, 10, ctypes.byref(h))
    assert st == 1 and not h.value
    assert b"max_points" in L.moea_last_error()
    st = L.moea_ndsort(None, None, None, 3, 10, 5, None, None, None)
    assert st == 1
    cnt = ctypes.c_int(0)
    assert L.moea_reference_directions(7, 10, 3, None, 0, ctypes.byref(cnt)) == 1


def test_host_reference_directions_match_oracle(oracle):
    from cuda_moea import stages
    for mode, n, M in [(0, 92, 3), (1, 12, 3), (0, 1024, 8), (2, 1024, 8), (1, 254, 3),
                       (0, 16384, 10), (2, 2048, 5)]:
        got = stages.reference_directions(mode, n, M).numpy()
        want = oracle.reference_directions(mode, n, M)
        assert got.shape == want.shape
        np.testing.assert_array_equal(got, want)


def test_config_struct_matches_header_defaults():
    from cuda_moea import _lib
    cfg = _lib.AlgorithmConfig()
    _lib.lib().moea_algorithm_config_defaults(ctypes.byref(cfg), 0)
    assert cfg.population_size == 1024 and cfg.max_generations == 100 and cfg.seed == 2887
    assert cfg.sbx_eta_initial == 30.0 and cfg.pm_eta_initial == 20.0 and cfg.mating == 1
    assert abs(cfg.sparse_ratio - 0.5) < 1e-7 and cfg.rvea_alpha == 2.0 and cfg.use_graphs == 1
    _lib.lib().moea_algorithm_config_defaults(ctypes.byref(cfg), 1)
    assert cfg.mating == 0 and cfg.directions == 1 and abs(cfg.adapt_frequency - 0.1) < 1e-7


def test_association_wrappers_reject_mismatched_arguments():
    """The torch wrappers check dtype, shape and device before any launch: a
    float64 matrix or a direction matrix with fewer rows than objectives would
    make the kernels read past their buffers."""
    import pytest
    import torch
    from cuda_moea import stages as st
    x = torch.zeros((3, 10), dtype=torch.float32)
    good = torch.ones((3, 4), dtype=torch.float32)
    for bad_x, bad_r in [(x.double(), good), (x, good.double()), (x, good[:2]), (x[0], good)]:
        with pytest.raises(ValueError):
            st.associate_static(bad_x, bad_r)
        with pytest.raises(ValueError):
            st.associate(None, bad_x, bad_r)
