"""CPU: the Das-Dennis directions of the oracle and of the product's host
generator against the reference's own generators (compiled from its sources
into oracle/_ref/libmoea_ref_host.so by oracle/ref/Makefile), bit for bit.

The enumeration order decides which index wins an association tie, and the
two FP32 normalisations differ between the reference's functions
(nsga3_reference_generator.cu:153-182 divides by sqrtf, :184-221 multiplies by
1/std::sqrt), so equality of every bit is the check."""
import numpy as np
import pytest

from oracle.ref import ref as R

pytestmark = pytest.mark.skipif(not R.host_available(),
                                reason="oracle/_ref not built (needs the reference sources)")

CASES = [(0, 92, 3), (0, 32768, 3), (0, 1024, 3), (0, 1000, 5), (0, 4200, 8), (0, 300, 10),
         (0, 16384, 10), (0, 2, 2), (1, 12, 3), (1, 254, 3), (1, 255, 3), (1, 3, 8), (1, 8, 8),
         (1, 1, 4), (2, 1024, 8), (2, 92, 3), (2, 1024, 3), (2, 16384, 10), (2, 4096, 5)]


@pytest.mark.parametrize("mode,n,M", CASES)
def test_oracle_directions_equal_reference(oracle, mode, n, M):
    want = R.directions(mode, n, M)
    got = oracle.reference_directions(mode, n, M)
    assert got.shape == want.shape
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("mode,n,M", CASES)
def test_product_directions_equal_reference(mode, n, M):
    from cuda_moea import _lib
    import ctypes
    L = _lib.lib()
    count = ctypes.c_int(0)
    _lib.check(L.moea_reference_directions(mode, n, M, None, 0, ctypes.byref(count)))
    out = np.zeros((M, count.value), np.float32)
    _lib.check(L.moea_reference_directions(mode, n, M, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                           out.size, ctypes.byref(count)))
    want = R.directions(mode, n, M)
    np.testing.assert_array_equal(out.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("name", ["libmoea_ref.so", "libmoea_ref_algo.so", "libmoea_ref_host.so"])
def test_reference_pin_libraries_resolve_every_symbol(name):
    """The pin libraries load with every symbol bound now (RTLD_NOW), so a
    reference source missing from oracle/ref/Makefile shows here, on the CPU,
    rather than on the GPU box."""
    import ctypes
    path = R.LIB_PATH.parent / name
    if not path.exists():
        pytest.skip(f"{name} not built")
    ctypes.CDLL(str(path), mode=2)  # RTLD_NOW
