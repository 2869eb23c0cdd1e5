"""GPU: generations assembled from the strategy handles of the C ABI
(moea_create_* : directions, mating, crossover, mutation, environmental
selection, the reference's strategy interfaces) equal the algorithm object's
generations bit for bit.  The driver is a C++ program compiled against
include/moea_b200.h (tests/capi/strategy_generation.cpp)."""
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
LIBDIR = ROOT / "cuda-moea_b200" / "cuda_moea"


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    exe = tmp_path_factory.mktemp("capi") / "strategy_generation"
    cmd = ["g++", "-std=c++17", "-O2", str(ROOT / "tests" / "capi" / "strategy_generation.cpp"), "-o", str(exe),
           f"-I{ROOT / 'include'}", "-I/usr/local/cuda/include", f"-L{LIBDIR}", "-lmoea_b200",
           "-L/usr/local/cuda/lib64", "-lcudart", f"-Wl,-rpath,{LIBDIR}", "-Wl,-rpath,/usr/local/cuda/lib64"]
    subprocess.run(cmd, check=True)
    return exe


@pytest.mark.parametrize("algorithm,kind,D,M,N,G", [
    (0, 1, 7, 3, 2048, 6),       # NSGA-III DTLZ1 (fused generation path in the algorithm object)
    (0, 2, 12, 3, 8192, 4),      # NSGA-III DTLZ2, staged path
    (0, 9, 14, 5, 1000, 5),      # constrained C1-DTLZ1
    (1, 2, 17, 8, 1024, 6),      # RVEA DTLZ2, adaptive directions adapting on the reference's schedule
    (1, 7, 22, 3, 500, 5),       # RVEA DTLZ7
])
def test_handle_generations_equal_algorithm(driver, algorithm, kind, D, M, N, G):
    r = subprocess.run([str(driver), str(algorithm), str(kind), str(D), str(M), str(N), str(G)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().startswith("OK")
