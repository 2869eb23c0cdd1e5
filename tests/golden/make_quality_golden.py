"""Generates tests/golden/quality_reference.json from the reference's own
evaluation code (tests/evaluation/pareto_front.py and
tests/evaluation/metrics/igd.py of CUDA-MOEA, imported from a checkout given
as the first argument or CUDA_MOEA_REFERENCE).  Run here, on the CPU:

    python tests/golden/make_quality_golden.py <path of the CUDA-MOEA checkout>

It records (1) the SHA-256 of the FP32 bytes of the seeded analytic-front
samples the reference's published IGD numbers use, and (2) the reference's IGD
of seeded approximations (regenerated by the tests from the same numpy
seeds) against small sphere/simplex fronts, with and without the
non-dominated filter."""
import hashlib
import json
import os
import sys
from pathlib import Path

import numpy as np
import torch

sys.path.insert(0, str(Path(__file__).resolve().parent))
from quality_inputs import approximation  # noqa: E402


def main():
    root = Path(sys.argv[1] if len(sys.argv) > 1 else os.environ["CUDA_MOEA_REFERENCE"])
    sys.path.insert(0, str(root))
    from tests.evaluation.metrics.igd import igd
    from tests.evaluation.pareto_front import pareto_front_points
    out = {"fronts": [], "igd": []}
    for problem, count in [("dtlz1", 20000), ("dtlz2", 20000), ("dtlz2", 50000), ("dtlz3", 1000)]:
        p = pareto_front_points(problem, 3, count=count, device="cpu", seed=2887)
        out["fronts"].append({"problem": problem, "objectives": 3, "count": count, "seed": 2887,
                              "sha256_f32": hashlib.sha256(p.numpy().tobytes()).hexdigest()})
    for seed, n, M, count, filt in [(1, 500, 3, 2000, True), (2, 1000, 3, 3000, False), (3, 300, 5, 1500, True),
                                    (4, 64, 3, 20000, True)]:
        ref = pareto_front_points("dtlz2", M, count=count, device="cpu", seed=2887).to(torch.float64)
        value = igd(approximation(seed, n, M), ref, filter_nondominated=filt)
        out["igd"].append({"seed": seed, "n": n, "objectives": M, "front_count": count,
                           "filter_nondominated": filt, "igd": value})
    path = Path(__file__).resolve().parent / "quality_reference.json"
    path.write_text(json.dumps(out, indent=1) + "\n")
    print("wrote", path)


if __name__ == "__main__":
    main()
