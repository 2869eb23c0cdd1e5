"""CPU: the seeded analytic-front samples of cuda_moea.metrics against the
reference's own sampler (tests/evaluation/pareto_front.py), through the
SHA-256 of their FP32 bytes recorded in tests/golden/quality_reference.json
by tests/golden/make_quality_golden.py."""
import hashlib
import json
from pathlib import Path

import pytest

GOLDEN = json.loads((Path(__file__).resolve().parent / "golden" / "quality_reference.json").read_text())


@pytest.mark.parametrize("case", GOLDEN["fronts"], ids=lambda c: f"{c['problem']}-{c['count']}")
def test_front_samples_equal_reference_sampler(case):
    from cuda_moea.metrics import pareto_front_points
    p = pareto_front_points(case["problem"], case["objectives"], case["count"], case["seed"])
    assert hashlib.sha256(p.numpy().tobytes()).hexdigest() == case["sha256_f32"]
