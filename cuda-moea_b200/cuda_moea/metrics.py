"""Quality metrics on the GPU in FP64.

igd() follows the reference's evaluation metric (tests/evaluation/metrics/
igd.py): rows with a non-finite objective are dropped, optionally only the
non-dominated rows are kept, and the result is the mean distance from every
reference point to its nearest kept row.  The distances and the mean are
computed in FP64 on the device (moea_igd in libmoea_b200).

dtlz_reference_front() gives deterministic points of the analytic Pareto
fronts of DTLZ1-4: Das-Dennis points on the simplex sum(f) = 0.5 (DTLZ1) or
on the unit sphere (DTLZ2-4).

pareto_front_points() draws the seeded analytic-front samples that the
reference's published quality numbers are measured against
(tests/evaluation/pareto_front.py:17-33, 142-175): for DTLZ1 normalised
exponentials on the simplex sum(f) = 0.5, for DTLZ2-4 uniform points of the
positive orthant scaled onto the unit sphere, both from torch's CPU
generator seeded with `seed`, in FP32.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from ._lib import check, lib
from .stages import Workspace, _p, _stream


def igd(approximated_front: torch.Tensor, reference_front: torch.Tensor, *,
        filter_nondominated: bool = True, workspace: Workspace | None = None) -> float:
    """IGD of an (N, M) approximation against an (R, M) reference front."""
    approx = torch.as_tensor(approximated_front)
    ref = torch.as_tensor(reference_front)
    if approx.dim() != 2 or ref.dim() != 2 or approx.shape[1] != ref.shape[1]:
        raise ValueError("approximated_front (N, M) and reference_front (R, M) must share M")
    n, M = approx.shape
    device = approx.device if approx.is_cuda else torch.device("cuda")
    objs = approx.to(device=device, dtype=torch.float32).t().contiguous()   # (M, N)
    r = ref.to(device=device, dtype=torch.float64).contiguous()              # (R, M)
    own = workspace is None
    ws = workspace or Workspace(max_points=max(2, n), max_objectives=M, max_directions=1)
    try:
        d_min = torch.empty(r.shape[0], dtype=torch.float64, device=device)
        out = ctypes.c_double(0.0)
        check(lib().moea_igd(ws.handle, _p(objs), n, M, _p(r), r.shape[0], 1 if filter_nondominated else 0,
                             _p(d_min), ctypes.byref(out), _stream()))
        return float(out.value)
    finally:
        if own:
            ws.close()


def dtlz_reference_front(problem: str, objectives: int, partitions: int) -> torch.Tensor:
    """(R, M) FP64 points of the analytic front of DTLZ1-4 from Das-Dennis
    partitions of the simplex."""
    from itertools import combinations

    M, h = int(objectives), int(partitions)
    pts = []
    for bars in combinations(range(h + M - 1), M - 1):
        prev, row = -1, []
        for b in bars:
            row.append(b - prev - 1)
            prev = b
        row.append(h + M - 2 - prev)
        pts.append(row)
    w = np.asarray(pts, dtype=np.float64) / h
    name = problem.upper()
    if name == "DTLZ1":
        f = 0.5 * w
    elif name in ("DTLZ2", "DTLZ3", "DTLZ4"):
        f = w / np.linalg.norm(w, axis=1, keepdims=True)
    else:
        raise ValueError("analytic fronts are provided for DTLZ1-4")
    return torch.from_numpy(f)


def pareto_front_points(problem: str, objectives: int, count: int = 20000, seed: int = 2887) -> torch.Tensor:
    """(count, M) FP32 samples of the analytic front of DTLZ1-4 (CPU)."""
    name = problem.upper()
    if objectives < 2 or count <= 0:
        raise ValueError("need at least two objectives and a positive count")
    gen = torch.Generator(device="cpu").manual_seed(seed)
    u = torch.rand((count, objectives), generator=gen, dtype=torch.float32)
    if name == "DTLZ1":
        e = -torch.log(u.clamp_min(torch.finfo(torch.float32).tiny))
        return 0.5 * e / e.sum(dim=1, keepdim=True)
    if name in ("DTLZ2", "DTLZ3", "DTLZ4"):
        return u / u.norm(dim=1, keepdim=True).clamp_min(torch.finfo(torch.float32).eps)
    raise ValueError("seeded front samples are provided for DTLZ1-4")
