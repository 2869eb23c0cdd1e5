"""Generates tests/golden/reference_stages.npz: outputs of CUDA-MOEA's own
stage code (oracle/_ref/libmoea_ref.so, built from the reference sources by
oracle/ref/Makefile) on seeded inputs.  Needs a CUDA device; run as

    python tests/golden/make_golden.py <output.npz>

The CPU tests (tests/test_golden.py) check the oracle against these vectors,
which pins the oracle to the reference without a GPU.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402  (inputs only: directions, DTLZ1 objectives)
from oracle.ref import ref as R  # noqa: E402

PROBLEMS = [(1, 7, 3), (2, 12, 3), (3, 12, 3), (4, 12, 3), (5, 12, 3), (6, 12, 3), (7, 22, 3),
            (8, 12, 3), (2, 17, 8), (9, 12, 3), (10, 12, 3), (11, 12, 3), (12, 12, 3), (13, 12, 3),
            (14, 12, 3), (15, 7, 3), (1, 600, 5)]


def main(out: str) -> None:
    g: dict[str, np.ndarray] = {}
    rng = np.random.default_rng(2887)
    # ---- non-dominated sort
    nds_cases = [(3, 512, 256, "dtlz1", False), (2, 400, 200, "ties", True), (5, 600, 300, "uniform", True),
                 (8, 256, 128, "uniform", False), (3, 300, 300, "uniform", False)]
    for i, (M, n, N, kind, mixed) in enumerate(nds_cases):
        if kind == "dtlz1":
            objs, _ = O.evaluate("DTLZ1", rng.random((n, M + 4)).astype(np.float32), M)
        elif kind == "ties":
            objs = rng.integers(0, 6, (M, n)).astype(np.float32)
        else:
            objs = rng.random((M, n)).astype(np.float32)
        cv = np.zeros(n, np.float32)
        if mixed:
            cv = np.where(rng.random(n) < 0.3, rng.integers(1, 4, n) * 0.5, 0).astype(np.float32)
        fr, mf = R.ndsort(cv, objs, N)
        g.update({f"nds{i}_objs": objs, f"nds{i}_cv": cv, f"nds{i}_N": np.int32(N),
                  f"nds{i}_fronts": fr, f"nds{i}_max_front": np.int32(mf)})
    # ---- normalisation
    for i, (M, n) in enumerate([(3, 500), (5, 400)]):
        f = (rng.random((M, n)) * rng.random(n) * 4 + 0.1).astype(np.float32)
        ideal = (f.min(1) - 0.05).astype(np.float32)
        fn, rcp = R.normalize(f, ideal)
        g.update({f"norm{i}_f": f, f"norm{i}_ideal": ideal, f"norm{i}_out": fn, f"norm{i}_rcp": rcp})
    # ---- association
    for i, (M, n, N) in enumerate([(3, 500, 92), (5, 300, 200), (8, 256, 1024)]):
        refs = O.reference_directions(0, N, M)
        x = (rng.random((M, n)) * rng.random(n) * 2).astype(np.float32)
        x[:, :8] = refs[:, :8] * 1.5
        idx, dist = R.associate(x, refs)
        g.update({f"assoc{i}_x": x, f"assoc{i}_refs": refs, f"assoc{i}_idx": idx, f"assoc{i}_dist": dist})
    # ---- niching
    for i, (N, H, np_, nl) in enumerate([(200, 91, 120, 150), (256, 120, 0, 400), (300, 64, 250, 80)]):
        nds = np_ + nl
        gidx = rng.permutation(2 * N)[:nds].astype(np.int32)
        idx = rng.integers(0, H, nds).astype(np.int32)
        dist = (rng.integers(0, 40, nds) / 9.0).astype(np.float32)
        sizes = np.array([np_, nl, N - np_, nds], np.int32)
        sel, off = R.niching(1234567, 40 + i, gidx, dist, idx, sizes, H, N)
        g.update({f"nich{i}_gidx": gidx, f"nich{i}_idx": idx, f"nich{i}_dist": dist, f"nich{i}_sizes": sizes,
                  f"nich{i}_H": np.int32(H), f"nich{i}_N": np.int32(N), f"nich{i}_offset": np.uint64(40 + i),
                  f"nich{i}_sel": sel, f"nich{i}_offset_out": np.uint64(off)})
    # ---- problems
    for i, (kind, D, M) in enumerate(PROBLEMS):
        if kind == 15:
            lo = np.array([0.5, 0.45, 0.5, 0.5, 0.875, 0.4, 0.4], np.float32)
            hi = np.array([1.5, 1.35, 1.5, 1.5, 2.625, 1.2, 1.2], np.float32)
            x = (lo + rng.random((64, D)) * (hi - lo)).astype(np.float32)
        else:
            x = rng.random((64, D)).astype(np.float32)
            x[:3] = 0.5
        f, cv = R.problem(kind, x, M)
        g.update({f"prob{i}_kind": np.int32(kind), f"prob{i}_x": x, f"prob{i}_M": np.int32(M),
                  f"prob{i}_objs": f, f"prob{i}_cv": cv})
    # ---- RVEA
    M, N = 3, 150
    objs = (rng.random((M, 2 * N)) + 0.2).astype(np.float32)
    objs[:, 130:N] = 1e15  # dead parent slots
    cv = np.where(rng.random(2 * N) < 0.15, rng.random(2 * N), 0).astype(np.float32)
    refs = O.reference_directions(2, N, M)
    t, z = R.rvea_translate(objs)
    th, idx = R.rvea_partition(t, refs, 130, N)
    gam = R.rvea_gamma(refs)
    apd = R.rvea_apd(t, th, gam, idx, 10, 100, 2.0)
    sel, act = R.rvea_elitism(idx, cv, apd, N, refs.shape[1])
    g.update({"rvea_objs": objs, "rvea_cv": cv, "rvea_refs": refs, "rvea_t": t, "rvea_z": z,
              "rvea_theta": th, "rvea_idx": idx, "rvea_gamma": gam, "rvea_apd": apd,
              "rvea_sel": sel, "rvea_active": np.int32(act)})
    # ---- reproduction: tournament, SBX, PM on explicit draws
    n, D = 65, 9
    parents = rng.random((n, D)).astype(np.float32)
    bounds = np.tile([0.0, 1.0], D).astype(np.float32)
    pcv = np.where(rng.random(n) < 0.3, rng.integers(0, 4, n) * 0.5, 0).astype(np.float32)
    rank = rng.integers(0, 4, n).astype(np.int32)
    cand = rng.integers(0, n, (n, 2)).astype(np.int32)
    win = R.tournament(cand, rank, pcv)
    pairs = n // 2
    u = rng.random((pairs * D, 2)).astype(np.float32)
    sign = rng.integers(0, 2, pairs * D).astype(np.int32)
    copy = rng.random(pairs * D).astype(np.float32)
    off = R.sbx(parents, win, bounds, u, sign, copy, 15.0, 0.9, 0.3, n)
    um = rng.random((n * D, 2)).astype(np.float32)
    um[:, 0] *= 2.0 / D
    mut = R.pm(off, bounds, um, 20.0, 1.0)
    g.update({"rep_parents": parents, "rep_bounds": bounds, "rep_cv": pcv, "rep_rank": rank, "rep_cand": cand,
              "rep_winners": win, "rep_u": u, "rep_sign": sign, "rep_copy": copy, "rep_sbx": off, "rep_um": um,
              "rep_pm": mut, "rep_annealed": np.array([R.annealed(5.0, 40.0, 37, 100),
                                                       R.annealed(20.0, 3.0, 150, 100)], np.float32)})
    # ---- CV quantisation (linear and log mapping)
    qcv = (rng.random(400) * 3).astype(np.float32)
    qcv[:50] = 0.0
    qcv[50:53] = np.nan
    g.update({"quant_cv": qcv, "quant_lin": R.quantize_cv(qcv, 0.0, 2.0, 0.0, 16),
              "quant_log": R.quantize_cv(qcv, 1e-3, 2.5, 3.0, 64)})
    # ---- RVEA direction adaptation and survivor update with sentinels
    M, N, active = 5, 120, 100
    v0 = O.reference_directions(2, N, M)
    aobjs = (rng.random((M, N)) * rng.random(M)[:, None] * 3).astype(np.float32)
    aobjs[:, active:] = 1e15
    g.update({"adapt_v0": v0, "adapt_objs": aobjs, "adapt_active": np.int32(active),
              "adapt_out": R.rvea_adapt(v0, aobjs, active)})
    import torch
    D = 6
    px, ox = rng.random((N, D)).astype(np.float32), rng.random((N, D)).astype(np.float32)
    pf, of = rng.random((M, N)).astype(np.float32), rng.random((M, N)).astype(np.float32)
    pc, oc = rng.random(N).astype(np.float32), rng.random(N).astype(np.float32)
    usel = rng.permutation(2 * N)[:active].astype(np.int32)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    nx, nf, nc = R.rvea_update_t(t(px), t(ox), t(pf), t(of), t(pc), t(oc), t(usel), active)
    g.update({"upd_px": px, "upd_ox": ox, "upd_pf": pf, "upd_of": of, "upd_pc": pc, "upd_oc": oc,
              "upd_sel": usel, "upd_x": nx.cpu().numpy(), "upd_f": nf.cpu().numpy(), "upd_cv": nc.cpu().numpy()})
    np.savez_compressed(out, **g)
    print("wrote", out, len(g), "arrays")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else str(ROOT / "tests" / "golden" / "reference_stages.npz"))
