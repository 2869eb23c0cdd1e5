"""Stage-level calls of the generation hot path on CUDA tensors.

Thin torch-facing wrappers of the stage entry points of libmoea_b200 (one per
hot-path stage of CUDA-MOEA).  Tensors must be contiguous CUDA tensors on the
same device; work is ordered on the current torch stream.
"""
from __future__ import annotations

import ctypes

import torch

from ._lib import check, lib


def _p(t: torch.Tensor | None) -> int | None:
    if t is None:
        return None
    if not t.is_cuda or not t.is_contiguous():
        raise ValueError("expected a contiguous CUDA tensor")
    return t.data_ptr()


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


class Workspace:
    """Device scratch for the stage entry points (moea_workspace)."""

    def __init__(self, max_points: int, max_objectives: int, max_directions: int,
                 device: int | None = None):
        self.device = torch.cuda.current_device() if device is None else device
        h = ctypes.c_void_p()
        check(lib().moea_workspace_create(self.device, max_points, max_objectives,
                                          max_directions, ctypes.byref(h)))
        self.handle = h

    @property
    def nbytes(self) -> int:
        return int(lib().moea_workspace_bytes(self.handle))

    def set_peel(self, general: bool) -> None:
        """True: every sort takes the general peel; False: the automatic choice."""
        check(lib().moea_workspace_set_peel(self.handle, 1 if general else 0))

    def set_tiles(self, word: bool) -> None:
        """True: every sort builds its dominance rows from the per-word tables;
        False: from the block prefix sets (the default)."""
        check(lib().moea_workspace_set_tiles(self.handle, 1 if word else 0))

    def close(self) -> None:
        if getattr(self, "handle", None) is not None and self.handle.value:
            lib().moea_workspace_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ndsort(ws: Workspace, cv: torch.Tensor, objs: torch.Tensor, target: int):
    """Fronts (int32, -1 past the stop rule) and the last front index."""
    M, n = objs.shape
    fronts = torch.empty(n, dtype=torch.int32, device=objs.device)
    mf = ctypes.c_int(0)
    check(lib().moea_ndsort(ws.handle, _p(cv), _p(objs), M, n, target, _p(fronts),
                            ctypes.byref(mf), _stream()))
    return fronts, int(mf.value)


def nds_extract(ws: Workspace, fronts: torch.Tensor, max_front: int, N: int):
    n = fronts.numel()
    gidx = torch.empty(n, dtype=torch.int32, device=fronts.device)
    sizes = torch.empty(4, dtype=torch.int32, device=fronts.device)
    mf = torch.tensor([max_front], dtype=torch.int32, device=fronts.device)
    check(lib().moea_nds_extract(ws.handle, _p(fronts), n, _p(mf), N, _p(gidx), _p(sizes), _stream()))
    return gidx, sizes


def ideal_point(ws: Workspace, objs: torch.Tensor) -> torch.Tensor:
    M, n = objs.shape
    out = torch.empty(M, dtype=torch.float32, device=objs.device)
    check(lib().moea_ideal_point(ws.handle, _p(objs), M, n, _p(out), _stream()))
    return out


def normalize(ws: Workspace, objs: torch.Tensor, ideal: torch.Tensor):
    """Returns (normalised objectives, reciprocal intercepts, extreme indices)."""
    f = objs.clone()
    M, n = f.shape
    rcp = torch.empty(M, dtype=torch.float32, device=f.device)
    ext = torch.empty(M, dtype=torch.int32, device=f.device)
    check(lib().moea_normalize(ws.handle, _p(f), _p(ideal), M, n, _p(rcp), _p(ext), _stream()))
    return f, rcp, ext


ASSOC_TREE = 0    # cone-tree search (default)
ASSOC_SCAN = 1    # every direction visited
ASSOC_TENSOR = 2  # dots on the tensor cores, exact FP32 re-score of the candidates


def _check_association(x: torch.Tensor, refs: torch.Tensor) -> None:
    """Points (M,n) and directions (M,H): both FP32 matrices with the same M
    on the same device (the kernels read M rows of each)."""
    if x.dtype != torch.float32 or refs.dtype != torch.float32:
        raise ValueError("points and directions must be float32")
    if x.dim() != 2 or refs.dim() != 2:
        raise ValueError("points (M, n) and directions (M, H) must be matrices")
    if refs.shape[0] != x.shape[0]:
        raise ValueError(f"directions have {refs.shape[0]} rows for {x.shape[0]} objectives")
    if x.device != refs.device:
        raise ValueError("points and directions must be on the same device")


def associate(ws: Workspace, x: torch.Tensor, refs: torch.Tensor, mode: int = ASSOC_TREE):
    _check_association(x, refs)
    M, n = x.shape
    idx = torch.empty(n, dtype=torch.int32, device=x.device)
    dist = torch.empty(n, dtype=torch.float32, device=x.device)
    check(lib().moea_associate(ws.handle, _p(x), _p(refs), M, n, refs.shape[1], _p(idx),
                               _p(dist), mode, _stream()))
    return idx, dist


def associate_static(x: torch.Tensor, refs: torch.Tensor):
    """Full-scan association through the allocation-free entry point."""
    _check_association(x, refs)
    M, n = x.shape
    idx = torch.empty(n, dtype=torch.int32, device=x.device)
    dist = torch.empty(n, dtype=torch.float32, device=x.device)
    check(lib().moea_associate_static(_p(x), _p(refs), M, n, refs.shape[1], _p(idx), _p(dist),
                                      _stream()))
    return idx, dist


def niching(ws: Workspace, seed: int, offset: int, nds_gidx, dist, idx, sizes, H: int, N: int):
    sel = torch.empty(N, dtype=torch.int32, device=dist.device)
    off = ctypes.c_uint64(offset)
    check(lib().moea_niching(ws.handle, seed, ctypes.byref(off), _p(nds_gidx), _p(dist), _p(idx),
                             _p(sizes), H, N, _p(sel), _stream()))
    return sel, int(off.value)


def nsga3_select(ws: Workspace, mix_cv, mix_objs, refs, seed: int, offset: int, ideal_last,
                 assoc_mode: int = 0):
    M, n_mix = mix_objs.shape
    N = n_mix // 2
    surv = torch.empty(N, dtype=torch.int32, device=mix_objs.device)
    fr = torch.empty(N, dtype=torch.int32, device=mix_objs.device)
    sizes = torch.empty(4, dtype=torch.int32, device=mix_objs.device)
    ideal = ideal_last.clone()
    off = ctypes.c_uint64(offset)
    check(lib().moea_nsga3_select(ws.handle, _p(mix_cv), _p(mix_objs), M, N, _p(refs), refs.shape[1],
                                  seed, ctypes.byref(off), _p(ideal), _p(surv), _p(fr), _p(sizes),
                                  assoc_mode, _stream()))
    return dict(survivors=surv, fronts=fr, sizes=sizes, ideal=ideal, offset=int(off.value))


def quantize_cv(cv, eps, clip, log_alpha, bins):
    out = torch.empty_like(cv)
    check(lib().moea_quantize_cv(_p(cv), _p(out), cv.numel(), eps, clip, log_alpha, bins, _stream()))
    return out


def rvea_translate(ws, objs):
    M, n = objs.shape
    out = torch.empty_like(objs)
    z = torch.empty(M, dtype=torch.float32, device=objs.device)
    check(lib().moea_rvea_translate(ws.handle, _p(objs), M, n, _p(out), _p(z), _stream()))
    return out, z


def rvea_partition(ws, t, refs, n_active, n_parent):
    M, n = t.shape
    theta = torch.empty(n, dtype=torch.float32, device=t.device)
    idx = torch.empty(n, dtype=torch.int32, device=t.device)
    check(lib().moea_rvea_partition(ws.handle, _p(t), _p(refs), M, n, refs.shape[1], n_active,
                                    n_parent, _p(theta), _p(idx), _stream()))
    return theta, idx


def rvea_gamma(ws, refs):
    M, K = refs.shape
    g = torch.empty(K, dtype=torch.float32, device=refs.device)
    check(lib().moea_rvea_gamma(ws.handle, _p(refs), M, K, _p(g), _stream()))
    return g


def rvea_apd(ws, t, theta, gamma, idx, gen, max_gen, alpha):
    M, n = t.shape
    out = torch.empty(n, dtype=torch.float32, device=t.device)
    check(lib().moea_rvea_apd(ws.handle, _p(t), _p(theta), _p(gamma), _p(idx), M, n, gamma.numel(),
                              gen, max_gen, alpha, _p(out), _stream()))
    return out


def rvea_elitism(ws, idx, cv, apd, N, K):
    sel = torch.empty(N, dtype=torch.int32, device=idx.device)
    act = ctypes.c_int(0)
    check(lib().moea_rvea_elitism(ws.handle, _p(idx), _p(cv), _p(apd), N, idx.numel(), K, _p(sel),
                                  ctypes.byref(act), _stream()))
    return sel[: act.value].clone(), int(act.value)


def rvea_adapt(ws, v0, objs, n_active):
    M, K = v0.shape
    out = torch.empty_like(v0)
    check(lib().moea_rvea_adapt(ws.handle, _p(v0), _p(objs), M, K, n_active, objs.shape[1],
                                _p(out), _stream()))
    return out


def tournament(cand, rank, cv):
    w = torch.empty(cand.shape[0], dtype=torch.int32, device=cand.device)
    check(lib().moea_tournament(_p(cand), _p(rank), _p(cv), cand.shape[0], _p(w), _stream()))
    return w


def sbx(parents, pidx, bounds, u, sign, copy, eta, prob, copy_prob, n_off):
    D = parents.shape[1]
    off = torch.empty((n_off, D), dtype=torch.float32, device=parents.device)
    check(lib().moea_sbx(_p(parents), _p(pidx), _p(bounds), _p(u), _p(sign), _p(copy), _p(off), eta,
                         prob, copy_prob, n_off, D, _stream()))
    return off


def pm(off, bounds, u, eta, prob):
    out = off.clone()
    n, D = out.shape
    check(lib().moea_pm(_p(out), _p(bounds), _p(u), eta, prob, n, D, _stream()))
    return out


def reproduce(parents, parent_cv, rank, active, bounds, n_off, *, mating=1, sbx_eta=30.0,
              sbx_prob=1.0, sbx_copy_prob=0.0, mutate=1, pm_eta=20.0, pm_prob=1.0, seed=0,
              generation=0):
    n_par, D = parents.shape
    off = torch.empty((n_off, D), dtype=torch.float32, device=parents.device)
    pidx = torch.empty(n_off, dtype=torch.int32, device=parents.device)
    check(lib().moea_reproduce(_p(parents), _p(parent_cv), _p(rank), active, _p(bounds), _p(off),
                               _p(pidx), n_par, n_off, D, mating, sbx_eta, sbx_prob, sbx_copy_prob,
                               mutate, pm_eta, pm_prob, seed, generation, _stream()))
    return off, pidx


def rng_blocks(seed: int, generation: int, tag: int, count: int, device=None):
    out = torch.empty((count, 4), dtype=torch.int32, device=device or "cuda")
    check(lib().moea_rng_blocks(seed, generation, tag, count, _p(out), _stream()))
    return out


def problem_evaluate(kind: int, x: torch.Tensor, M: int):
    N, D = x.shape
    objs = torch.empty((M, N), dtype=torch.float32, device=x.device)
    cv = torch.empty(N, dtype=torch.float32, device=x.device)
    check(lib().moea_problem_evaluate(kind, _p(x), N, D, M, _p(objs), _p(cv), _stream()))
    return objs, cv


def reference_directions(mode: int, n: int, M: int) -> torch.Tensor:
    """Das-Dennis directions on the host, objective-major (M, count)."""
    count = ctypes.c_int(0)
    check(lib().moea_reference_directions(mode, n, M, None, 0, ctypes.byref(count)))
    out = torch.empty((M, count.value), dtype=torch.float32)
    buf = ctypes.cast(out.data_ptr(), ctypes.POINTER(ctypes.c_float))
    check(lib().moea_reference_directions(mode, n, M, buf, out.numel(), ctypes.byref(count)))
    return out
