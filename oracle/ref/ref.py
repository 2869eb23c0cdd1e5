"""ctypes wrapper of oracle/_ref/libmoea_ref.so -- TEST INFRASTRUCTURE ONLY.

libmoea_ref.so is CUDA-MOEA's own stage code (built by oracle/ref/Makefile
from the reference sources) behind the C entry points of ref_harness.cu.
Used only by tests and by tests/golden/make_golden.py to obtain the
reference's outputs on given inputs.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np
import torch

LIB_PATH = Path(__file__).resolve().parents[1] / "_ref" / "libmoea_ref.so"
_lib = None
vp, c_int, c_float, c_u64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_uint64


def available() -> bool:
    return LIB_PATH.exists()


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(str(LIB_PATH))
        ip = ctypes.POINTER(c_int)
        sig = {
            "ref_ndsort": [vp, vp, c_int, c_int, c_int, vp, ip],
            "ref_normalize": [vp, vp, c_int, c_int, vp],
            "ref_associate": [vp, vp, c_int, c_int, c_int, vp, vp],
            "ref_niching": [c_u64, ctypes.POINTER(c_u64), vp, vp, vp, ip, c_int, c_int, vp],
            "ref_problem": [c_int, vp, c_int, c_int, c_int, vp, vp],
            "ref_rvea_translate": [vp, c_int, c_int, vp, vp],
            "ref_rvea_partition": [vp, vp, c_int, c_int, c_int, c_int, c_int, vp, vp],
            "ref_rvea_gamma": [vp, c_int, c_int, vp],
            "ref_rvea_apd": [vp, vp, vp, vp, c_int, c_int, c_int, c_int, c_int, c_float, vp],
            "ref_rvea_elitism": [vp, vp, vp, c_int, c_int, c_int, vp, ip],
            "ref_quantize_cv": [vp, vp, c_int, c_float, c_float, c_float, c_int],
            "ref_rvea_adapt": [vp, vp, c_int, c_int, c_int, c_int, vp],
            "ref_sbx": [vp, vp, vp, vp, vp, vp, vp, c_float, c_float, c_float, c_int, c_int],
            "ref_pm": [vp, vp, vp, c_float, c_float, c_int, c_int],
            "ref_tournament": [vp, vp, vp, c_int, vp],
            "ref_rvea_update": [vp, vp, vp, vp, vp, vp, vp, c_int, c_int, c_int, c_int, vp, vp, vp],
        }
        for name, args in sig.items():
            f = getattr(L, name)
            f.restype = c_int
            f.argtypes = args
        L.ref_set_repeat.restype = None
        L.ref_set_repeat.argtypes = [c_int]
        L.ref_last_ms.restype = c_float
        L.ref_last_ms.argtypes = []
        L.ref_annealed.restype = c_float
        L.ref_annealed.argtypes = [c_float, c_float, c_int, c_int]
        _lib = L
    return _lib


HOST_LIB_PATH = LIB_PATH.parent / "libmoea_ref_host.so"
_host = None


def host_available() -> bool:
    return HOST_LIB_PATH.exists()


def host_lib():
    """The reference's host-side direction generators (no CUDA runtime needed)."""
    global _host
    if _host is None:
        L = ctypes.CDLL(str(HOST_LIB_PATH))
        L.ref_directions.restype = c_int
        L.ref_directions.argtypes = [c_int, c_int, c_int, vp, ctypes.c_size_t]
        _host = L
    return _host


def directions(mode, n, M):
    """Normalised directions (M, count) from the reference's generators: mode 0
    NSGA-III auto layers, 1 NSGA-III by partitions, 2 RVEA auto layers."""
    count = host_lib().ref_directions(mode, n, M, None, 0)
    if count < 0:
        raise ValueError("reference generator rejected the request")
    out = np.zeros((M, count), np.float32)
    host_lib().ref_directions(mode, n, M, out.ctypes.data, out.size)
    return out


_LIVE: list = []


def _d(a, dtype=None):
    """Device copy of a, kept alive until the current call has returned (the
    pointer is handed to C; a temporary tensor would go back to the caching
    allocator immediately and the next argument could reuse its memory)."""
    t = torch.from_numpy(np.ascontiguousarray(a))
    t = (t.to(dtype) if dtype else t).cuda()
    _LIVE.append(t)
    return t


def _chk(rc):
    torch.cuda.synchronize()
    _LIVE.clear()
    if rc != 0:
        raise RuntimeError("reference stage failed")


def ndsort(cv, objs, N):
    M, n = objs.shape
    fr = torch.empty(n, dtype=torch.int32, device="cuda")
    mf = c_int(0)
    _chk(lib().ref_ndsort(_d(cv).data_ptr(), _d(objs).data_ptr(), M, n, N, fr.data_ptr(), ctypes.byref(mf)))
    return fr.cpu().numpy(), mf.value


def normalize(f, ideal):
    M, n = f.shape
    t = _d(f)
    rcp = torch.empty(M, dtype=torch.float32, device="cuda")
    _chk(lib().ref_normalize(t.data_ptr(), _d(ideal).data_ptr(), M, n, rcp.data_ptr()))
    return t.cpu().numpy(), rcp.cpu().numpy()


def associate(x, refs):
    M, n = x.shape
    idx = torch.empty(n, dtype=torch.int32, device="cuda")
    dist = torch.empty(n, dtype=torch.float32, device="cuda")
    _chk(lib().ref_associate(_d(x).data_ptr(), _d(refs).data_ptr(), M, n, refs.shape[1],
                             idx.data_ptr(), dist.data_ptr()))
    return idx.cpu().numpy(), dist.cpu().numpy()


def niching(seed, offset, gidx, dist, idx, sizes, H, N):
    sel = torch.zeros(N, dtype=torch.int32, device="cuda")
    off = c_u64(offset)
    hs = (c_int * 4)(*[int(v) for v in sizes])
    _chk(lib().ref_niching(seed, ctypes.byref(off), _d(gidx).data_ptr(), _d(dist).data_ptr(),
                           _d(idx).data_ptr(), hs, H, N, sel.data_ptr()))
    return sel.cpu().numpy(), off.value


def problem(kind, x, M):
    N, D = x.shape
    objs = torch.empty((M, N), dtype=torch.float32, device="cuda")
    cv = torch.empty(N, dtype=torch.float32, device="cuda")
    _chk(lib().ref_problem(kind, _d(x).data_ptr(), N, D, M, objs.data_ptr(), cv.data_ptr()))
    return objs.cpu().numpy(), cv.cpu().numpy()


def rvea_translate(objs):
    M, n = objs.shape
    out = torch.empty((M, n), dtype=torch.float32, device="cuda")
    z = torch.empty(M, dtype=torch.float32, device="cuda")
    _chk(lib().ref_rvea_translate(_d(objs).data_ptr(), M, n, out.data_ptr(), z.data_ptr()))
    return out.cpu().numpy(), z.cpu().numpy()


def rvea_partition(t, refs, n_active, n_parent):
    M, n = t.shape
    th = torch.empty(n, dtype=torch.float32, device="cuda")
    idx = torch.empty(n, dtype=torch.int32, device="cuda")
    _chk(lib().ref_rvea_partition(_d(t).data_ptr(), _d(refs).data_ptr(), M, n, refs.shape[1], n_active,
                                  n_parent, th.data_ptr(), idx.data_ptr()))
    return th.cpu().numpy(), idx.cpu().numpy()


def rvea_gamma(refs):
    M, K = refs.shape
    g = torch.empty(K, dtype=torch.float32, device="cuda")
    _chk(lib().ref_rvea_gamma(_d(refs).data_ptr(), M, K, g.data_ptr()))
    return g.cpu().numpy()


def rvea_apd(t, theta, gamma, idx, gen, max_gen, alpha):
    M, n = t.shape
    out = torch.empty(n, dtype=torch.float32, device="cuda")
    _chk(lib().ref_rvea_apd(_d(t).data_ptr(), _d(theta).data_ptr(), _d(gamma).data_ptr(), _d(idx).data_ptr(),
                            M, n, len(gamma), gen, max_gen, alpha, out.data_ptr()))
    return out.cpu().numpy()


def rvea_elitism(idx, cv, apd, N, K):
    sel = torch.zeros(N, dtype=torch.int32, device="cuda")
    act = c_int(0)
    _chk(lib().ref_rvea_elitism(_d(idx).data_ptr(), _d(cv).data_ptr(), _d(apd).data_ptr(), N, len(idx), K,
                                sel.data_ptr(), ctypes.byref(act)))
    return np.sort(sel.cpu().numpy()[: act.value]), act.value


def quantize_cv(cv, eps, clip, log_alpha, bins):
    out = torch.empty(len(cv), dtype=torch.float32, device="cuda")
    _chk(lib().ref_quantize_cv(_d(cv).data_ptr(), out.data_ptr(), len(cv), eps, clip, log_alpha, bins))
    return out.cpu().numpy()


def rvea_adapt(v0, objs, n_active):
    M, K = v0.shape
    out = torch.empty((M, K), dtype=torch.float32, device="cuda")
    _chk(lib().ref_rvea_adapt(_d(v0).data_ptr(), _d(objs).data_ptr(), M, K, n_active, objs.shape[1],
                              out.data_ptr()))
    return out.cpu().numpy()


def annealed(begin, end, generation, total):
    return lib().ref_annealed(begin, end, generation, total)


def sbx_t(parents, pidx, bounds, u, sign, copy, eta, prob, copy_prob, n_off):
    """SBX with device tensors in and out (large populations stay on the GPU)."""
    D = parents.shape[1]
    off = torch.empty((n_off, D), dtype=torch.float32, device=parents.device)
    rc = lib().ref_sbx(parents.data_ptr(), pidx.data_ptr(), bounds.data_ptr(), u.data_ptr(), sign.data_ptr(),
                       copy.data_ptr(), off.data_ptr(), eta, prob, copy_prob, n_off, D)
    _chk(rc)
    return off


def pm_t(off, bounds, u, eta, prob):
    """Polynomial mutation of a device tensor in place."""
    n, D = off.shape
    _chk(lib().ref_pm(off.data_ptr(), bounds.data_ptr(), u.data_ptr(), eta, prob, n, D))
    return off


def sbx(parents, pidx, bounds, u, sign, copy, eta, prob, copy_prob, n_off):
    out = sbx_t(_d(parents), _d(pidx), _d(bounds), _d(u), _d(sign), _d(copy), eta, prob, copy_prob, n_off)
    return out.cpu().numpy()


def pm(off, bounds, u, eta, prob):
    t = _d(off).clone()
    return pm_t(t, _d(bounds), _d(u), eta, prob).cpu().numpy()


def tournament(cand, rank, cv):
    n = cand.shape[0]
    w = torch.empty(n, dtype=torch.int32, device="cuda")
    _chk(lib().ref_tournament(_d(cand).data_ptr(), _d(rank).data_ptr(), _d(cv).data_ptr(), n, w.data_ptr()))
    return w.cpu().numpy()


def problem_t(kind, x, M):
    """Objectives (M,N) and violation (N) of device variables x (N,D)."""
    N, D = x.shape
    objs = torch.empty((M, N), dtype=torch.float32, device=x.device)
    cv = torch.empty(N, dtype=torch.float32, device=x.device)
    _chk(lib().ref_problem(kind, x.data_ptr(), N, D, M, objs.data_ptr(), cv.data_ptr()))
    return objs, cv


def rvea_update_t(par_x, off_x, par_f, off_f, par_cv, off_cv, sel, active):
    """The reference's RVEA merge + survivor update on device tensors: the next
    population's variables (N,D), objectives (M,N) and violations (N)."""
    N, D = par_x.shape
    M = par_f.shape[0]
    nx = torch.empty_like(par_x)
    nf = torch.empty_like(par_f)
    nc = torch.empty_like(par_cv)
    s = sel.clone()
    _chk(lib().ref_rvea_update(par_x.data_ptr(), off_x.data_ptr(), par_f.data_ptr(), off_f.data_ptr(),
                               par_cv.data_ptr(), off_cv.data_ptr(), s.data_ptr(), active, N, D, M,
                               nx.data_ptr(), nf.data_ptr(), nc.data_ptr()))
    return nx, nf, nc


def set_repeat(repeat: int) -> None:
    """Timing mode of the stage calls: after the call that produces the
    outputs, `repeat` more calls between CUDA events (0 = off)."""
    lib().ref_set_repeat(repeat)


def last_ms() -> float:
    """Mean device time of the repeats of the last stage call (timing mode)."""
    return float(lib().ref_last_ms())


ALGO_LIB_PATH = LIB_PATH.parent / "libmoea_ref_algo.so"


def algo_available() -> bool:
    return ALGO_LIB_PATH.exists()


def algo_time(algorithm, problem_kind, D, M, N, partitions, max_gen, sparse_ratio, seed, warmup, steps):
    """Per-step times (ms) of the reference's own algorithm on the GPU
    (EvolutionaryAlgorithm::step, each step bracketed by device synchronises)."""
    L = ctypes.CDLL(str(ALGO_LIB_PATH))
    L.ref_algo_time.restype = c_int
    L.ref_algo_time.argtypes = [c_int, c_int, c_int, c_int, c_int, c_int, c_int, c_float, ctypes.c_ulonglong,
                                c_int, c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_char_p, ctypes.c_size_t]
    ms = (ctypes.c_double * max(1, steps))()
    err = ctypes.create_string_buffer(512)
    rc = L.ref_algo_time(algorithm, problem_kind, D, M, N, partitions, max_gen, sparse_ratio, seed, warmup, steps,
                         ms, err, 512)
    if rc != 0:
        raise RuntimeError(f"reference algorithm failed ({rc}): {err.value.decode(errors='replace')}")
    return [ms[i] for i in range(steps)]


def algo_run(algorithm, problem_kind, D, M, N, max_gen, seed, sbx_eta, copy_prob, init, dirs=None, frequency=0.1):
    """One run of the reference's own algorithm (see ref_algo_run): final
    objectives (M, N), active count and its RunResult.total_ms."""
    L = ctypes.CDLL(str(ALGO_LIB_PATH))
    fp = ctypes.POINTER(c_float)
    L.ref_algo_run.restype = c_int
    L.ref_algo_run.argtypes = [c_int, c_int, c_int, c_int, c_int, c_int, ctypes.c_ulonglong, c_float, c_float, fp,
                               fp, c_int, c_float, fp, ctypes.POINTER(c_int), ctypes.POINTER(ctypes.c_double),
                               ctypes.c_char_p, ctypes.c_size_t]
    init = np.ascontiguousarray(init, np.float32)
    objs = np.zeros((M, N), np.float32)
    act, ms = c_int(0), ctypes.c_double(0.0)
    err = ctypes.create_string_buffer(512)
    H = 0
    dptr = None
    if dirs is not None:
        dirs = np.ascontiguousarray(dirs, np.float32)
        H = dirs.shape[1]
        dptr = dirs.ctypes.data_as(fp)
    rc = L.ref_algo_run(algorithm, problem_kind, D, M, N, max_gen, seed, sbx_eta, copy_prob, init.ctypes.data_as(fp),
                        dptr, H, frequency, objs.ctypes.data_as(fp), ctypes.byref(act), ctypes.byref(ms), err, 512)
    if rc != 0:
        raise RuntimeError(f"reference algorithm failed ({rc}): {err.value.decode(errors='replace')}")
    return objs, act.value, ms.value
