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
        }
        for name, args in sig.items():
            f = getattr(L, name)
            f.restype = c_int
            f.argtypes = args
        _lib = L
    return _lib


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
