"""ctypes/numpy wrapper of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

The oracle restates the CUDA-MOEA hot path on the CPU (see moea_oracle.c).  It
is the checker for the CUDA kernels: only tests/, the smoke check and the
CPU-baseline leg of bench.py import this module.  The product never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB_PATH = _HERE / "_build" / "libmoea_oracle.so"
_lib = None

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_c_int, _c_u64, _c_f = ctypes.c_int, ctypes.c_uint64, ctypes.c_float


def build() -> Path:
    """Compile the oracle (gcc + OpenMP) if the shared object is missing or stale."""
    src = [_HERE / "moea_oracle.c", _HERE / "moea_oracle.h"]
    if _LIB_PATH.exists() and all(_LIB_PATH.stat().st_mtime >= s.stat().st_mtime for s in src):
        return _LIB_PATH
    subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(_LIB_PATH))
        L.orc_splitmix_u32.restype = ctypes.c_uint32
        L.orc_splitmix_u32.argtypes = [_c_u64, _c_u64]
        L.orc_derive_seed.restype = _c_u64
        L.orc_derive_seed.argtypes = [_c_u64]
        L.orc_philox4x32_10.argtypes = [_u32p, _u32p, _u32p]
        L.orc_philox_stream.argtypes = [_c_u64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int64, _u32p]
        L.orc_dominates.restype = _c_int
        L.orc_dominates.argtypes = [_f32p, _f32p, _c_int, _c_int, _c_int, _c_int]
        L.orc_ndsort.restype = _c_int
        L.orc_ndsort.argtypes = [_f32p, _f32p, _c_int, _c_int, _c_int, _i32p]
        L.orc_nds_extract.argtypes = [_i32p, _c_int, _c_int, _c_int, _i32p, _i32p]
        L.orc_ideal_point.argtypes = [_f32p, _c_int, _c_int, _f32p]
        L.orc_normalize.restype = _c_int
        L.orc_normalize.argtypes = [_f32p, _f32p, _c_int, _c_int, _f32p, _i32p]
        L.orc_associate.argtypes = [_f32p, _f32p, _c_int, _c_int, _c_int, _i32p, _f32p]
        L.orc_niching.argtypes = [_c_u64, ctypes.POINTER(_c_u64), _i32p, _f32p, _i32p, _i32p,
                                  _c_int, _c_int, _i32p]
        L.orc_nsga3_select.restype = _c_int
        L.orc_nsga3_select.argtypes = [_f32p, _f32p, _c_int, _c_int, _f32p, _c_int, _c_u64,
                                       ctypes.POINTER(_c_u64), _f32p, ctypes.c_void_p, _i32p,
                                       _i32p, _i32p]
        L.orc_quantize_cv.argtypes = [_f32p, _f32p, _c_int, _c_f, _c_f, _c_f, _c_int]
        L.orc_rvea_translate.argtypes = [_f32p, _c_int, _c_int, _f32p, _f32p]
        L.orc_rvea_partition.argtypes = [_f32p, _f32p, _c_int, _c_int, _c_int, _c_int, _c_int,
                                         _f32p, _i32p]
        L.orc_rvea_gamma.argtypes = [_f32p, _c_int, _c_int, _f32p]
        L.orc_rvea_apd.argtypes = [_f32p, _f32p, _f32p, _i32p, _c_int, _c_int, _c_int, _c_int,
                                   _c_int, _c_f, _f32p]
        L.orc_rvea_elitism.restype = _c_int
        L.orc_rvea_elitism.argtypes = [_i32p, _f32p, _f32p, _c_int, _c_int, _c_int, _i32p]
        L.orc_rvea_adapt.argtypes = [_f32p, _f32p, _c_int, _c_int, _c_int, _c_int, _f32p]
        L.orc_tournament.argtypes = [_i32p, _i32p, _f32p, _c_int, _i32p]
        L.orc_annealed.restype = _c_f
        L.orc_annealed.argtypes = [_c_f, _c_f, _c_int, _c_int]
        L.orc_sbx.argtypes = [_f32p, _i32p, _f32p, _f32p, _i32p, _f32p, _f32p, _c_f, _c_f, _c_f,
                              _c_int, _c_int]
        L.orc_pm.argtypes = [_f32p, _f32p, _f32p, _c_f, _c_f, _c_int, _c_int]
        L.orc_problem_evaluate.restype = _c_int
        L.orc_problem_evaluate.argtypes = [_c_int, _f32p, _c_int, _c_int, _c_int, _f32p, _f32p,
                                           _c_int]
        L.orc_reference_directions.restype = _c_int
        L.orc_reference_directions.argtypes = [_c_int, _c_int, _c_int, ctypes.c_void_p]
        _lib = L
    return _lib


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def set_threads(n: int) -> None:
    os.environ["OMP_NUM_THREADS"] = str(n)


# ---------------------------------------------------------------- RNG
def splitmix_u32(counter: int, seed: int) -> int:
    return lib().orc_splitmix_u32(counter, seed)


def derive_seed(seed: int) -> int:
    return lib().orc_derive_seed(seed)


def philox(ctr, key) -> np.ndarray:
    out = np.zeros(4, np.uint32)
    lib().orc_philox4x32_10(np.asarray(ctr, np.uint32), np.asarray(key, np.uint32), out)
    return out


def philox_stream(seed: int, generation: int, tag: int, count: int) -> np.ndarray:
    out = np.zeros((count, 4), np.uint32)
    lib().orc_philox_stream(seed, generation, tag, count, out)
    return out


# ---------------------------------------------------------------- NSGA-III stages
def dominates(cv, objs, p, q) -> bool:
    objs = _f32(objs)
    M, n = objs.shape
    return lib().orc_dominates(_f32(cv), objs, M, n, p, q) == 1


def ndsort(cv, objs, target):
    objs = _f32(objs)
    M, n = objs.shape
    fronts = np.zeros(n, np.int32)
    mf = lib().orc_ndsort(_f32(cv), objs, M, n, target, fronts)
    return fronts, mf


def nds_extract(fronts, max_front, N):
    fronts = _i32(fronts)
    gidx = np.zeros(len(fronts), np.int32)
    sizes = np.zeros(4, np.int32)
    lib().orc_nds_extract(fronts, len(fronts), max_front, N, gidx, sizes)
    return gidx[: sizes[3]].copy(), sizes


def ideal_point(objs):
    objs = _f32(objs)
    out = np.zeros(objs.shape[0], np.float32)
    lib().orc_ideal_point(objs, objs.shape[0], objs.shape[1], out)
    return out


def normalize(objs_nds, ideal):
    f = _f32(objs_nds).copy()
    M, n = f.shape
    rcp = np.zeros(M, np.float32)
    ext = np.zeros(M, np.int32)
    ill = lib().orc_normalize(f, _f32(ideal), M, n, rcp, ext)
    return f, rcp, ext, ill


def associate(x, refs):
    x = _f32(x)
    refs = _f32(refs)
    M, n = x.shape
    idx = np.zeros(n, np.int32)
    dist = np.zeros(n, np.float32)
    lib().orc_associate(x, refs, M, n, refs.shape[1], idx, dist)
    return idx, dist


def niching(seed, offset, nds_gidx, dist, idx, sizes, H, N):
    off = _c_u64(offset)
    sel = np.zeros(N, np.int32)
    g = _i32(nds_gidx) if len(nds_gidx) else np.zeros(1, np.int32)
    d = _f32(dist) if len(dist) else np.zeros(1, np.float32)
    i = _i32(idx) if len(idx) else np.zeros(1, np.int32)
    lib().orc_niching(seed, ctypes.byref(off), g, d, i, _i32(sizes), H, N, sel)
    return sel, off.value


def nsga3_select(mix_cv, mix_objs, refs, seed, offset, ideal_last):
    mix_objs = _f32(mix_objs)
    M, n_mix = mix_objs.shape
    N = n_mix // 2
    refs = _f32(refs)
    ideal = _f32(ideal_last).copy()
    off = _c_u64(offset)
    surv = np.zeros(N, np.int32)
    fr = np.zeros(N, np.int32)
    sizes = np.zeros(4, np.int32)
    mf = lib().orc_nsga3_select(_f32(mix_cv), mix_objs, M, N, refs, refs.shape[1], seed,
                                ctypes.byref(off), ideal, None, surv, fr, sizes)
    return dict(survivors=surv, fronts=fr, max_front=mf, ideal=ideal, offset=off.value,
                sizes=sizes)


def quantize_cv(cv, eps, clip, log_alpha, bins):
    cv = _f32(cv)
    out = np.zeros_like(cv)
    lib().orc_quantize_cv(cv, out, len(cv), eps, clip, log_alpha, bins)
    return out


# ---------------------------------------------------------------- RVEA stages
def rvea_translate(objs):
    objs = _f32(objs)
    M, n = objs.shape
    out = np.zeros_like(objs)
    z = np.zeros(M, np.float32)
    lib().orc_rvea_translate(objs, M, n, out, z)
    return out, z


def rvea_partition(t, refs, n_active, n_parent):
    t = _f32(t)
    refs = _f32(refs)
    M, n = t.shape
    th = np.zeros(n, np.float32)
    idx = np.zeros(n, np.int32)
    lib().orc_rvea_partition(t, refs, M, n, refs.shape[1], n_active, n_parent, th, idx)
    return th, idx


def rvea_gamma(refs):
    refs = _f32(refs)
    g = np.zeros(refs.shape[1], np.float32)
    lib().orc_rvea_gamma(refs, refs.shape[0], refs.shape[1], g)
    return g


def rvea_apd(t, theta, gamma, idx, gen, max_gen, alpha):
    t = _f32(t)
    M, n = t.shape
    out = np.zeros(n, np.float32)
    lib().orc_rvea_apd(t, _f32(theta), _f32(gamma), _i32(idx), M, n, len(gamma), gen, max_gen,
                       alpha, out)
    return out


def rvea_elitism(idx, cv, apd, N, K):
    sel = np.zeros(N, np.int32)
    act = lib().orc_rvea_elitism(_i32(idx), _f32(cv), _f32(apd), N, len(idx), K, sel)
    return sel[:act].copy(), act


def rvea_adapt(v0, objs, n_active):
    v0 = _f32(v0)
    objs = _f32(objs)
    out = np.zeros_like(v0)
    lib().orc_rvea_adapt(v0, objs, v0.shape[0], v0.shape[1], n_active, objs.shape[1], out)
    return out


# ---------------------------------------------------------------- reproduction
def tournament(cand, rank, cv):
    cand = _i32(cand)
    w = np.zeros(cand.shape[0], np.int32)
    lib().orc_tournament(cand, _i32(rank), _f32(cv), cand.shape[0], w)
    return w


def annealed(b, e, gen, total):
    return lib().orc_annealed(b, e, gen, total)


def sbx(parents, pidx, bounds, u, sign, copy, eta, prob, copy_prob, n_off):
    parents = _f32(parents)
    D = parents.shape[1]
    off = np.zeros((n_off, D), np.float32)
    lib().orc_sbx(parents, _i32(pidx), _f32(bounds), _f32(u), _i32(sign), _f32(copy), off, eta,
                  prob, copy_prob, n_off, D)
    return off


def pm(off, bounds, u, eta, prob):
    off = _f32(off).copy()
    n, D = off.shape
    lib().orc_pm(off, _f32(bounds), _f32(u), eta, prob, n, D)
    return off


# ---------------------------------------------------------------- problems / directions
PROBLEM_KINDS = {"DTLZ1": 1, "DTLZ2": 2, "DTLZ3": 3, "DTLZ4": 4, "DTLZ5": 5, "DTLZ6": 6,
                 "DTLZ7": 7, "ConvexDTLZ2": 8, "C1DTLZ1": 9, "C1DTLZ3": 10, "C2DTLZ2": 11,
                 "C2ConvexDTLZ2": 12, "C3DTLZ1": 13, "C3DTLZ4": 14, "CSDP": 15}


def evaluate(kind, x, M, precision=0):
    x = _f32(x)
    N, D = x.shape
    k = PROBLEM_KINDS[kind] if isinstance(kind, str) else int(kind)
    objs = np.zeros((M, N), np.float32)
    cv = np.zeros(N, np.float32)
    rc = lib().orc_problem_evaluate(k, x, N, D, M, objs, cv, precision)
    if rc != 0:
        raise ValueError("invalid problem configuration")
    return objs, cv


def reference_directions(mode, n_or_partitions, M):
    L = lib()
    count = L.orc_reference_directions(mode, n_or_partitions, M, None)
    if count < 0:
        raise ValueError("invalid reference-direction request")
    out = np.zeros((M, count), np.float32)
    L.orc_reference_directions(mode, n_or_partitions, M, out.ctypes.data_as(ctypes.c_void_p))
    return out
