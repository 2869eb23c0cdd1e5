"""Problem plugins written in C++/CUDA: build, inspect, use.

A plugin implements ``cuda_moea::IProblemEvaluator`` against the plugin SDK
(``sdk_directory()/include``) and registers itself with
``CUDA_MOEA_REGISTER_PROBLEM``; sources written for CUDA-MOEA's SDK build
unchanged.  ``NativeProblem`` builds (or reuses) the library and is passed to
an algorithm like any other problem::

    problem = NativeProblem("path/to/plugin", name="BiSphere", dimension=30,
                            objectives=2, parameters={"radius": 2.0})
    cm.NSGA3(problem=problem, population_size=1024).run()

Command line (same subcommands as the reference's cuda_moea.native):
``python -m cuda_moea.native build SOURCE | inspect LIBRARY | clean | sdk``.
"""
from __future__ import annotations

import argparse
import copy
import ctypes
import json
import math
import struct
import time
from pathlib import Path

from ._lib import MoeaError, check, lib
from ._native_build import build_problem, cache_directory, clear_cache, export_problem, sdk_directory

__all__ = ["NativeProblem", "benchmark", "build_problem", "cache_directory", "clear_cache",
           "export_problem", "sdk_directory", "schema", "main"]


def _open(library: str) -> ctypes.c_void_p:
    handle = ctypes.c_void_p()
    check(lib().moea_native_open(str(library).encode(), ctypes.byref(handle)))
    return handle


def _schema_of(handle) -> dict:
    needed = ctypes.c_size_t(0)
    check(lib().moea_native_schema(handle, None, 0, ctypes.byref(needed)))
    buf = ctypes.create_string_buffer(needed.value)
    check(lib().moea_native_schema(handle, buf, needed.value, ctypes.byref(needed)))
    return json.loads(buf.value.decode())


def schema(library) -> dict:
    """Registered name, build id and parameters ({name: {type, default, description}})."""
    handle = _open(library)
    try:
        return _schema_of(handle)
    finally:
        lib().moea_native_close(handle)


_VALID = {
    "int": lambda v: type(v) is int and -(2 ** 63) <= v < 2 ** 63,
    "float": lambda v: type(v) in (int, float) and math.isfinite(v),
    "bool": lambda v: type(v) is bool,
    "str": lambda v: isinstance(v, str),
    "float_list": lambda v: isinstance(v, (list, tuple)) and all(
        type(x) in (int, float) and math.isfinite(x) for x in v),
}


class NativeProblem:
    """A plugin problem: ``source_dir`` (built on demand, or only looked up
    with ``build="never"``) or a prebuilt ``library``.  ``name`` must be the
    registered name; parameters are checked against the registered schema."""

    def __init__(self, source_dir=None, *, name: str, dimension: int, objectives: int,
                 lower_bounds=0.0, upper_bounds=1.0, parameters=None, library=None, build: str = "auto",
                 **build_options):
        if (source_dir is None) == (library is None):
            raise ValueError("Provide exactly one of source_dir or library")
        if build not in ("auto", "never"):
            raise ValueError("build must be 'auto' or 'never'")
        for key, value in (("dimension", dimension), ("objectives", objectives)):
            if isinstance(value, bool) or not isinstance(value, int) or value <= 0:
                raise ValueError(f"{key} must be a positive integer")
        if not isinstance(name, str) or not name:
            raise ValueError("name must be a nonempty string")
        lower = self._bounds(lower_bounds, dimension)
        upper = self._bounds(upper_bounds, dimension)
        if any(a >= b for a, b in zip(lower, upper)):
            raise ValueError("Each lower bound must be less than its upper bound")
        if library is not None and build_options:
            raise ValueError("Build options are only applicable to source_dir")
        if library is None:
            library = build_problem(source_dir, mode=build, **build_options)
        self.library = Path(library).expanduser().resolve()
        if not self.library.is_file():
            raise FileNotFoundError(self.library)
        self.schema = schema(self.library)
        if self.schema["name"] != name:
            raise ValueError(f"Library registers {self.schema['name']!r}, not {name!r}")
        self._config = {"type": "NativeProblem", "library": str(self.library), "name": name,
                        "dimension": dimension, "objectives": objectives,
                        "lower_bounds": lower, "upper_bounds": upper,
                        "parameters": copy.deepcopy(dict(parameters or {}))}
        for key, value in self._config["parameters"].items():
            if key not in self.schema["parameters"]:
                raise ValueError(f"Unknown native problem parameter: {key}")
            kind = self.schema["parameters"][key]["type"]
            if not _VALID[kind](value):
                raise ValueError(f"Native parameter {key!r} must be {kind}")

    name = property(lambda self: self._config["name"])
    dimension = property(lambda self: self._config["dimension"])
    objectives = property(lambda self: self._config["objectives"])
    lower_bounds = property(lambda self: list(self._config["lower_bounds"]))
    upper_bounds = property(lambda self: list(self._config["upper_bounds"]))
    parameters = property(lambda self: copy.deepcopy(self._config["parameters"]))

    @staticmethod
    def _bounds(value, dimension):
        values = [float(value)] * dimension if isinstance(value, (int, float)) else [float(x) for x in value]
        if len(values) != dimension or not all(math.isfinite(x) and abs(x) <= 3.4028234663852886e38
                                               for x in values):
            raise ValueError("Bounds must be finite float32 values with length dimension")
        return [struct.unpack("f", struct.pack("f", x))[0] for x in values]

    def _spec(self) -> dict:
        return copy.deepcopy(self._config)


class NativeInstance:
    """One constructed plugin problem (the library loaded, the evaluator
    created); closed when garbage-collected.  ``ptr`` is the user pointer of
    the algorithm's evaluate / prepare / reset hooks.  The specification is
    checked again against the library's schema here, since it may have been
    changed after the NativeProblem was made (the reference's bridge does the
    same, python/csrc/native_problem.cpp:38-44, 86-92)."""

    def __init__(self, spec: dict):
        self.handle = _open(spec["library"])
        try:
            kinds = _schema_of(self.handle)["parameters"]
            L = lib()
            for key, value in spec["parameters"].items():
                if key not in kinds:
                    raise ValueError(f"Unknown native problem parameter: {key}")
                kind = kinds[key]["type"]
                if not _VALID[kind](value):
                    raise ValueError(f"Invalid type/value for native parameter '{key}'")
                k = key.encode()
                if kind == "int":
                    check(L.moea_native_set_int(self.handle, k, int(value)))
                elif kind == "float":
                    check(L.moea_native_set_float(self.handle, k, float(value)))
                elif kind == "bool":
                    check(L.moea_native_set_bool(self.handle, k, 1 if value else 0))
                elif kind == "str":
                    check(L.moea_native_set_string(self.handle, k, str(value).encode()))
                else:
                    arr = (ctypes.c_double * len(value))(*[float(x) for x in value])
                    check(L.moea_native_set_floats(self.handle, k, arr, len(value)))
            D = spec["dimension"]
            lo = (ctypes.c_float * D)(*spec["lower_bounds"])
            hi = (ctypes.c_float * D)(*spec["upper_bounds"])
            check(L.moea_native_create(self.handle, spec["name"].encode(), D, spec["objectives"], lo, hi))
            cc = ctypes.c_int(0)
            check(L.moea_native_constraint_count(self.handle, ctypes.byref(cc)))
            self.constraint_count = cc.value
        except Exception:
            lib().moea_native_close(self.handle)
            self.handle = None
            raise
        self.spec = spec

    @property
    def ptr(self) -> int:
        return self.handle.value

    @staticmethod
    def hook(name: str) -> int:
        """Address of one of the library's hook functions."""
        return ctypes.cast(getattr(lib(), name), ctypes.c_void_p).value

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                lib().moea_native_close(h)
            except Exception:
                pass
            self.handle = None


def benchmark(problem: NativeProblem, variables, *, repeats: int = 100, warmup: int = 10) -> dict:
    """Times full evaluations of ``variables`` ((N, D) CUDA float32 tensor),
    excluding loading and construction: ``cuda_ms_per_eval`` from CUDA events
    on the current stream (launch gaps included), ``wall_ms_per_eval`` host
    time including the final wait.  Same keys as the reference's
    benchmark_problem."""
    import torch
    x = variables.to(dtype=torch.float32).contiguous()
    if not x.is_cuda or x.dim() != 2 or x.shape[1] != problem.dimension:
        raise ValueError("variables must be a CUDA (N, dimension) tensor")
    inst = NativeInstance(problem._spec())
    N = x.shape[0]
    objs = torch.empty((problem.objectives, N), dtype=torch.float32, device=x.device)
    cv = torch.empty(N, dtype=torch.float32, device=x.device)
    stream = torch.cuda.current_stream(x.device)

    def once():
        check(lib().moea_native_evaluate(inst.ptr, x.data_ptr(), objs.data_ptr(), cv.data_ptr(), N,
                                         problem.dimension, problem.objectives, 0, 1, stream.cuda_stream))

    with torch.cuda.device(x.device):
        for _ in range(warmup):
            once()
        stream.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record(stream)
        for _ in range(repeats):
            once()
        e1.record(stream)
        e1.synchronize()
        wall = time.perf_counter() - t0
    return {"repeats": repeats, "size": N, "cuda_ms_per_eval": e0.elapsed_time(e1) / repeats,
            "wall_ms_per_eval": 1e3 * wall / repeats}


def main(argv=None) -> None:
    parser = argparse.ArgumentParser(prog="python -m cuda_moea.native", description=__doc__.splitlines()[0])
    sub = parser.add_subparsers(dest="command", required=True)
    b = sub.add_parser("build", help="compile a plugin source directory or reuse its cached build")
    b.add_argument("source_dir")
    b.add_argument("--cache-dir")
    b.add_argument("--architectures")
    b.add_argument("--debug", action="store_true")
    b.add_argument("--force", action="store_true")
    b.add_argument("--verbose", action="store_true")
    b.add_argument("--dependency", action="append", default=[], help="extra include directory")
    b.add_argument("--jobs", type=int)
    b.add_argument("--output", help="also copy the build into this new directory")
    i = sub.add_parser("inspect", help="print a library's registered name and parameters")
    i.add_argument("library")
    c = sub.add_parser("clean", help="remove the cached builds")
    c.add_argument("--cache-dir")
    sub.add_parser("sdk", help="print the SDK directory")
    args = parser.parse_args(argv)
    if args.command == "build":
        path = build_problem(args.source_dir, cache_dir=args.cache_dir, architectures=args.architectures,
                             debug=args.debug, force=args.force, verbose=args.verbose,
                             dependencies=args.dependency, jobs=args.jobs)
        if args.output:
            path = export_problem(path, args.output)
        print(path)
    elif args.command == "inspect":
        print(json.dumps(schema(Path(args.library).expanduser().resolve()), indent=2))
    elif args.command == "clean":
        clear_cache(args.cache_dir)
    else:
        print(sdk_directory())


if __name__ == "__main__":
    try:
        main()
    except (MoeaError, ValueError, FileNotFoundError, RuntimeError) as e:
        raise SystemExit(str(e))
