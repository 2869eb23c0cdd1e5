"""NSGA3 / RVEA / Algorithm / AlgorithmBuilder on libmoea_b200.

Mirrors python/cuda_moea/algorithm.py of CUDA-MOEA: same constructor arguments,
methods and results (``Population``, ``Result`` with zero-copy CUDA tensors;
objectives are a transposed (N, M) view of the objective-major (M, N) buffer,
bindings.cpp:100-146 of the reference).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass
from pathlib import Path
from typing import Any

import torch

from . import _lib
from ._lib import AlgorithmConfig, PopulationViewC, check, lib
from ._specs import (
    AdaptiveRVEADirections, CudaConfig, DasDennisDirections, NSGA3EnvironmentSelector,
    PolynomialMutation, RandomMating, RVEAEnvironmentSelector, SBX, TournamentMating,
    specification,
)
from .problem import DTLZ2, PROBLEM_KINDS

NSGA3_KIND, RVEA_KIND = 0, 1


@dataclass(frozen=True)
class Population:
    variables: Any
    objectives: Any
    constraints: Any


@dataclass(frozen=True)
class Result(Population):
    auxiliary_indices: Any
    active_count: int
    total_ms: float


class _DeviceArray:
    """__cuda_array_interface__ holder; keeps the owning algorithm alive for as
    long as a tensor view of its memory exists."""

    def __init__(self, ptr: int, shape, typestr: str, owner: Any):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr,
                                         "data": (int(ptr), False), "version": 3,
                                         "strides": None}
        self._owner = owner


def _view(ptr: int, shape, dtype: torch.dtype, device: int, owner: Any) -> torch.Tensor:
    n = 1
    for s in shape:
        n *= s
    if n == 0 or not ptr:
        return torch.empty(shape, dtype=dtype, device=f"cuda:{device}")
    typestr = "<f4" if dtype == torch.float32 else "<i4"
    return torch.as_tensor(_DeviceArray(ptr, shape, typestr, owner), device=f"cuda:{device}")


def _float_ptr_array(values):
    if values is None:
        return None, None
    buf = (ctypes.c_float * len(values))(*[float(v) for v in values])
    return buf, ctypes.cast(buf, _lib.fp)


def _device_index(device: int | str) -> int:
    if isinstance(device, int):
        return device
    if device == "cuda":
        return 0
    if device.startswith("cuda:"):
        return int(device.split(":", 1)[1])
    raise ValueError("CUDA-MOEA only supports CUDA devices")


class _Native:
    """Owner of a moea_algorithm handle and of the callbacks it references."""

    def __init__(self, cfg: AlgorithmConfig, keep: list):
        self._keep = keep
        handle = ctypes.c_void_p()
        check(lib().moea_algorithm_create(ctypes.byref(cfg), ctypes.byref(handle)))
        self.handle = handle

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                lib().moea_algorithm_destroy(h)
            except Exception:
                pass
            self.handle = ctypes.c_void_p()


class Algorithm:
    def __init__(self, algorithm: str = "NSGA3", *, population_size: int = 1024,
                 max_generations: int = 100, problem: Any | None = None,
                 mating: Any | None = None, crossover: Any | None = None,
                 mutation: Any | None = None,
                 reference_directions: Any | None = None,
                 environment_selector: Any | None = None,
                 initial_population: Any | None = None,
                 cuda: CudaConfig | None = None, device: int | str | None = None,
                 seed: int | None = None, enable_warmup: bool | None = None,
                 progress_interval: int = 100, print_progress: bool = True,
                 save_data: str | Path | None = None,
                 save_interval: int = 1, use_graphs: bool = True, fuse_small: bool = True) -> None:
        kind = algorithm.upper().replace("-", "")
        if kind not in {"NSGA3", "RVEA"}:
            raise ValueError("algorithm must be 'NSGA3' or 'RVEA'")
        cuda = CudaConfig() if cuda is None else cuda
        if device is not None:
            cuda.device_id = _device_index(device)
        if seed is not None:
            cuda.seed = seed
        if enable_warmup is not None:
            cuda.enable_warmup = enable_warmup
        problem = DTLZ2() if problem is None else problem
        mating = (TournamentMating() if kind == "NSGA3" else RandomMating()) if mating is None else mating
        crossover = SBX() if crossover is None else crossover
        mutation = PolynomialMutation() if mutation is None else mutation
        reference_directions = (DasDennisDirections() if kind == "NSGA3" else AdaptiveRVEADirections()) \
            if reference_directions is None else reference_directions
        environment_selector = (NSGA3EnvironmentSelector() if kind == "NSGA3" else RVEAEnvironmentSelector()) \
            if environment_selector is None else environment_selector
        self._specs = {k: specification(v) for k, v in dict(
            problem=problem, mating=mating, crossover=crossover, mutation=mutation,
            reference_directions=reference_directions,
            environment_selector=environment_selector).items()}
        self._kind = kind
        self._cuda = cuda
        self._population_size = int(population_size)
        self._max_generations = int(max_generations)
        self._progress_interval = progress_interval
        self._print_progress = print_progress
        # snapshots in the reference's data-recorder layout (algorithm_factory.cu:80-86)
        if save_data is not None and not str(save_data):
            raise ValueError("saveData output directory cannot be empty")
        if save_data is not None and int(save_interval) <= 0:
            raise ValueError("saveData generation interval must be positive")
        self._save_data = save_data
        self._save_interval = int(save_interval)
        self._device = int(cuda.device_id)
        self._use_graphs = bool(use_graphs)
        self._fuse_small = bool(fuse_small)
        self._initial = None
        if initial_population is not None:
            t = torch.as_tensor(initial_population).detach().to("cpu", torch.float32).contiguous()
            if t.dim() != 2 or t.shape[0] != population_size:
                raise ValueError("initial_population must have shape (population_size, dimension)")
            self._initial = t
        self._problem_info = self._problem_dims(self._specs["problem"])
        # a plugin problem is constructed with the algorithm, so a plugin that
        # rejects its configuration fails here (as the reference's algorithm
        # constructor does); the instance outlives the algorithm handle
        self._plugin = None
        if self._specs["problem"]["type"] == "NativeProblem":
            from .native import NativeInstance
            self._plugin = NativeInstance(self._specs["problem"])
        self._validate_unsupported()
        self._native: _Native | None = None
        self._stream = None
        self._result_total_ms = 0.0

    # ------------------------------------------------------------------ config
    @staticmethod
    def _problem_dims(p: dict) -> tuple[int, int]:
        t = p["type"]
        if t in ("DTLZProblem",):
            return int(p["dimension"]), int(p["objectives"])
        if t in ("PythonProblem", "NativeProblem"):
            return int(p["dimension"]), int(p["objectives"])
        raise TypeError(f"unsupported problem specification {t}")

    def _validate_unsupported(self) -> None:
        """Python crossover, mutation and environmental selection (and a
        Python direction provider that updates) run through the composed
        step (composed.py): every generation assembled from strategy handles
        and Python objects, as the reference's adapters compose them."""
        from .composed import needs_composition
        self._compose = needs_composition(self._specs)
        self._composed = None
        self._deferred_error = None
        if self._compose and self._save_data is not None:
            self._deferred_error = NotImplementedError(
                "snapshots (save_data) are written by the algorithm object; strategies in Python run "
                "through the composed step, which does not write them")

    def _composed_run(self):
        """The composed step's run object (created on first use)."""
        if self._deferred_error is not None:
            raise self._deferred_error
        if self._composed is None:
            from .composed import ComposedRun
            self._composed = ComposedRun(self)
        return self._composed

    def _build_config(self) -> tuple[AlgorithmConfig, list]:
        keep: list = []
        cfg = AlgorithmConfig()
        sel = self._specs["environment_selector"]
        selector_kind = RVEA_KIND if sel["type"] == "RVEAEnvironmentSelector" else NSGA3_KIND
        lib().moea_algorithm_config_defaults(ctypes.byref(cfg), selector_kind)
        cfg.population_size = self._population_size
        cfg.max_generations = self._max_generations
        cfg.device = self._device
        cfg.seed = int(self._cuda.seed)
        # run on the caller's current torch stream, so tensor views of the
        # population are ordered with the algorithm's kernels; the legacy
        # default stream cannot be captured into a graph, so a dedicated
        # stream (self.stream) is used instead of it
        with torch.cuda.device(self._device):
            cur = torch.cuda.current_stream(self._device)
            if cur.cuda_stream == 0:
                cur = torch.cuda.Stream(self._device)
            self.stream = cur
            cfg.stream = cur.cuda_stream
        cfg.use_graphs = 1 if self._use_graphs else 0
        cfg.fused_small = 1 if self._fuse_small else 0
        if self._save_data is not None:
            directory = os.fsencode(os.fspath(self._save_data))
            keep.append(directory)
            cfg.save_directory = directory
            cfg.save_interval = self._save_interval
        D, M = self._problem_info
        cfg.dimension, cfg.objectives = D, M
        p = self._specs["problem"]
        if p["type"] == "DTLZProblem":
            cfg.problem_kind = PROBLEM_KINDS[p["kind"]]
            cfg.constraint_activation_ratio = float(p["constraint_activation_ratio"])
        elif p["type"] == "NativeProblem":
            # the plugin through the library's own hooks; the instance outlives
            # the algorithm handle (released after it in _Native)
            from .native import NativeInstance
            inst = self._plugin
            keep.append(inst)
            cfg.problem_kind = 0
            lo_buf, lo = _float_ptr_array(p["lower_bounds"])
            hi_buf, hi = _float_ptr_array(p["upper_bounds"])
            keep += [lo_buf, hi_buf]
            cfg.h_lower, cfg.h_upper = lo, hi
            cfg.evaluate = _lib.EVALUATE_FN(NativeInstance.hook("moea_native_evaluate"))
            cfg.prepare = _lib.PREPARE_FN(NativeInstance.hook("moea_native_prepare"))
            cfg.problem_reset = _lib.RESET_FN(NativeInstance.hook("moea_native_reset"))
            cfg.evaluate_user = inst.ptr
            name = p["name"].encode()
            keep.append(name)
            cfg.problem_name = name
            cfg.constraint_count = inst.constraint_count
        else:
            cfg.problem_kind = 0
            lo_buf, lo = _float_ptr_array(p["lower_bounds"])
            hi_buf, hi = _float_ptr_array(p["upper_bounds"])
            keep += [lo_buf, hi_buf]
            cfg.h_lower, cfg.h_upper = lo, hi
            fn = _lib.EVALUATE_FN(self._make_evaluate(p["object"]))
            keep.append(fn)
            cfg.evaluate = fn
            name = str(p.get("name") or "").encode()
            keep.append(name)
            cfg.problem_name = name or None
            cfg.constraint_count = int(p.get("constraints", 0))
        m = self._specs["mating"]
        if m["type"] == "TournamentMating":
            cfg.mating = 1
        elif m["type"] == "RandomMating":
            cfg.mating = 0
        elif m["type"] == "PythonMating":
            cfg.mating = 2
            fn = _lib.MATING_FN(self._make_mating(m["object"]))
            keep.append(fn)
            cfg.mate = fn
        c = self._specs["crossover"]
        if c["type"] == "SBX":
            cfg.sbx_eta_initial = c["eta_initial"]
            cfg.sbx_eta_final = c["eta_final"]
            cfg.sbx_probability = c["probability"]
            cfg.sbx_copy_probability = c["variable_copy_probability"]
        mu = self._specs["mutation"]
        if mu["type"] == "NoMutation":
            cfg.mutation = 0
        elif mu["type"] == "PolynomialMutation":
            cfg.mutation = 1
            cfg.pm_eta_initial = mu["eta_initial"]
            cfg.pm_eta_final = mu["eta_final"]
            cfg.pm_probability = mu["probability"]
        r = self._specs["reference_directions"]
        if r["type"] == "DasDennisDirections":
            if r["partitions"] < 0:
                raise ValueError("Das-Dennis partitions cannot be negative")
            cfg.directions = 0
            cfg.partitions = int(r["partitions"])
        elif r["type"] == "AdaptiveRVEADirections":
            cfg.directions = 1
            cfg.adapt_frequency = float(r["frequency"])
        else:
            if r["type"] == "UserDefinedDirections":
                values = torch.as_tensor(r["values"]).detach().to("cpu", torch.float32)
                normalize = bool(r["normalize"])
            else:  # PythonReferenceDirections
                values = torch.as_tensor(r["object"].initialize(
                    self._population_size, M, {"device": self._device})).detach().to("cpu", torch.float32)
                normalize = True
            if values.dim() != 2 or values.shape[1] != M:
                raise ValueError("User direction objective count does not match the problem")
            om = values.t().contiguous()  # objective-major (M, count)
            keep.append(om)
            cfg.directions = 2
            cfg.h_user_directions = ctypes.cast(om.data_ptr(), _lib.fp)
            cfg.user_direction_count = int(values.shape[0])
            cfg.normalize_user_directions = 1 if normalize else 0
        if sel["type"] == "NSGA3EnvironmentSelector":
            cfg.sparse_ratio = sel["sparse_ratio"]
            cfg.cv_bins = sel["cv_bins"]
            cfg.cv_clip_upper = sel["cv_clip_upper"]
            cfg.cv_log_alpha = sel["cv_log_alpha"]
            cfg.feasibility_epsilon = sel["feasibility_epsilon"]
            cfg.association_mode = sel.get("association_mode", 0)
        elif sel["type"] == "RVEAEnvironmentSelector":
            cfg.rvea_alpha = sel["alpha"]
        if self._initial is not None:
            if self._initial.shape[1] != D:
                raise ValueError("initial_population must have shape (population_size, dimension)")
            keep.append(self._initial)
            cfg.h_initial_population = ctypes.cast(self._initial.data_ptr(), _lib.fp)
        return cfg, keep

    def _make_evaluate(self, problem):
        device = self._device
        me = self

        def evaluate(user, vars_p, objs_p, cv_p, N, D, M, gen, max_gen, stream):
            try:
                with torch.cuda.device(device), torch.cuda.stream(torch.cuda.ExternalStream(stream, device=device)):
                    x = _view(vars_p, (N, D), torch.float32, device, me)
                    out = problem.evaluate(x, {"generation": gen, "max_generations": max_gen,
                                               "device": device})
                    objs = out
                    cons = None
                    if isinstance(out, dict):
                        objs = out["objectives"]
                        cons = out.get("constraints")
                    elif isinstance(out, tuple):
                        objs = out[0]
                        cons = out[1] if len(out) > 1 else None
                    objs = torch.as_tensor(objs).to(torch.float32)
                    if not objs.is_cuda or objs.shape != (N, M):
                        raise ValueError("objectives must have shape (population_size, objective_count)")
                    _view(objs_p, (M, N), torch.float32, device, me).copy_(objs.t())
                    cvv = _view(cv_p, (N,), torch.float32, device, me)
                    if cons is None:
                        cvv.zero_()
                    else:
                        cvv.copy_(torch.as_tensor(cons).to(torch.float32).reshape(N))
                return 0
            except Exception as exc:  # reported through moea_status
                me._callback_error = exc
                return 1
        return evaluate

    def _make_mating(self, mating):
        device = self._device
        me = self

        def select(user, vars_p, objs_p, cv_p, rank_p, active, out_p, N, D, M, gen, stream):
            try:
                with torch.cuda.device(device), torch.cuda.stream(torch.cuda.ExternalStream(stream, device=device)):
                    parents = {"variables": _view(vars_p, (N, D), torch.float32, device, me),
                               "objectives": _view(objs_p, (M, N), torch.float32, device, me).t(),
                               "constraints": _view(cv_p, (N,), torch.float32, device, me)}
                    state = {"active_count": active}
                    if rank_p:
                        state["rank"] = _view(rank_p, (N,), torch.int32, device, me)
                    out = mating.select(parents, state, {"generation": gen,
                                                         "max_generations": me._max_generations,
                                                         "device": device})
                    out = torch.as_tensor(out).to(torch.int32).reshape(-1)
                    if out.numel() != N:
                        raise ValueError("mating must return population_size indices")
                    _view(out_p, (N,), torch.int32, device, me).copy_(out)
                return 0
            except Exception as exc:
                me._callback_error = exc
                return 1
        return select

    # ------------------------------------------------------------------ native calls
    def _call(self, fn, *args):
        self._callback_error = None
        st = fn(*args)
        if st != 0:
            if self._callback_error is not None:
                raise self._callback_error
            check(st)

    def _ensure_native(self):
        if self._deferred_error is not None:
            raise self._deferred_error
        if self._native is None:
            cfg, keep = self._build_config()
            self._native = _Native(cfg, keep)
        return self._native.handle

    def initialize(self) -> None:
        if self._compose:
            self._composed_run().initialize()
            return
        h = self._ensure_native()
        self._call(lib().moea_algorithm_initialize, h)

    def step(self) -> None:
        if self._compose:
            self._composed_run().step()
        else:
            h = self._ensure_native()
            self._call(lib().moea_algorithm_step, h)
        if self._print_progress:
            g = self.generation
            if g == self._max_generations or (self._progress_interval > 0 and g % self._progress_interval == 0):
                print(f"Generation {g} / {self._max_generations} completed")

    def run(self, *, copy: bool = True) -> Result:
        if self._compose:
            self._result_total_ms = self._composed_run().run()
        else:
            h = self._ensure_native()
            total = ctypes.c_double(0.0)
            self._call(lib().moea_algorithm_run, h, ctypes.byref(total))
            self._result_total_ms = float(total.value)
        if self._print_progress:
            print(f"Generation {self.generation} / {self._max_generations} completed")
        return self.result(copy=copy)

    def result(self, *, copy: bool = True) -> Result:
        if self._compose:
            c = self._composed_run()
            aux, active = c.finalize()
            x, f, cv = c.P.x, c.P.f.t(), c.P.cv
            if copy:
                x, f, cv = x.clone(), f.contiguous(), cv.clone()
            return Result(x, f, cv, aux, int(active), float(c.total_ms))
        if self._native is None or not self.initialized:
            raise RuntimeError("Algorithm has not been initialized")
        h = self._native.handle
        self._call(lib().moea_algorithm_finalize, h)
        self._call(lib().moea_algorithm_synchronize, h)
        v = self._view_struct()
        pop = self._population_tensors(v, copy)
        if v.auxiliary_count > 0:
            aux = _view(v.d_auxiliary, (v.auxiliary_count,), torch.int32, v.device, self)
            if copy:
                aux = aux.clone()
        else:
            aux = torch.empty(0, dtype=torch.int32, device=f"cuda:{v.device}")
        return Result(pop.variables, pop.objectives, pop.constraints, aux, int(v.active_count),
                      float(v.total_ms))

    def _native_only(self, what: str) -> None:
        if self._compose:
            raise NotImplementedError(f"{what} belongs to the algorithm object; this run composes Python "
                                      "strategies")

    def profile_step(self) -> list[tuple[str, float]]:
        """Runs one generation with direct launches; device ms per stage."""
        self._native_only("profile_step")
        h = self._ensure_native()
        names = ctypes.create_string_buffer(4096)
        ms = (ctypes.c_float * 64)()
        cnt = ctypes.c_int(0)
        self._call(lib().moea_algorithm_profile_step, h, names, 4096, ms, 64, ctypes.byref(cnt))
        labels = names.value.decode().split("\n")
        return [(labels[i], float(ms[i])) for i in range(cnt.value)]

    def selection_stats(self) -> dict:
        """NSGA-III: last front index and sizes of the latest selection."""
        self._native_only("selection_stats")
        mf = ctypes.c_int(-1)
        sz = (ctypes.c_int * 4)()
        self._call(lib().moea_algorithm_selection_stats, self._ensure_native(), ctypes.byref(mf), sz)
        return {"max_front": mf.value, "N_prior": sz[0], "N_last": sz[1], "N_rem": sz[2], "N_nds": sz[3]}

    @property
    def graph_info(self) -> tuple[bool, int]:
        """(generations replay a CUDA graph, kernel nodes per generation)."""
        if self._compose:
            return False, 0
        v = self._view_struct()
        return bool(v.graph_active), int(v.kernels_per_generation)

    def reset(self) -> None:
        if self._compose:
            if self._composed is not None:
                self._composed.reset()
            return
        if self._native is None or not self.initialized:
            return
        self._call(lib().moea_algorithm_reset, self._native.handle)

    def load_snapshot(self, directory: str | Path) -> None:
        """Resumes from a generation directory written by ``save_data``
        snapshots (``<save_data>/generation_NNNNNN``): the population and the
        selection state are replaced, and the following steps equal those of
        the run that wrote it when the configuration is the same."""
        self._native_only("load_snapshot")
        h = self._ensure_native()
        self._call(lib().moea_algorithm_load_snapshot, h, os.fsencode(os.fspath(directory)))

    def flush_snapshots(self) -> None:
        """Waits until every snapshot queued so far is on disk."""
        if self._native is not None:
            self._call(lib().moea_algorithm_flush_snapshots, self._native.handle)

    def synchronize(self) -> None:
        if self._compose:
            if self._composed is not None and self._composed.stream is not None:
                self._composed.stream.synchronize()
            return
        if self._native is not None:
            self._call(lib().moea_algorithm_synchronize, self._native.handle)

    def _view_struct(self) -> PopulationViewC:
        v = PopulationViewC()
        self._call(lib().moea_algorithm_view, self._native.handle, ctypes.byref(v))
        return v

    def _population_tensors(self, v: PopulationViewC, copy: bool) -> Population:
        variables = _view(v.d_variables, (v.size, v.dimension), torch.float32, v.device, self)
        objectives = _view(v.d_objectives, (v.objectives, v.size), torch.float32, v.device, self).t()
        constraints = _view(v.d_constraints, (v.size,), torch.float32, v.device, self)
        if copy:
            variables, objectives, constraints = variables.clone(), objectives.contiguous(), constraints.clone()
        return Population(variables, objectives, constraints)

    @property
    def population(self) -> Population:
        if self._compose:
            c = self._composed
            if c is None or not c.initialized:
                raise RuntimeError("Algorithm has not been initialized")
            c.stream.synchronize()
            return Population(c.P.x, c.P.f.t(), c.P.cv)
        if self._native is None or not self.initialized:
            raise RuntimeError("Algorithm has not been initialized")
        self.synchronize()
        return self._population_tensors(self._view_struct(), False)

    def population_view(self) -> Population:
        """Zero-copy views of the current parents without synchronising; valid
        for work ordered on the algorithm's stream until the next step."""
        if self._compose:
            c = self._composed_run()
            return Population(c.P.x, c.P.f.t(), c.P.cv)
        return self._population_tensors(self._view_struct(), False)

    @property
    def reference_directions(self) -> torch.Tensor:
        """Directions in use, objective-major (M, count) view."""
        if self._compose:
            return self._composed_run().reference_directions
        ptr, count = ctypes.c_void_p(), ctypes.c_int()
        self._call(lib().moea_algorithm_directions, self._native.handle, ctypes.byref(ptr),
                   ctypes.byref(count))
        return _view(ptr.value, (self._problem_info[1], count.value), torch.float32, self._device, self)

    @property
    def initialized(self) -> bool:
        if self._compose:
            return self._composed is not None and self._composed.initialized
        if self._native is None:
            return False
        return bool(self._view_struct().initialized)

    @property
    def finished(self) -> bool:
        if self._compose:
            return self._composed is not None and self._composed.generation >= self._max_generations
        if self._native is None:
            return False
        return bool(self._view_struct().finished)

    @property
    def generation(self) -> int:
        if self._compose:
            return 0 if self._composed is None else self._composed.generation
        if self._native is None:
            return 0
        return int(self._view_struct().generation)


class NSGA3(Algorithm):
    def __init__(self, **kwargs: Any) -> None:
        super().__init__("NSGA3", **kwargs)


class RVEA(Algorithm):
    def __init__(self, **kwargs: Any) -> None:
        super().__init__("RVEA", **kwargs)


class AlgorithmBuilder:
    def __init__(self, algorithm: str) -> None:
        self.algorithm = algorithm
        self.options: dict[str, Any] = {}

    def set(self, **options: Any) -> "AlgorithmBuilder":
        self.options.update(options)
        return self

    def population_size(self, value: int) -> "AlgorithmBuilder":
        return self.set(population_size=value)

    def max_generations(self, value: int) -> "AlgorithmBuilder":
        return self.set(max_generations=value)

    def problem(self, value: Any) -> "AlgorithmBuilder":
        return self.set(problem=value)

    def mating(self, value: Any) -> "AlgorithmBuilder":
        return self.set(mating=value)

    def crossover(self, value: Any) -> "AlgorithmBuilder":
        return self.set(crossover=value)

    def mutation(self, value: Any) -> "AlgorithmBuilder":
        return self.set(mutation=value)

    def reference_directions(self, value: Any) -> "AlgorithmBuilder":
        return self.set(reference_directions=value)

    def environment_selector(self, value: Any) -> "AlgorithmBuilder":
        return self.set(environment_selector=value)

    def build(self) -> Algorithm:
        return Algorithm(self.algorithm, **self.options)
