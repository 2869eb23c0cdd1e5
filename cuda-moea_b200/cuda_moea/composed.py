"""Generations composed from strategy objects.

The reference runs every algorithm as EvolutionaryAlgorithm::step over six
strategy interfaces (nat/src/algorithm/algorithm.cu:104-286): mating,
crossover, mutation, evaluation, environmental selection and the direction
update, each a built-in C++ class or a Python object behind an adapter
(python/csrc/adapters.cpp:147-462).  The algorithm object of libmoea_b200
fuses the built-in strategies into one captured generation; this module is the
other form, used when any strategy is a Python object (PythonCrossover,
PythonMutation, PythonEnvironmentSelector, a PythonReferenceDirections with
update): the same step, with every built-in strategy a handle of the C ABI
(moea_create_*) and every Python strategy called on the algorithm's stream
with zero-copy tensor views, as the reference's adapters do.

With only built-in strategies it reproduces the algorithm object's runs bit
for bit (the handles share its draws and kernels), which the tests check.
"""
from __future__ import annotations

import ctypes
from typing import Any

import torch

from . import _lib
from ._lib import GenerationDesc, NSGA3SelectorConfig, PopulationDesc, check, lib
from .problem import PROBLEM_KINDS

PYTHON_STRATEGIES = ("PythonCrossover", "PythonMutation", "PythonEnvironmentSelector")


def needs_composition(specs: dict) -> bool:
    """Whether the strategies need the composed step (the algorithm object
    has callbacks for problems, mating and fixed Python directions only)."""
    for key in ("crossover", "mutation", "environment_selector"):
        if specs[key]["type"] in PYTHON_STRATEGIES:
            return True
    r = specs["reference_directions"]
    return r["type"] == "PythonReferenceDirections" and hasattr(r["object"], "update")


class _Handle:
    def __init__(self, ptr: ctypes.c_void_p, destroy):
        self.ptr = ptr
        self._destroy = destroy

    def __del__(self):
        if getattr(self, "ptr", None) is not None and self.ptr.value:
            try:
                self._destroy(self.ptr)
            except Exception:
                pass
            self.ptr = ctypes.c_void_p()


def _create(fn, destroy, *args) -> _Handle:
    h = ctypes.c_void_p()
    check(fn(*args, ctypes.byref(h)))
    return _Handle(h, destroy)


class _Slot:
    """One population: variables (N, D), objectives (M, N), violations (N)."""

    def __init__(self, N: int, D: int, M: int, bounds: torch.Tensor):
        dev = bounds.device
        self.x = torch.zeros((N, D), dtype=torch.float32, device=dev)
        self.f = torch.zeros((M, N), dtype=torch.float32, device=dev)
        self.cv = torch.zeros(N, dtype=torch.float32, device=dev)
        self.bounds = bounds
        self.desc = PopulationDesc(self.x.data_ptr(), self.f.data_ptr(), self.cv.data_ptr(), bounds.data_ptr(),
                                   N, D, M)

    def as_dict(self) -> dict:
        """The reference adapters' population dict (adapters.cpp:83-90)."""
        return {"variables": self.x, "objectives": self.f.t(), "constraints": self.cv,
                "bounds": self.bounds.view(-1, 2)}


class ComposedRun:
    """The generation loop of one algorithm over strategy objects."""

    def __init__(self, algo: Any):
        self.algo = algo
        self.specs = algo._specs
        self.N = algo._population_size
        self.T = algo._max_generations
        self.D, self.M = algo._problem_info
        self.device = algo._device
        self.seed = int(algo._cuda.seed)
        self.name = "NSGA3" if self.specs["environment_selector"]["type"] != "RVEAEnvironmentSelector" else "RVEA"
        self.initialized = False
        self.generation = 0
        self.epoch = 0
        self.total_ms = 0.0
        self.stream = None
        self._result_indices = None
        self._rank = None
        self._active = self.N
        self._state: dict = {}

    # ------------------------------------------------------------------ helpers
    @property
    def _s(self) -> int:
        return self.stream.cuda_stream

    def _ctx(self) -> GenerationDesc:
        return GenerationDesc(self.generation, self.T, self.seed)

    def _ctx_dict(self) -> dict:
        return {"generation": self.generation, "max_generations": self.T, "device": self.device}

    def _tensor(self, value, name: str, dtype) -> torch.Tensor:
        """checked_tensor of the reference's adapters (adapters.cpp:98-111)."""
        if not isinstance(value, torch.Tensor):
            raise ValueError(f"{name} must be a torch.Tensor")
        if not value.is_cuda or value.get_device() != self.device:
            raise ValueError(f"{name} must be on the algorithm CUDA device")
        return value.to(dtype).contiguous()

    def _copy_evaluation(self, output, slot: _Slot) -> None:
        """Objectives (N, M) and optional violations from a Python result
        (adapters.cpp:113-143)."""
        objectives, constraints = output, None
        if isinstance(output, dict):
            objectives, constraints = output["objectives"], output.get("constraints")
        elif isinstance(output, tuple):
            objectives = output[0]
            constraints = output[1] if len(output) > 1 else None
        src = self._tensor(objectives, "objectives", torch.float32)
        if src.dim() != 2 or tuple(src.shape) != (self.N, self.M):
            raise ValueError("objectives must have shape (population_size, objective_count)")
        slot.f.copy_(src.t())
        if constraints is None:
            slot.cv.zero_()
        else:
            cv = self._tensor(constraints, "constraints", torch.float32)
            if cv.numel() != self.N:
                raise ValueError("constraints must contain population_size values")
            slot.cv.copy_(cv.reshape(self.N))

    # ------------------------------------------------------------------ set-up
    def initialize(self) -> None:
        if self.initialized:
            return
        a = self.algo
        torch.cuda.set_device(self.device)
        cur = torch.cuda.current_stream(self.device)
        self.stream = cur if cur.cuda_stream != 0 else torch.cuda.Stream(self.device)
        a.stream = self.stream
        with torch.cuda.stream(self.stream):
            self._setup()
            self._start()
        self.initialized = True

    def _bounds(self) -> torch.Tensor:
        p = self.specs["problem"]
        D = self.D
        lo, hi = [0.0] * D, [1.0] * D
        if p["type"] in ("PythonProblem", "NativeProblem"):
            lo, hi = list(p["lower_bounds"]), list(p["upper_bounds"])
        elif p["type"] == "DTLZProblem" and p["kind"] == "CSDP":
            lo = [0.5, 0.45, 0.5, 0.5, 0.875, 0.4, 0.4]
            hi = [1.5, 1.35, 1.5, 1.5, 2.625, 1.2, 1.2]
        b = torch.tensor([v for pair in zip(lo, hi) for v in pair], dtype=torch.float32)
        return b.to(f"cuda:{self.device}")

    def _setup(self) -> None:
        L, N, D, M = lib(), self.N, self.D, self.M
        specs = self.specs
        self.bounds = self._bounds()
        self.P, self.O, self.X = (_Slot(N, D, M, self.bounds) for _ in range(3))
        self.pidx = torch.zeros(N, dtype=torch.int32, device=self.bounds.device)
        # problem
        p = specs["problem"]
        self.problem_kind = PROBLEM_KINDS[p["kind"]] if p["type"] == "DTLZProblem" else 0
        self.problem = p.get("object")
        self.activation = float(p["constraint_activation_ratio"]) if p["type"] == "DTLZProblem" else 0.0
        self._last_prepared = -2
        self.plugin = None
        if p["type"] == "NativeProblem":
            self.plugin = self.algo._plugin
        if self.problem is not None and hasattr(self.problem, "initialize"):
            self.problem.initialize({"device": self.device})
        # reference directions
        r = specs["reference_directions"]
        self.py_dirs = r["object"] if r["type"] == "PythonReferenceDirections" else None
        if r["type"] == "DasDennisDirections":
            self.dirs = _create(L.moea_create_dasdennis, L.moea_directions_destroy, int(r["partitions"]))
        elif r["type"] == "AdaptiveRVEADirections":
            self.dirs = _create(L.moea_create_adaptive_directions, L.moea_directions_destroy, float(r["frequency"]))
        else:
            if r["type"] == "UserDefinedDirections":
                values = torch.as_tensor(r["values"]).detach().to("cpu", torch.float32)
                normalize = bool(r["normalize"])
            else:
                values = self._tensor(self.py_dirs.initialize(N, M, {"device": self.device}),
                                      "reference directions", torch.float32).cpu()
                normalize = False  # the Python provider's values are used as given (adapters.cpp:371-380)
            if values.dim() != 2 or values.shape[1] != M:
                raise ValueError("reference directions must have shape (count, objective_count)")
            self._user_dirs = values.t().contiguous()
            self.dirs = _create(L.moea_create_user_directions, L.moea_directions_destroy,
                                ctypes.cast(self._user_dirs.data_ptr(), _lib.fp), M, int(values.shape[0]),
                                1 if normalize else 0)
        check(L.moea_directions_initialize(self.dirs.ptr, N, M, self.device, self._s))
        # reproduction
        m = specs["mating"]
        self.py_mating = m["object"] if m["type"] == "PythonMating" else None
        if m["type"] == "TournamentMating":
            self.mating = _create(L.moea_create_tournament, L.moea_mating_destroy)
        elif m["type"] == "RandomMating":
            self.mating = _create(L.moea_create_random_mating, L.moea_mating_destroy)
        c = specs["crossover"]
        self.py_crossover = c["object"] if c["type"] == "PythonCrossover" else None
        if c["type"] == "SBX":
            self.crossover = _create(L.moea_create_sbx, L.moea_crossover_destroy, float(c["eta_initial"]),
                                     float(c["eta_final"]), float(c["probability"]),
                                     float(c["variable_copy_probability"]))
        mu = specs["mutation"]
        self.py_mutation = mu["object"] if mu["type"] == "PythonMutation" else None
        self.mutation = None
        if mu["type"] == "PolynomialMutation":
            self.mutation = _create(L.moea_create_pm, L.moea_mutation_destroy, float(mu["eta_initial"]),
                                    float(mu["eta_final"]), float(mu["probability"]))
        info = {"name": self.name, "population_size": N, "dimension": D, "objective_count": M,
                "max_generations": self.T, "device": self.device}
        for obj in (self.py_mating, self.py_crossover, self.py_mutation):
            if obj is not None and hasattr(obj, "initialize"):
                obj.initialize(dict(info))
        # environmental selection
        sel = specs["environment_selector"]
        self.py_selector = sel["object"] if sel["type"] == "PythonEnvironmentSelector" else None
        if self.py_selector is None:
            if sel["type"] == "NSGA3EnvironmentSelector":
                mode = int(sel.get("association_mode", 0))
                if self.py_dirs is not None:
                    mode = 1  # directions a Python provider may change on the device are scanned
                cfg = NSGA3SelectorConfig(float(sel["sparse_ratio"]), int(sel["cv_bins"]),
                                          float(sel["cv_clip_upper"]), float(sel["cv_log_alpha"]),
                                          float(sel["feasibility_epsilon"]), mode)
                self.selector = _create(L.moea_create_nsga3_selector, L.moea_selector_destroy, ctypes.byref(cfg))
            else:
                self.selector = _create(L.moea_create_rvea_selector, L.moea_selector_destroy, float(sel["alpha"]))
            check(L.moea_selector_initialize(self.selector.ptr, N, D, M, self.T, self.dirs.ptr, self.device,
                                             self._s))
        else:
            refs = self.reference_directions.t() if self.dirs is not None else None
            self.py_selector.initialize({k: v for k, v in info.items() if k != "device"}, refs,
                                        {"device": self.device})

    def _cv_active(self, it: int) -> bool:
        """MOEAStdTestEvaluator::is_cv_active (dtlz_kernels.cu:1302-1312)."""
        if self.activation <= 0.0:
            return True
        if it < 0 or self.T <= 0:
            return False
        return (it + 1) / self.T >= self.activation

    def _cv_switch(self, target: int) -> bool:
        """The generation whose parents are re-evaluated with their violations
        (dtlz_kernels.cu:1361-1394)."""
        if target < 0 or self._last_prepared == target:
            return False
        if target == 0:
            return self._cv_active(0)
        return not self._cv_active(target - 1) and self._cv_active(target)

    def _evaluate(self, slot: _Slot, generation: int) -> None:
        L, N, D, M = lib(), self.N, self.D, self.M
        if self.problem_kind:
            check(L.moea_problem_evaluate(self.problem_kind, slot.x.data_ptr(), N, D, M, slot.f.data_ptr(),
                                          slot.cv.data_ptr(), self._s))
            if 9 <= self.problem_kind <= 14 and not self._cv_active(generation):
                slot.cv.zero_()
        elif self.problem is not None:
            out = self.problem.evaluate(slot.x, {"generation": generation, "max_generations": self.T,
                                                 "device": self.device})
            self._copy_evaluation(out, slot)
        else:
            rc = L.moea_native_evaluate(self.plugin.ptr, slot.x.data_ptr(), slot.f.data_ptr(), slot.cv.data_ptr(),
                                        N, D, M, generation, self.T, self._s)
            check(rc)

    def _start(self) -> None:
        L, N, D = lib(), self.N, self.D
        init = self.algo._initial
        if init is not None and self.epoch == 0:
            if tuple(init.shape) != (N, D):
                raise ValueError("initial_population must have shape (population_size, dimension)")
            lo, hi = self.bounds[0::2].cpu(), self.bounds[1::2].cpu()
            if not torch.isfinite(init).all() or (init < lo).any() or (init > hi).any():
                raise ValueError("initial_population contains a non-finite or out-of-bounds value")
            self.P.x.copy_(init.to(self.P.x.device))
        else:
            check(L.moea_initialize_population(self.seed, self.epoch, self.bounds.data_ptr(), N, D,
                                               self.P.x.data_ptr(), self._s))
        self._evaluate(self.P, -1)
        self.generation = 0
        self._active = N
        self._last_prepared = -2
        self._prepare()

    # ------------------------------------------------------------------ selector state
    def _prepare(self) -> None:
        if self.py_selector is None:
            check(lib().moea_selector_prepare(self.selector.ptr, ctypes.byref(self.P.desc), ctypes.byref(self._ctx()),
                                              self._s))
        else:
            self._update_state(self.py_selector.prepare(self.P.as_dict(), self._ctx_dict()))

    def _update_state(self, output) -> None:
        """The Python selector's state (adapters.cpp:450-458)."""
        if not isinstance(output, dict):
            return
        if "rank" in output:
            self._state["rank"] = self._tensor(output["rank"], "rank", torch.int32)
        if "reference_index" in output:
            self._state["reference_index"] = self._tensor(output["reference_index"], "reference_index", torch.int32)
        if "score" in output:
            self._state["score"] = self._tensor(output["score"], "score", torch.float32)
        if "result_indices" in output:
            self._state["result_indices"] = self._tensor(output["result_indices"], "result_indices", torch.int32)
        if "active_count" in output:
            self._active = int(output["active_count"])

    def _mating_state(self):
        """(rank tensor or None, device active pointer or None, host active)."""
        if self.py_selector is None:
            rank, active = ctypes.c_void_p(), ctypes.c_void_p()
            check(lib().moea_selector_mating_state(self.selector.ptr, ctypes.byref(rank), ctypes.byref(active)))
            return rank.value, active.value, None
        rank = self._state.get("rank")
        return (rank.data_ptr() if rank is not None else None), None, self._active

    # ------------------------------------------------------------------ the step
    def step(self) -> None:
        if not self.initialized:
            self.initialize()
        if self.generation >= self.T:
            return
        with torch.cuda.stream(self.stream):
            self._step()

    def _step(self) -> None:
        L, N = lib(), self.N
        ctx = self._ctx()
        # problem.prepare_parent -> selector.prepare (algorithm.cu:227-235)
        if self.problem_kind and 9 <= self.problem_kind <= 15 and self._cv_switch(self.generation):
            check(L.moea_problem_evaluate(self.problem_kind, self.P.x.data_ptr(), N, self.D, self.M,
                                          self.P.f.data_ptr(), self.P.cv.data_ptr(), self._s))
            self._last_prepared = self.generation
            self._prepare()
        elif self.plugin is not None:
            changed = ctypes.c_int(0)
            check(L.moea_native_prepare(self.plugin.ptr, self.P.x.data_ptr(), self.P.f.data_ptr(),
                                        self.P.cv.data_ptr(), N, self.D, self.M, self.generation, self.T, self._s,
                                        ctypes.byref(changed)))
            if changed.value:
                self._prepare()
        elif self.problem is not None and hasattr(self.problem, "prepare_parent"):
            out = self.problem.prepare_parent(self.P.as_dict(), {"generation": self.generation,
                                                                  "max_generations": self.T, "device": self.device})
            changed = bool(out) if isinstance(out, bool) else out is not None
            if out is not None and not isinstance(out, bool):
                self._copy_evaluation(out, self.P)
            if changed:
                self._prepare()
        # reproduction (reproduction_pipeline.cu:40-58)
        rank_p, active_p, active_h = self._mating_state()
        if self.py_mating is not None:
            state = {"active_count": self._active if active_h is None else active_h}
            if self.py_selector is None:
                state["active_count"] = self._active_count_sync()
                if rank_p:
                    state["rank"] = torch.as_tensor(_lib_view_int(rank_p, N, self), device=self.P.x.device)
            else:
                state.update({k: v for k, v in self._state.items() if k in ("rank", "reference_index", "score")})
            out = self._tensor(self.py_mating.select(self.P.as_dict(), state, self._ctx_dict()), "parent_indices",
                               torch.int32)
            if out.numel() != N:
                raise ValueError("parent_indices has the wrong number of elements")
            self.pidx.copy_(out.reshape(N))
        else:
            if active_p is None and active_h is not None:
                self._active_buf = torch.tensor([active_h], dtype=torch.int32, device=self.P.x.device)
                active_p = self._active_buf.data_ptr()
            check(L.moea_mating_select(self.mating.ptr, ctypes.byref(self.P.desc), rank_p, active_p,
                                       self.pidx.data_ptr(), N, ctypes.byref(ctx), self._s))
        if self.py_crossover is not None:
            out = self._tensor(self.py_crossover.apply(self.P.as_dict(), self.pidx, self._ctx_dict()),
                               "offspring variables", torch.float32)
            if tuple(out.shape) != (N, self.D):
                raise ValueError("crossover output must have shape (population_size, dimension)")
            self.O.x.copy_(out)
        else:
            check(L.moea_crossover_apply(self.crossover.ptr, ctypes.byref(self.P.desc), self.pidx.data_ptr(),
                                         ctypes.byref(self.O.desc), ctypes.byref(ctx), self._s))
        if self.py_mutation is not None:
            out = self.py_mutation.mutate(self.O.as_dict(), self._ctx_dict())
            if out is not None:
                out = self._tensor(out, "mutated variables", torch.float32)
                if tuple(out.shape) != (N, self.D):
                    raise ValueError("mutation output must have shape (population_size, dimension)")
                self.O.x.copy_(out)
        elif self.mutation is not None:
            check(L.moea_mutation_apply(self.mutation.ptr, ctypes.byref(self.O.desc), ctypes.byref(ctx), self._s))
        self._evaluate(self.O, self.generation)
        # environmental selection
        if self.py_selector is None:
            check(L.moea_selector_select(self.selector.ptr, ctypes.byref(self.P.desc), ctypes.byref(self.O.desc),
                                         ctypes.byref(self.X.desc), ctypes.byref(ctx), self._s))
        else:
            self._python_select()
        # direction update on the next population (algorithm.cu:262-268)
        if self.py_dirs is not None and hasattr(self.py_dirs, "update"):
            out = self.py_dirs.update(self.X.as_dict(), self.reference_directions.t(), self._active_count_sync(),
                                      self._ctx_dict())
            if out is not None:
                v = self._tensor(out, "reference directions", torch.float32)
                cur = self.reference_directions
                if v.dim() != 2 or tuple(v.shape) != (cur.shape[1], self.M):
                    raise ValueError("updated reference directions cannot change count")
                cur.copy_(v.t())
        else:
            active = None
            if self.py_selector is None:
                _, active, _ = self._mating_state()
            else:
                self._active_buf = torch.tensor([self._active], dtype=torch.int32, device=self.P.x.device)
                active = self._active_buf.data_ptr()
            check(L.moea_directions_update(self.dirs.ptr, ctypes.byref(self.X.desc), active, ctypes.byref(ctx),
                                           self._s))
        self.P, self.X = self.X, self.P
        self.generation += 1

    def _python_select(self) -> None:
        out = self.py_selector.select(self.P.as_dict(), self.O.as_dict(), self._ctx_dict())
        if not isinstance(out, dict):
            raise ValueError("environment select must return a dict")
        if "indices" in out:
            idx = self._tensor(out["indices"], "selected indices", torch.int64)
            if idx.numel() != self.N:
                raise ValueError("selected indices must contain population_size values")
            idx = idx.reshape(self.N)
            self.X.x.copy_(torch.cat([self.P.x, self.O.x]).index_select(0, idx))
            self.X.f.copy_(torch.cat([self.P.f, self.O.f], 1).index_select(1, idx))
            self.X.cv.copy_(torch.cat([self.P.cv, self.O.cv]).index_select(0, idx))
        else:
            v = self._tensor(out["variables"], "variables", torch.float32)
            if tuple(v.shape) != (self.N, self.D):
                raise ValueError("variables must have shape (population_size, dimension)")
            self.X.x.copy_(v)
            self._copy_evaluation(out, self.X)
        self._update_state(out)

    def _active_count_sync(self) -> int:
        if self.py_selector is not None:
            return self._active
        a = ctypes.c_int(0)
        check(lib().moea_selector_active_count(self.selector.ptr, ctypes.byref(a), self._s))
        return a.value

    # ------------------------------------------------------------------ results
    def run(self) -> float:
        if not self.initialized:
            self.initialize()
        with torch.cuda.stream(self.stream):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(self.stream)
            while self.generation < self.T:
                self._step()
            e1.record(self.stream)
            e1.synchronize()
        self.total_ms += e0.elapsed_time(e1)
        return self.total_ms

    def finalize(self) -> tuple[torch.Tensor, int]:
        """(result indices, active count) after the selector's finalize."""
        if not self.initialized:
            raise RuntimeError("Algorithm has not been initialized")
        with torch.cuda.stream(self.stream):
            if self.py_selector is None:
                L = lib()
                check(L.moea_selector_finalize(self.selector.ptr, ctypes.byref(self.P.desc), self._s))
                ptr, count = ctypes.c_void_p(), ctypes.c_int(0)
                check(L.moea_selector_result_indices(self.selector.ptr, ctypes.byref(ptr), ctypes.byref(count)))
                idx = _lib_view_int(ptr.value, count.value, self) if count.value > 0 else None
                aux = (torch.as_tensor(idx, device=self.P.x.device).clone() if idx is not None
                       else torch.empty(0, dtype=torch.int32, device=self.P.x.device))
                active = self._active_count_sync()
            else:
                if hasattr(self.py_selector, "finalize"):
                    self._update_state(self.py_selector.finalize(self.P.as_dict(), self._ctx_dict()))
                aux = self._state.get("result_indices")
                if aux is None:
                    aux = torch.empty(0, dtype=torch.int32, device=self.P.x.device)
                active = self._active
        self.stream.synchronize()
        return aux, active

    @property
    def reference_directions(self) -> torch.Tensor:
        ptr, count, M = ctypes.c_void_p(), ctypes.c_int(0), ctypes.c_int(0)
        check(lib().moea_directions_view(self.dirs.ptr, ctypes.byref(ptr), None, None, ctypes.byref(M),
                                         ctypes.byref(count)))
        from .algorithm import _view
        return _view(ptr.value, (M.value, count.value), torch.float32, self.device, self)

    def reset(self) -> None:
        if not self.initialized:
            return
        L = lib()
        self.stream.synchronize()
        self.epoch += 1
        with torch.cuda.stream(self.stream):
            check(L.moea_directions_reset(self.dirs.ptr, self._s))
            if self.py_dirs is not None and hasattr(self.py_dirs, "reset"):
                self.py_dirs.reset()
            if self.py_selector is None:
                check(L.moea_selector_reset(self.selector.ptr, self._s))
            else:
                self._state = {}
                self._active = self.N
                if hasattr(self.py_selector, "reset"):
                    self.py_selector.reset()
            if self.problem is not None and hasattr(self.problem, "reset"):
                self.problem.reset()
            elif self.plugin is not None:
                L.moea_native_reset(self.plugin.ptr)
            self.total_ms = 0.0
            self._start()


def _lib_view_int(ptr: int, n: int, owner: "ComposedRun"):
    from .algorithm import _view
    return _view(ptr, (n,), torch.int32, owner.device, owner)
