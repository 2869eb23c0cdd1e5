"""Batched instances: many independent NSGA-III / RVEA algorithms advance
together, one CUDA graph launch per generation (moea_batch_* in
include/moea_b200.h).  Every instance computes exactly what it computes when
run alone; the batch only changes how the work is launched.

The reference runs one algorithm at a time; this is the batching form of the
B200 build, for many small instances of uneven size.
"""
from __future__ import annotations

import ctypes
from typing import Sequence

import torch

from ._lib import AlgorithmConfig, PopulationViewC, check, lib
from .algorithm import Algorithm, Population, Result, _view


class Batch:
    """Advance ``algorithms`` (not yet initialised, built-in problems and
    mating, same device and max_generations) as one batch."""

    def __init__(self, algorithms: Sequence[Algorithm], *, fuse: bool = True, groups: int = 0,
                 autotune: bool = False, half_tiles: bool = False):
        """``groups`` fixes the number of graph branches of the fused
        generation; ``autotune`` lets the library choose the schedule and the
        dominance tile shape per objective count by timing candidates on a
        scratch copy of the batch (MOEA_BATCH_AUTOTUNE; cached per instance
        mix); ``half_tiles`` uses half-width dominance tiles throughout
        (MOEA_BATCH_HALF_TILES).  Results never depend on any of them."""
        if not algorithms:
            raise ValueError("Batch needs at least one algorithm")
        n = len(algorithms)
        cfgs = (AlgorithmConfig * n)()
        keep: list = []
        for i, a in enumerate(algorithms):
            if a._deferred_error is not None:
                raise a._deferred_error
            if a._native is not None:
                raise ValueError("batched algorithms must not be initialised on their own")
            cfg, k = a._build_config()
            cfgs[i] = cfg
            keep.extend(k)
        self._keep = keep
        self._device = algorithms[0]._device
        with torch.cuda.device(self._device):
            self.stream = torch.cuda.Stream(self._device)
        handle = ctypes.c_void_p()
        # MOEA_BATCH_NO_FUSION = 1, MOEA_BATCH_AUTOTUNE = 2, MOEA_BATCH_HALF_TILES = 4;
        # MOEA_BATCH_GROUPS(g) = g << 8 (0: library default)
        flags = ((0 if fuse else 1) | ((int(groups) & 0xFF) << 8) | (2 if autotune else 0)
                 | (4 if half_tiles else 0))
        check(lib().moea_batch_create(cfgs, n, ctypes.c_void_p(self.stream.cuda_stream), flags,
                                      ctypes.byref(handle)))
        self._handle = handle
        self._count = n
        self._total_ms = 0.0

    def __len__(self) -> int:
        return self._count

    def __del__(self):
        self.close()

    def close(self) -> None:
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            try:
                lib().moea_batch_destroy(h)
            except Exception:
                pass
            self._handle = ctypes.c_void_p()

    def step(self) -> None:
        check(lib().moea_batch_step(self._handle))

    def run(self, generations: int | None = None) -> float:
        """Runs `generations` more generations (all remaining when None);
        returns the device milliseconds they took."""
        ms = ctypes.c_double(0.0)
        check(lib().moea_batch_run(self._handle, -1 if generations is None else int(generations),
                                   ctypes.byref(ms)))
        self._total_ms += float(ms.value)
        return float(ms.value)

    def synchronize(self) -> None:
        check(lib().moea_batch_synchronize(self._handle))

    def _info(self) -> tuple[int, int, int, int]:
        c, g, k, f = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(lib().moea_batch_info(self._handle, ctypes.byref(c), ctypes.byref(g), ctypes.byref(k),
                                    ctypes.byref(f)))
        return c.value, g.value, k.value, f.value

    @property
    def fused(self) -> bool:
        """True when every stage runs as one launch for all instances."""
        return bool(self._info()[3])

    @property
    def generation(self) -> int:
        return self._info()[1]

    @property
    def graph_kernels(self) -> int:
        """Kernel nodes in one generation's graph (all instances)."""
        return self._info()[2]

    @property
    def schedule(self) -> dict:
        """Groups of the fused generation and how they were chosen
        ("default", "autotuned", "autotuned (cached)"), with the autotuner's
        measured generation times of the chosen and the default schedule."""
        g, src = ctypes.c_int(), ctypes.c_int()
        t, d, slow, ser = ctypes.c_float(), ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
        group_of = (ctypes.c_int * self._count)()
        check(lib().moea_batch_schedule(self._handle, ctypes.byref(g), ctypes.byref(src), ctypes.byref(t),
                                        ctypes.byref(d), ctypes.byref(slow), ctypes.byref(ser), group_of))
        shapes = (ctypes.c_int * 17)()
        check(lib().moea_batch_tile_shapes(self._handle, shapes, 17))
        return {"groups": g.value, "source": ("default", "autotuned", "autotuned (cached)")[src.value],
                "tuned_ms": t.value, "default_ms": d.value, "slowest_instance_ms": slow.value,
                "instances_serial_ms": ser.value, "group_of": list(group_of),
                "half_tiles": [m for m in range(17) if shapes[m]]}

    def _view_struct(self, index: int) -> PopulationViewC:
        v = PopulationViewC()
        check(lib().moea_batch_view(self._handle, int(index), ctypes.byref(v)))
        return v

    def population(self, index: int, *, copy: bool = True) -> Population:
        self.synchronize()
        v = self._view_struct(index)
        variables = _view(v.d_variables, (v.size, v.dimension), torch.float32, v.device, self)
        objectives = _view(v.d_objectives, (v.objectives, v.size), torch.float32, v.device, self).t()
        constraints = _view(v.d_constraints, (v.size,), torch.float32, v.device, self)
        if copy:
            variables, objectives, constraints = variables.clone(), objectives.contiguous(), constraints.clone()
        return Population(variables, objectives, constraints)

    def result(self, index: int, *, copy: bool = True) -> Result:
        """Population of instance `index` with its front indices (NSGA-III)."""
        pop = self.population(index, copy=copy)
        v = self._view_struct(index)
        if v.auxiliary_count > 0:
            aux = _view(v.d_auxiliary, (v.auxiliary_count,), torch.int32, v.device, self)
            if copy:
                aux = aux.clone()
        else:
            aux = torch.empty(0, dtype=torch.int32, device=f"cuda:{v.device}")
        return Result(pop.variables, pop.objectives, pop.constraints, aux, int(v.active_count),
                      self._total_ms)
