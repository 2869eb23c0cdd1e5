#!/usr/bin/env python
"""Benchmark of the NSGA-III generation hot path on B200.

Workload (the configuration the headline metric is quoted on): NSGA-III on
DTLZ1, M=3 objectives, D=7 FP32 variables, population N=32768 (merged 65536),
Das-Dennis directions with H=254 partitions (32640 directions), SBX eta=30
pc=1, polynomial mutation eta=20 pm=1/D, tournament mating.  Synthetic data:
the initial population is drawn uniformly in [0,1]^D from the seed.

One step = one generation (mating, SBX+PM, DTLZ1 evaluation, environmental
selection).  Every step is timed with CUDA events on the algorithm's stream;
between timed steps the L2 cache is flushed by writing a 256 MiB buffer
(outside the timed intervals).  Multi-GPU: one independent replica per GPU
(a single instance does not shard), value = total generations/s,
max-over-ranks time; the batched record shards its instances over the ranks.

The default line also carries `rvea_large_d` (RVEA DTLZ2 M=8 D=131072 N=1024,
10 timed generations) and the batched record.

Other workloads (--workload): dtlz2-small (N=92), rvea-large-d (D=131072),
c1dtlz1-m10 and constrained-batch (ten objectives, 275 two-layer
directions, 64 seeds per batched launch), dtlz2-m8 (tensor-core
association), dtlz1-h255 (the headline configuration with 255 partitions,
32896 directions).

`--impl reference` times the CPU restatement of the reference path (oracle/)
on the host cores, same metric and workload (the reference itself has no CPU
implementation and no B200 build of its own GPU path runs here unmodified).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "cuda-moea_b200"))
sys.path.insert(0, str(ROOT))

METRIC = "NSGA-III gen/s @N=32768,M=3; batched instance-gen/s vs plain, identical ranks"
WORKLOAD = "NSGA-III DTLZ1 M=3 D=7 N=32768, Das-Dennis H=254 (32640 directions), 1 generation per step"
N_POP, D_VAR, M_OBJ, PARTITIONS = 32768, 7, 3, 254
# dram__bytes_read.sum + dram__bytes_write.sum of one nds_block_rows launch at
# this workload (one ncu --set full capture of the launch)
ROWS_DRAM_BYTES = 5.80e6 + 217.07e6
# dram__bytes_read.sum + dram__bytes_write.sum of one nds_peel_owned launch at
# this workload (one ncu --set full capture of the launch)
PEEL_DRAM_BYTES = 134.72e6 + 3.56e6
# l1tex__data_pipe_lsu_wavefronts of one nds_block_rows launch at this
# workload (shared-memory loads and stores 24.15e6, global row stores and
# table copies the rest): the work of the unit that bounds the kernel
ROWS_LSU_WAVEFRONTS = 29.17e6
# smsp__inst_executed.sum of the same launch: warp instructions, 32 lane-ops
# each, for its n(n-1)/2 pair tests
ROWS_WARP_INSTR = 86.95e6


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]
        return False

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in getattr(self, "lines", []):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def kernel_rooflines(stage_ms: dict, n_mix: int, headline: bool):
    """Roofline entries of the heavy kernels of one headline generation, the
    largest stage time first.

    - nds_peel (ndsort.peel): against the measured HBM copy bandwidth; its
      algorithmic bytes are the lower-triangle relation rows, each read at
      most once: n(n-1)/2 bits.
    - nds_block_rows (ndsort.dominance_tiles, with the block tables): bound
      by the LSU data pipe (shared-memory tree descents and prefix-set reads,
      row stores), so against that pipe's peak of one wavefront per SM and
      clock (148 SMs x max SM clock), with ROWS_LSU_WAVEFRONTS per launch;
      the pair tests/s, the HBM fraction on the rows written and the fraction
      of the SIMT lane-op peak (148 SMs x 128 lanes x max SM clock) at the
      kernel's counted lane-ops per pair go beside it.
    """
    hbm, peak_kind = _peaks()
    tri_pairs = n_mix * (n_mix - 1) / 2
    rel_bytes = tri_pairs / 8
    out = []
    peel = stage_ms.get("ndsort.peel")
    if peel:
        a = rel_bytes / (peel / 1e3) / 1e9
        out.append({"kernel": "nds_peel_owned (front peeling)", "bound": "hbm", "achieved": a, "peak": hbm,
                    "unit": "GB/s", "frac": a / hbm, "peak_source": peak_kind, "algorithmic_bytes": rel_bytes,
                    "traffic": PEEL_DRAM_BYTES if headline else None, "ms": peel})
    tiles = stage_ms.get("ndsort.dominance_tiles")
    if tiles and headline:
        lsu_peak = 148 * 1.965e9
        a = ROWS_LSU_WAVEFRONTS / (tiles / 1e3)
        out.append({"kernel": "nds_block_rows (dominance rows)", "bound": "lsu", "achieved": a, "peak": lsu_peak,
                    "unit": "LSU wavefronts/s", "frac": a / lsu_peak,
                    "peak_source": "148 SMs x 1 LSU data-pipe wavefront/clk x 1965 MHz",
                    "pair_tests_per_s": tri_pairs / (tiles / 1e3),
                    "lane_ops_per_pair": ROWS_WARP_INSTR * 32 / tri_pairs,
                    "simt_frac": tri_pairs / (tiles / 1e3) * (ROWS_WARP_INSTR * 32 / tri_pairs) / (148 * 128 * 1.965e9),
                    "algorithmic_bytes": rel_bytes, "hbm_frac": rel_bytes / (tiles / 1e3) / 1e9 / hbm,
                    "traffic": ROWS_DRAM_BYTES, "ms": tiles})
    out.sort(key=lambda r: -r["ms"])
    return out


def cpu_generation_time(n: int, threads: int, seed: int = 1):
    """One CPU generation of the restated reference path (oracle, OpenMP)."""
    import numpy as np
    from oracle import oracle as O
    O.build()
    os.environ["OMP_NUM_THREADS"] = str(threads)
    rng = np.random.default_rng(seed)
    x = rng.random((n, D_VAR)).astype(np.float32)
    f, cv = O.evaluate("DTLZ1", x, M_OBJ)
    refs = O.reference_directions(1, PARTITIONS, M_OBJ)
    bounds = np.tile([0.0, 1.0], D_VAR).astype(np.float32)
    fronts, _ = O.ndsort(cv, f, n)
    ideal = f.min(1).astype(np.float32)
    t0 = time.perf_counter()
    seed64 = O.derive_seed(2887)
    mate = O.philox_stream(seed64, 0, 2, n)
    cand = np.stack([mate[:, 0] % n, mate[:, 1] % n], 1).astype(np.int32)
    pidx = O.tournament(cand, fronts, cv)
    # the product's draw layout: one crossover block per four variables of a
    # pair (spread draw and sign per word; the crossover probability is 1 and
    # the copy probability 0, so no test or copy blocks), mutation at
    # geometric sites with limit pm_prob / D
    pairs, D4 = n // 2, (D_VAR + 3) // 4
    unit = lambda u: (u >> 8).astype(np.float32) * np.float32(1.0 / 16777216.0)
    cx = O.philox_stream(seed64, 0, 3, pairs * D4).reshape(pairs, D4 * 4)[:, :D_VAR].reshape(-1)
    off = O.sbx(x, pidx, bounds, np.stack([unit(cx), np.zeros_like(unit(cx))], 1), (cx & 1).astype(np.int32),
                np.zeros(pairs * D_VAR, np.float32), 30.0, 1.0, 0.0, n)
    limit = np.float32(1.0) / np.float32(D_VAR)
    log_keep = float(np.log1p(-np.float64(limit)))
    um = np.zeros((n * D_VAR, 2), np.float32)
    um[:, 0] = 2.0
    site, live, k = np.full(n, -1, np.int64), np.ones(n, bool), 0
    while live.any():
        w = O.philox_stream(seed64, 0, 4, (k + 1) * n)[k * n:]
        u = ((w[:, 0] >> 8) + 1).astype(np.float64) * (1.0 / 16777216.0)
        site = np.where(live, site + 1 + np.minimum(np.floor(np.log(u) / log_keep), D_VAR).astype(np.int64), site)
        live &= site < D_VAR
        c = np.nonzero(live)[0]
        um[c * D_VAR + site[c]] = np.stack([np.zeros(len(c), np.float32), unit(w[c, 1])], 1)
        k += 1
    off = O.pm(off, bounds, um, 20.0, 1.0)
    of, ocv = O.evaluate("DTLZ1", off, M_OBJ)
    O.nsga3_select(np.concatenate([cv, ocv]), np.concatenate([f, of], 1), refs, seed64, 0, ideal)
    return time.perf_counter() - t0


STAGE_SEED = 12345  # the fixed generation-0 population both arms time stages on


def stage_population(n: int):
    """The fixed merged population of the per-stage comparison: 2n points
    uniform in [0,1]^D_VAR from STAGE_SEED (parents first, then offspring)."""
    import numpy as np
    rng = np.random.default_rng(STAGE_SEED)
    return rng.random((2 * n, D_VAR)).astype(np.float32)


class _QuietStdout:
    """Sends file descriptor 1 to /dev/null for the duration (the reference's
    library prints progress lines on stdout; the bench prints one JSON line)."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(null, 1)
        os.close(null)
        return self

    def __exit__(self, *exc):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)
        return False


def reference_gpu_record(steps: int):
    with _QuietStdout():
        return _reference_gpu_record(steps)


def _reference_gpu_record(steps: int):
    """The reference's own GPU path on this GPU, as a second baseline: its
    complete NSGA-III generation (all of its native sources compiled in place
    into oracle/_ref/libmoea_ref_algo.so, built through its C++ builder, each
    step bracketed by device synchronises) on the headline and the small
    workload, looped over a sample of the batched workload's instances, and
    its stage functions (oracle/_ref/libmoea_ref.so) timed with
    CUDA events on the fixed generation-0 merged population of
    stage_population."""
    try:
        import torch
        if not torch.cuda.is_available():
            return {"unavailable": "no CUDA device visible to the reference arm"}
        from oracle.ref import ref as R
        if not (R.algo_available() and R.available()):
            return {"unavailable": "oracle/_ref not built (needs the reference sources at build time)"}
        import numpy as np
        rec = {"source": "CUDA-MOEA's own kernels and algorithm, compiled for sm_100a from its sources",
               "timing": "host clock around each device-synchronised step (the reference's step waits on "
                         "the host for its front sizes); stages: CUDA events over repeated calls",
               "sparse_ratio": 1.0, "algorithm": []}
        for desc, kind, D, M, N, parts, gens, warm, k in [
                (WORKLOAD, 1, D_VAR, M_OBJ, N_POP, PARTITIONS, 50, 5, steps),
                ("NSGA-III DTLZ2 M=3 D=12 N=92, 91 directions", 2, 12, 3, 92, 0, 100, 5, 50)]:
            ms = R.algo_time(0, kind, D, M, N, parts, gens, 1.0, 2887, warm, k)
            rec["algorithm"].append({"workload": desc, "steps": k, "warmup": warm,
                                     "gen_per_s": k / (sum(ms) / 1e3),
                                     "ms_per_gen_median": statistics.median(ms)})
        # the batched workload: the reference runs one algorithm at a time, so
        # its rate is the instances looped; every 8th instance, 5 steps each
        specs = batch_specs(256)[::8]
        tot_ms, steps_b = 0.0, 5
        for kind, M, N, D, seed in specs:
            tot_ms += sum(R.algo_time(0, kind, D, M, N, 0, 200, 1.0, seed, 3, steps_b))
        rec["batched_looped"] = {"workload": BATCH_WORKLOAD, "sample": f"{len(specs)} of the 256 instances "
                                 f"(every 8th), {steps_b} generations each after 3 warm-up",
                                 "instance_gen_per_s": len(specs) * steps_b / (tot_ms / 1e3)}
        # stages on the fixed population
        from oracle import oracle as O
        x = stage_population(N_POP)
        rep = 5
        stages = {}
        R.set_repeat(rep)
        objs, _ = R.problem(1, x[N_POP:], M_OBJ)
        stages["evaluate (DTLZ1, N offspring)"] = R.last_ms()
        R.set_repeat(0)
        objs, _ = R.problem(1, x, M_OBJ)
        cv = np.zeros(2 * N_POP, np.float32)
        R.set_repeat(rep)
        fronts, mf = R.ndsort(cv, objs, N_POP)
        stages["ndsort"] = R.last_ms()
        R.set_repeat(0)
        gidx, sizes = O.nds_extract(fronts, mf, N_POP)
        ideal = objs.min(1).astype(np.float32)
        f_nds = objs[:, gidx]
        fn, _ = R.normalize(f_nds, ideal)
        R.set_repeat(rep)
        R.normalize(f_nds, ideal)
        stages["normalize"] = R.last_ms()
        refs = O.reference_directions(1, PARTITIONS, M_OBJ)
        idx, dist = R.associate(fn, refs)
        stages["associate"] = R.last_ms()
        R.niching(O.derive_seed(2887), 0, gidx, dist, idx, sizes, refs.shape[1], N_POP)
        stages["niching"] = R.last_ms()
        R.set_repeat(0)
        rec["stages_ms_generation0"] = stages
        rec["stage_population"] = (f"2x{N_POP} points uniform in [0,1]^{D_VAR} (numpy seed {STAGE_SEED}), "
                                   f"DTLZ1 objectives; max_front {mf}, sizes {[int(v) for v in sizes]}")
        return rec
    except Exception as exc:  # the baseline is reported, never fatal
        return {"unavailable": f"{type(exc).__name__}: {exc}"}


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    budget = float(os.environ.get("MOEA_REFERENCE_BUDGET_S", "150"))
    times = [cpu_generation_time(N_POP, threads, seed=1)]
    while len(times) < args.steps and sum(times) + times[0] < budget:
        times.append(cpu_generation_time(N_POP, threads, seed=len(times) + 1))
    total = sum(times)
    value = len(times) / total
    sample = (f"{len(times)} full generation(s) of the workload on the CPU oracle "
              f"(OpenMP, {threads} threads); warm-up skipped; time-boxed to {budget:.0f} s")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "gen/s",
        "n_gpus": args.gpus, "steps": len(times), "warmup": 0,
        "ms_per_step": 1000.0 * total / len(times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "population": N_POP, "merged": 2 * N_POP, "directions": 32640,
                   "l2": "host CPU run: no device cache between generations",
                   "parallelism": "host threads (OpenMP)", "cuda_graph": False},
        "device": "host CPU",
        "cpu_baseline": {"value": value, "unit": "gen/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "gen/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_gpu": reference_gpu_record(max(5, min(args.steps, 20))),
    }))


def over_ranks(value: float, op: str, world: int, device) -> float:
    """value combined over the ranks of the process group: "max" for device
    times (the job's time is its slowest replica), "sum" for rates of
    independent replicas.  A single process returns value unchanged."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def replica_seed(seed: int, rank: int) -> int:
    """Seed of the replica on `rank` (independent replicas, one per GPU)."""
    return seed + rank


BATCH_WORKLOAD = ("batched NSGA-III: 256 independent instances, DTLZ1-7 uniform, M in {3,5,8}, "
                  "N uniform even in 92..4096, D=M+9 (M+19 for DTLZ7), seeds 0..255, 200-generation runs")


def batch_specs(count: int, seed: int = 0):
    """The batched workload: (kind, M, N, D, seed) per instance."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        kind = int(rng.integers(1, 8))
        M = int(rng.choice([3, 5, 8]))
        N = int(rng.integers(46, 2049)) * 2
        D = M + (19 if kind == 7 else 9)
        out.append((kind, M, N, D, i))
    return out


def shard_instances(specs, world: int, rank: int):
    """Indices of the instances `rank` runs: largest first, each to the rank
    with the least work so far, work = pair tests (2N)^2.  Every instance is
    on exactly one rank; with one rank, all of them in order."""
    loads = [0] * world
    own = []
    for i in sorted(range(len(specs)), key=lambda i: (-(2 * specs[i][2]) ** 2, i)):
        r = min(range(world), key=lambda j: (loads[j], j))
        loads[r] += (2 * specs[i][2]) ** 2
        if r == rank:
            own.append(i)
    return sorted(own)


def batched_measure(args, torch, cm, world: int = 1, rank: int = 0):
    """Instance-generations/s of the batch (one graph launch per generation,
    schedule chosen by the library's autotuner) against the same instances
    looped one after another through the plain path on one stream, both over
    the whole 200-generation run (every generation timed with CUDA events),
    with the rates of three windows (early, middle, late) beside it.  After
    the run every instance's front indices and objectives are compared.  With
    several ranks the instances are sharded (shard_instances) and the job's
    rate is all instances over the slowest rank's time."""
    all_specs = batch_specs(args.batch_instances)
    specs = [all_specs[i] for i in shard_instances(all_specs, world, rank)]
    T = args.batch_generations

    def make(spec):
        kind, M, N, D, seed = spec
        return cm.NSGA3(population_size=N, max_generations=T, problem=getattr(cm, f"DTLZ{kind}")(D, M),
                        seed=seed, print_progress=False)

    def timed_run(step, stream):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(T)]
        for e0, e1 in ev:
            e0.record(stream)
            step()
            e1.record(stream)
        torch.cuda.synchronize()
        return [e0.elapsed_time(e1) for e0, e1 in ev]

    t0 = time.perf_counter()
    batch = cm.Batch([make(s) for s in specs], autotune=not args.batch_default_schedule)
    tune_s = time.perf_counter() - t0
    torch.cuda.synchronize()
    batch_ms = timed_run(batch.step, batch.stream)

    shared = torch.cuda.Stream()
    with torch.cuda.stream(shared):
        plain = [make(s) for s in specs]
        for a in plain:
            a.initialize()
        torch.cuda.synchronize()

        def plain_step():
            for a in plain:
                a.step()
        plain_ms = timed_run(plain_step, shared)
    identical = True
    for i, a in enumerate(plain):
        r_b, r_p = batch.result(i), a.result()
        identical &= bool(torch.equal(r_b.auxiliary_indices, r_p.auxiliary_indices))
        identical &= bool(torch.equal(r_b.objectives, r_p.objectives))
    identical = over_ranks(0.0 if identical else 1.0, "max", world, "cuda") == 0.0
    n = len(all_specs)
    windows = {}
    for name, (lo, hi) in (("generations 1-5", (0, 5)), ("generations 96-100", (95, 100)),
                           ("generations 196-200", (195, 200))):
        if hi > T:
            continue
        b = over_ranks(sum(batch_ms[lo:hi]), "max", world, "cuda")
        p = over_ranks(sum(plain_ms[lo:hi]), "max", world, "cuda")
        windows[name] = {"instance_gen_per_s": n * (hi - lo) / (b / 1e3),
                         "plain_loop_instance_gen_per_s": n * (hi - lo) / (p / 1e3), "speedup": p / b}
    b_total = over_ranks(sum(batch_ms), "max", world, "cuda")
    p_total = over_ranks(sum(plain_ms), "max", world, "cuda")
    sched = batch.schedule
    out = {"workload": BATCH_WORKLOAD, "instances": n, "span": f"all {T} generations, each timed",
           "instance_gen_per_s": n * T / (b_total / 1e3),
           "plain_loop_instance_gen_per_s": n * T / (p_total / 1e3),
           "speedup_vs_plain_loop": p_total / b_total, "windows": windows,
           "identical_ranks": identical, "fused": batch.fused,
           "graph_kernels_per_generation": batch.graph_kernels,
           "schedule": {"groups": sched["groups"], "source": sched["source"], "tuned_ms": sched["tuned_ms"],
                        "default_ms": sched["default_ms"], "slowest_instance_ms": sched["slowest_instance_ms"],
                        "instances_serial_ms": sched["instances_serial_ms"], "tuning_and_setup_s": tune_s,
                        "half_width_tiles_for_M": sched["half_tiles"]},
           "pair_tests_per_generation": sum((2 * s[2]) ** 2 for s in all_specs),
           "sharding": f"{world} rank(s), instances balanced by pair tests"}
    batch.close()
    del plain
    return out


# Further workloads of the path (one JSON line each, same timing rules): the
# small NSGA-III run, RVEA at large D (HBM-bound variation and evaluation) and
# constrained NSGA-III with ten objectives.
OTHER_WORKLOADS = {
    "dtlz2-small": dict(desc="NSGA-III DTLZ2 M=3 D=12 N=92, Das-Dennis H=12 (91 directions), 100-generation run",
                        algo="NSGA3", problem=("DTLZ2", 12, 3), N=92, T=100, dirs=("dd", 12)),
    "rvea-large-d": dict(desc="RVEA DTLZ2 M=8 D=131072 N=1024, adaptive two-layer directions, 100-generation run",
                         algo="RVEA", problem=("DTLZ2", 131072, 8), N=1024, T=100, dirs=None),
    "c1dtlz1-m10": dict(desc="constrained NSGA-III C1-DTLZ1 M=10 D=14 N=16384, two-layer (3,2) user "
                             "directions (275), 100-generation run",
                        algo="NSGA3", problem=("C1DTLZ1", 14, 10), N=16384, T=100, dirs=("two", 3, 2)),
    # the headline configuration's other reading: 255 partitions give the
    # 32896 directions its description quotes (254 give 32640)
    "dtlz1-h255": dict(desc="NSGA-III DTLZ1 M=3 D=7 N=32768, Das-Dennis 255 partitions (32896 directions), "
                            "50-generation run",
                       algo="NSGA3", problem=("DTLZ1", 7, 3), N=32768, T=50, dirs=("dd", 255)),
    # many objectives: the default association is the tensor-core search here
    "dtlz2-m8": dict(desc="NSGA-III DTLZ2 M=8 D=17 N=6436, Das-Dennis H=8 (6435 directions), 100-generation run",
                     algo="NSGA3", problem=("DTLZ2", 17, 8), N=6436, T=100, dirs=("dd", 8)),
}


# association searches compared on the same runs (all give identical results)
ASSOC_FORMS = {0: "cone tree", 1: "FP32 scan", 2: "tensor cores (split TF32, exact re-score)"}
PRECISION_WORKLOADS = [
    {"desc": "headline: DTLZ1 M=3 D=7 N=32768, 32640 directions", "problem": "DTLZ1", "D": D_VAR, "M": M_OBJ,
     "N": N_POP, "partitions": PARTITIONS, "modes": (0, 1, 2)},
    {"desc": "many objectives: DTLZ2 M=8 D=17 N=6436, 6435 directions", "problem": "DTLZ2", "D": 17, "M": 8,
     "N": 6436, "partitions": 8, "modes": (1, 2)},
    # the constrained config: below the default's 2^24-pair threshold the
    # default takes the FP32 scan; both are timed here
    {"desc": "constrained, ten objectives: C1-DTLZ1 M=10 D=14 N=16384, two-layer (3,2) directions (275)",
     "problem": "C1DTLZ1", "D": 14, "M": 10, "N": 16384, "two_layer": (3, 2), "modes": (1, 2)},
]


def precision_form(torch, cm, seed: int, gens: int = 4):
    """Association stage time of each search on the same seeded run, and
    whether the runs stay identical.  At M=3 the cone tree visits about 1% of
    the directions, so the dense tensor-core contraction does not beat it; above
    five objectives the default search is the tensor-core one."""
    out = []
    for w in PRECISION_WORKLOADS:
        rec = {"workload": w["desc"], "associate_ms": {}, "identical_runs": True}
        ref = None
        for mode in w["modes"]:
            dirs = (cm.UserDefinedDirections(cm.two_layer_directions(w["M"], *w["two_layer"]))
                    if "two_layer" in w else cm.DasDennisDirections(w["partitions"]))
            algo = cm.NSGA3(population_size=w["N"], max_generations=gens + 4, problem=getattr(cm, w["problem"])(w["D"], w["M"]),
                            reference_directions=dirs, seed=seed, print_progress=False,
                            environment_selector=cm.NSGA3EnvironmentSelector(association_mode=mode))
            algo.initialize()
            for _ in range(gens):
                algo.step()
            times = [dict(algo.profile_step())["select.associate"] for _ in range(3)]
            x = algo.population.variables.cpu()
            rec["associate_ms"][ASSOC_FORMS[mode]] = sorted(times)[1]
            if ref is None:
                ref = x
            elif not torch.equal(ref, x):
                rec["identical_runs"] = False
            del algo
            torch.cuda.empty_cache()
        out.append(rec)
    return out


def measure_workload(name, steps, warmup, seed, torch, cm):
    """One of OTHER_WORKLOADS timed like the headline: `steps` generations
    after `warmup`, CUDA events on the algorithm's stream, L2 flushed before
    every timed generation, clocks sampled during the timed region."""
    w = OTHER_WORKLOADS[name]
    kind, D, M = w["problem"]
    kw = {}
    if w["dirs"] and w["dirs"][0] == "dd":
        kw["reference_directions"] = cm.DasDennisDirections(w["dirs"][1])
    elif w["dirs"]:
        kw["reference_directions"] = cm.UserDefinedDirections(cm.two_layer_directions(M, *w["dirs"][1:]))
    algo = cm.Algorithm(w["algo"], population_size=w["N"], max_generations=w["T"],
                        problem=getattr(cm, kind)(D, M), seed=seed, print_progress=False, **kw)
    stream = torch.cuda.current_stream()
    algo.initialize()
    for _ in range(warmup):
        algo.step()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(steps)]
    torch.cuda.synchronize()
    with ClockSampler(torch.cuda.current_device()) as clocks:
        for e0, e1 in events:
            flush.fill_(1)
            e0.record(stream)
            algo.step()
            e1.record(stream)
        torch.cuda.synchronize()
    total_ms = sum(e0.elapsed_time(e1) for e0, e1 in events)
    graph_on, kernels = algo.graph_info
    out = {"metric": f"{w['algo']} gen/s", "value": steps / (total_ms / 1e3), "unit": "gen/s",
           "n_gpus": 1, "steps": steps, "warmup": warmup, "ms_per_step": total_ms / steps,
           "higher_is_better": True, "dtype": "f32", "data": "synthetic",
           "config": {"workload": w["desc"], "cuda_graph": graph_on, "kernels_per_generation": kernels,
                      "l2": "flushed (256 MiB write) before every timed generation"},
           "clocks": clocks.summary()}
    if name in ("dtlz2-m8", "c1dtlz1-m10", "dtlz1-h255"):
        out["stages_ms"] = dict(algo.profile_step())
    if name == "rvea-large-d":
        # the generation's streamed bytes, 8 N D: the variation reads two
        # parents and writes two children per pair element (8 N D); the
        # evaluation reads the children, the survivor update reads and writes
        # the surviving rows (both bounded by further 4 N D each, not counted)
        bytes_ = 8.0 * w["N"] * D
        hbm, kind_ = _peaks()
        ms = total_ms / steps
        out["roofline"] = {"kernel": "whole generation (crossover_philox, mutation_philox, dtlz_block_rows, "
                                     "RVEA selection, rvea_update)", "bound": "hbm",
                           "achieved": bytes_ / (ms / 1e3) / 1e9, "peak": hbm, "unit": "GB/s",
                           "frac": bytes_ / (ms / 1e3) / 1e9 / hbm, "peak_source": kind_,
                           "algorithmic_bytes": bytes_}
        out["stages_ms"] = dict(algo.profile_step())
    del algo
    torch.cuda.empty_cache()
    return out


def other_workload(args, torch, cm):
    print(json.dumps(measure_workload(args.workload, args.steps, args.warmup, args.seed, torch, cm)))


QUALITY = ("DTLZ2 M=3 D=12, N=1024 (RVEA: 990), 500 generations, seeds 0..29: the reference's published "
           "quality protocol (tests/benchmark/DTLZ/plan.py quality_jobs, adapters/dtlz.py _run_cuda): initial "
           "population uniform from torch's CPU generator seeded per run, SBX eta 30 pc 1 copy 0.5, PM eta 20, "
           "NSGA-III on 990 Das-Dennis directions (H=43, clamped >= 1e-6), RVEA adaptive (frequency 0.1, "
           "alpha 2); IGD in FP64 against 20000 seeded sphere samples (tests/evaluation/pareto_front.py)")
# tests/benchmark/DTLZ/results/data/quality_summary.csv:14-16, 20-22 (30 runs each, RTX PRO 6000)
PUBLISHED_QUALITY = {"NSGA3": {"igd_mean": 0.0168882529505434, "igd_std": 2.1336646294516216e-05,
                               "ms_per_gen_mean": 0.4569740997314453},
                     "RVEA": {"igd_mean": 0.01699151074727422, "igd_std": 4.04198196642769e-06,
                              "ms_per_gen_mean": 0.13019642740885418}}


def quality_runs(torch, cm, seeds: int = 30, generations: int = 500):
    """Final IGD and mean ms per generation of NSGA-III and RVEA over seeded
    runs of the reference's quality protocol, beside its published numbers
    (Welch's t of the mean IGD difference)."""
    from cuda_moea import metrics, stages
    ref = metrics.pareto_front_points("DTLZ2", 3, 20000, 2887).to(torch.float64).cuda()
    dirs = stages.reference_directions(2, 1024, 3).t().contiguous()   # 990 x 3, clamped
    out = {}
    for name in ("NSGA3", "RVEA"):
        N = 1024 if name == "NSGA3" else 990
        igds, mss = [], []
        for seed in range(seeds):
            gen = torch.Generator(device="cpu").manual_seed(seed)
            x0 = torch.empty((N, 12), dtype=torch.float32).uniform_(0.0, 1.0, generator=gen)
            kw = dict(population_size=N, max_generations=generations, problem=cm.DTLZ2(12, 3), seed=seed,
                      print_progress=False, initial_population=x0,
                      crossover=cm.SBX(probability=1.0, eta_initial=30.0, eta_final=30.0,
                                       variable_copy_probability=0.5),
                      mutation=cm.PolynomialMutation(probability=1.0, eta_initial=20.0, eta_final=20.0))
            if name == "NSGA3":
                kw["environment_selector"] = cm.NSGA3EnvironmentSelector(sparse_ratio=1.0)
                kw["reference_directions"] = cm.UserDefinedDirections(dirs)
            else:
                kw["environment_selector"] = cm.RVEAEnvironmentSelector(alpha=2.0)
                kw["reference_directions"] = cm.AdaptiveRVEADirections(frequency=0.1)
            r = cm.Algorithm(name, **kw).run()
            front = r.objectives[: r.active_count]
            igds.append(metrics.igd(front, ref))
            mss.append(r.total_ms / generations)
        pub = PUBLISHED_QUALITY[name]
        mean, std = statistics.mean(igds), statistics.stdev(igds)
        welch = (mean - pub["igd_mean"]) / ((std ** 2 + pub["igd_std"] ** 2) / seeds) ** 0.5
        out[name] = {"runs": seeds, "population": N, "igd_mean": mean, "igd_std": std,
                     "igd_median": statistics.median(igds), "ms_per_gen_mean": statistics.mean(mss),
                     "published": pub, "welch_t_vs_published": welch}
    return out


CONSTRAINED_BATCH = ("batched constrained NSGA-III: 64 seeds per launch of C1-DTLZ1 and of C3-DTLZ4, M=10, D=14, "
                     "N=16384, two-layer (3,2) user directions (275), 100-generation runs")


def constrained_batch(args, torch, cm):
    """The constrained ten-objective configuration: for each problem, 64
    seeded instances advance together (one graph launch per generation,
    instances as parallel branches), against the same instances looped
    through the plain path; afterwards every instance's ranks and objectives
    are compared.  value = instance-generations/s over both problems."""
    D, M, N, T, seeds = 14, 10, 16384, 100, 64
    dirs = cm.two_layer_directions(M, 3, 2)
    warm, K = max(args.warmup, 3), max(1, min(args.steps, 5))

    def make(kind, seed):
        return cm.NSGA3(population_size=N, max_generations=T, problem=getattr(cm, kind)(D, M), seed=seed,
                        reference_directions=cm.UserDefinedDirections(dirs), print_progress=False)

    records, batch_total, plain_total, gens = [], 0.0, 0.0, 0
    with ClockSampler(0) as clocks:
        for kind in ("C1DTLZ1", "C3DTLZ4"):
            batch = cm.Batch([make(kind, s) for s in range(seeds)])
            batch.run(warm)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(batch.stream)
            for _ in range(K):
                batch.step()
            e1.record(batch.stream)
            torch.cuda.synchronize()
            batch_ms = e0.elapsed_time(e1)
            shared = torch.cuda.Stream()
            with torch.cuda.stream(shared):
                plain = [make(kind, s) for s in range(seeds)]
                for a in plain:
                    a.initialize()
                for _ in range(warm):
                    for a in plain:
                        a.step()
                torch.cuda.synchronize()
                p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                p0.record(shared)
                for _ in range(K):
                    for a in plain:
                        a.step()
                p1.record(shared)
                torch.cuda.synchronize()
            plain_ms = p0.elapsed_time(p1)
            identical = True
            feasible = 0
            for i, a in enumerate(plain):
                r_b, r_p = batch.result(i), a.result()
                identical &= bool(torch.equal(r_b.auxiliary_indices, r_p.auxiliary_indices))
                identical &= bool(torch.equal(r_b.objectives, r_p.objectives))
                identical &= bool(torch.equal(r_b.constraints, r_p.constraints))
                feasible += int((r_b.constraints == 0).sum())
            records.append({"problem": kind, "instances": seeds, "generations_timed": K,
                            "instance_gen_per_s": seeds * K / (batch_ms / 1e3),
                            "plain_loop_instance_gen_per_s": seeds * K / (plain_ms / 1e3),
                            "speedup_vs_plain_loop": plain_ms / batch_ms, "identical_ranks": identical,
                            "feasible_fraction": feasible / (seeds * N), "fused": batch.fused,
                            "graph_kernels_per_generation": batch.graph_kernels})
            batch_total += batch_ms
            plain_total += plain_ms
            gens += seeds * K
            batch.close()
            del plain, batch
            torch.cuda.empty_cache()
    print(json.dumps({
        "metric": "batched constrained NSGA-III instance-gen/s", "value": gens / (batch_total / 1e3),
        "unit": "instance-gen/s", "n_gpus": 1, "steps": K, "warmup": warm,
        "ms_per_step": batch_total / (2 * K), "higher_is_better": True, "dtype": "f32", "data": "synthetic",
        "config": {"workload": CONSTRAINED_BATCH, "directions": int(dirs.shape[0]),
                   "l2": "inputs larger than L2 (64 dominance relations of 128 MiB per generation)"},
        "clocks": clocks.summary(), "plain_loop_value": gens / (plain_total / 1e3),
        "records": records}))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--population", type=int, default=N_POP)
    ap.add_argument("--seed", type=int, default=2887)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=40.0)
    ap.add_argument("--batch-instances", type=int, default=256)
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--batch-generations", type=int, default=200,
                    help="generations of the batched record (fewer only for launch-list captures)")
    ap.add_argument("--batch-default-schedule", action="store_true",
                    help="the batch's default schedule instead of the autotuned one (launch-list captures)")
    ap.add_argument("--no-precision", action="store_true", help="skip the association-search comparison")
    ap.add_argument("--no-rvea", action="store_true", help="skip the RVEA large-D record")
    ap.add_argument("--workload", default="dtlz1-n32768",
                    choices=["dtlz1-n32768", "constrained-batch", "quality", *OTHER_WORKLOADS])
    ap.add_argument("--quality-seeds", type=int, default=30)
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
        return
    args.warmup = max(args.warmup, 3)

    import torch
    if args.workload != "dtlz1-n32768":
        import cuda_moea as cm
        torch.cuda.set_stream(torch.cuda.Stream(0))
        if args.workload == "constrained-batch":
            constrained_batch(args, torch, cm)
        elif args.workload == "quality":
            q = quality_runs(torch, cm, seeds=args.quality_seeds)
            print(json.dumps({"metric": "final IGD (DTLZ2, 500 generations)", "value": q["NSGA3"]["igd_mean"],
                              "unit": "IGD", "higher_is_better": False, "n_gpus": 1, "dtype": "f32",
                              "data": "synthetic", "config": {"workload": QUALITY}, "quality": q}))
        else:
            other_workload(args, torch, cm)
        return
    import torch.distributed as dist
    import cuda_moea as cm

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    # one non-default stream for the algorithm, the timing events and the copies
    torch.cuda.set_stream(torch.cuda.Stream(local))
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    N = args.population
    gens = args.warmup + 3 + 2 * args.steps + 2
    algo = cm.NSGA3(population_size=N, max_generations=gens, problem=cm.DTLZ1(D_VAR, M_OBJ),
                    reference_directions=cm.DasDennisDirections(PARTITIONS), seed=replica_seed(args.seed, rank),
                    print_progress=False, device=local)
    stream = torch.cuda.current_stream()
    algo.initialize()
    for _ in range(args.warmup):
        algo.step()
    torch.cuda.synchronize()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    # host buffers of the end-to-end path (pinned): the population in, the results out
    pop = algo.population
    h_vars = torch.empty((N, D_VAR), dtype=torch.float32, pin_memory=True)
    h_vars.copy_(pop.variables)
    h_objs = torch.empty((N, M_OBJ), dtype=torch.float32, pin_memory=True)
    h_cv = torch.empty(N, dtype=torch.float32, pin_memory=True)

    def e2e_step(e0=None, e1=None):
        """One generation through the public API from and to host memory."""
        flush.fill_(1)
        if e0 is not None:
            e0.record(stream)
        p = algo.population_view()
        p.variables.copy_(h_vars, non_blocking=True)
        algo.step()
        p = algo.population_view()
        # the whole next population back to the host: objectives, violations
        # and the decision vectors (the next step's input)
        h_objs.copy_(p.objectives, non_blocking=True)
        h_cv.copy_(p.constraints, non_blocking=True)
        h_vars.copy_(p.variables, non_blocking=True)
        if e1 is not None:
            e1.record(stream)
        torch.cuda.synchronize()

    for _ in range(3):  # untimed warm-up of the host-copy path
        e2e_step()

    # ---- timed region: K generations with inputs resident in HBM (device
    # time), each followed by one end-to-end generation with host copies, so
    # that both figures sample the same stretch of the run
    events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(args.steps)]
    ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        for (e0, e1), (f0, f1) in zip(events, ev2):
            flush.fill_(1)
            e0.record(stream)
            algo.step()
            e1.record(stream)
            e2e_step(f0, f1)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    total_ms = sum(e0.elapsed_time(e1) for e0, e1 in events)
    max_ms = over_ranks(total_ms, "max", world, "cuda")
    value = world * args.steps / (max_ms / 1000.0)
    graph_on, kernels = algo.graph_info
    e2e_ms = sum(e0.elapsed_time(e1) for e0, e1 in ev2)
    e2e_value = world * args.steps / (over_ranks(e2e_ms, "max", world, "cuda") / 1000.0)

    # ---- per-stage device times of one generation (direct launches, events)
    stages = algo.profile_step()
    stage_ms = {}
    for name, ms in stages:
        stage_ms[name] = stage_ms.get(name, 0.0) + ms
    n_mix = 2 * N
    rooflines = kernel_rooflines(stage_ms, n_mix, N == N_POP)

    # the same stages at generation 0 from the fixed population that the
    # reference arm times its own stages on (stage_population): same parents
    stages0 = None
    if N == N_POP:
        del pop
        algo0 = cm.NSGA3(population_size=N, max_generations=gens, problem=cm.DTLZ1(D_VAR, M_OBJ),
                         reference_directions=cm.DasDennisDirections(PARTITIONS), seed=args.seed,
                         initial_population=stage_population(N)[:N], print_progress=False, device=local)
        algo0.initialize()
        stages0 = {}
        for name, ms in algo0.profile_step():
            stages0[name] = stages0.get(name, 0.0) + ms
        del algo0

    precision = None
    if not args.no_precision:
        precision = precision_form(torch, cm, replica_seed(args.seed, rank))

    # RVEA at large D (the HBM-streaming workload) as a record of the line
    rvea = None
    if not args.no_rvea:
        algo = None
        torch.cuda.empty_cache()
        rvea = measure_workload("rvea-large-d", 10, 3, replica_seed(args.seed, rank), torch, cm)

    batched = None
    if not args.no_batch:
        algo = None
        torch.cuda.empty_cache()
        batched = batched_measure(args, torch, cm, world, rank)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        t_cpu = cpu_generation_time(N, threads)
        cpu = {"value": 1.0 / t_cpu, "unit": "gen/s", "cores": threads, "kind": "port",
               "sample": f"1 full generation of the workload on the CPU oracle (OpenMP, {threads} threads)"}

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": "gen/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": max_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "population": N, "merged": n_mix, "directions": 32640,
                       "l2": "flushed (256 MiB write) before every timed generation",
                       "parallelism": f"replicas x{world}", "cuda_graph": graph_on},
            "clocks": clocks.summary(),
            "e2e": {"value": e2e_value, "unit": "gen/s",
                    "h2d_bytes_per_step": N * D_VAR * 4, "d2h_bytes_per_step": N * (D_VAR + M_OBJ + 1) * 4},
            # graph kernels of the K device-timed and the K end-to-end generations
            "gpu_launches": kernels * 2 * args.steps,
            "stages_ms": stage_ms,
            # the dominant kernel of the generation, then every heavy kernel
            "roofline": rooflines[0],
            "roofline_kernels": rooflines,
            "stages_ms_generation0": stages0,
            "cpu_baseline": cpu,
            "precision_form": precision,
            "batched": batched,
            "rvea_large_d": rvea,
        }
        print(json.dumps(out))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
