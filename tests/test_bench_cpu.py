"""CPU: the measurement arithmetic of bench.py (no GPU).

The roofline entries restate the algorithmic work per launch and divide by
the stage time; these checks recompute them from the constants they are
built on, so that a changed constant or unit shows up here rather than as
a silently wrong fraction in the JSON line.  The batched workload's sharding
must put every instance on exactly one rank and balance the pair tests."""
import bench


def test_peel_roofline_is_lower_triangle_bytes_over_time():
    n = 65536
    ms = 0.28
    [peel] = [r for r in bench.kernel_rooflines({"ndsort.peel": ms}, n, True)]
    tri_bytes = n * (n - 1) / 2 / 8
    assert peel["algorithmic_bytes"] == tri_bytes
    assert abs(peel["achieved"] - tri_bytes / (ms / 1e3) / 1e9) < 1e-6
    assert abs(peel["frac"] - peel["achieved"] / peel["peak"]) < 1e-12
    assert peel["unit"] == "GB/s" and peel["bound"] == "hbm"
    assert peel["traffic"] == bench.PEEL_DRAM_BYTES


def test_dominance_roofline_counts_lsu_wavefronts_and_lane_ops():
    n = 65536
    ms = 0.16
    rows = {r["kernel"]: r for r in bench.kernel_rooflines({"ndsort.dominance_tiles": ms}, n, True)}
    [r] = [v for k, v in rows.items() if k.startswith("nds_block_rows")]
    peak = 148 * 1.965e9
    assert abs(r["peak"] - peak) < 1.0
    assert abs(r["achieved"] - bench.ROWS_LSU_WAVEFRONTS / (ms / 1e3)) < 1.0
    pairs = n * (n - 1) / 2
    assert abs(r["lane_ops_per_pair"] - bench.ROWS_WARP_INSTR * 32 / pairs) < 1e-12
    simt = pairs / (ms / 1e3) * r["lane_ops_per_pair"] / (148 * 128 * 1.965e9)
    assert abs(r["simt_frac"] - simt) < 1e-12
    # the counted work is what a launch at this size does: about 1.3 lane-ops per pair
    assert 1.0 < r["lane_ops_per_pair"] < 2.0
    # other workloads carry no dominance entry (the counts are for this size)
    assert not [k for k in (x["kernel"] for x in bench.kernel_rooflines({"ndsort.dominance_tiles": ms}, n, False))
                if k.startswith("nds_block_rows")]


def test_rooflines_are_sorted_by_stage_time():
    out = bench.kernel_rooflines({"ndsort.peel": 0.1, "ndsort.dominance_tiles": 0.2}, 65536, True)
    assert [r["ms"] for r in out] == sorted((r["ms"] for r in out), reverse=True)


def test_batch_shards_cover_every_instance_once_and_balance_pairs():
    specs = bench.batch_specs(256)
    for world in (1, 2, 3, 8):
        owned = [bench.shard_instances(specs, world, r) for r in range(world)]
        flat = sorted(i for o in owned for i in o)
        assert flat == list(range(len(specs)))
        loads = [sum((2 * specs[i][2]) ** 2 for i in o) for o in owned]
        # greedy largest-first: no rank exceeds the mean by more than the largest instance
        biggest = max((2 * s[2]) ** 2 for s in specs)
        assert max(loads) - sum(loads) / world <= biggest


def test_batch_specs_match_the_workload_description():
    specs = bench.batch_specs(256)
    assert len(specs) == 256
    for kind, M, N, D, seed in specs:
        assert 1 <= kind <= 7 and M in (3, 5, 8)
        assert 92 <= N <= 4096 and N % 2 == 0
        assert D == M + (19 if kind == 7 else 9)
    assert [s[4] for s in specs] == list(range(256))
