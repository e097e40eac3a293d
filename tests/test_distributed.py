"""N > 1 paths on CPU with gloo, world size 2: the rank aggregation bench.py
uses (max time, summed units), and one matrix split into disjoint stripe
windows, one per rank, computed independently and gathered — no exchange
during compute — equal to the single-process matrix."""
import os
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, out_q):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    for p in ("unifrac-binaries_b200", "oracle"):
        sys.path.insert(0, os.path.join(ROOT, p))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        import oracle_py
        import ssu_synth
        step, e2e, units, pair = bench.combine_ranks([10.0 + rank, 5.0 * (rank + 1), 100.0, 2.0 - rank], world, "cpu")
        tree = ssu_synth.random_binary_tree(80, 0.1, 5)
        table = ssu_synth.geometric_table(tree.tip_names(), 45, 0.15, 8.0, 6)
        start, stop = bench.stripe_window(table.n_samples, rank, world)
        part = oracle_py.oracle_one_off(tree, table, "weighted_normalized_fp64", stripe_start=start,
                                        stripe_stop=stop)["stripes"]
        gathered = [None] * world
        dist.all_gather_object(gathered, (start, stop, part))
        if rank == 0:
            out_q.put({"agg": (step, e2e, units, pair), "gathered": gathered})
    finally:
        dist.destroy_process_group()


@pytest.fixture(scope="module")
def two_rank_result():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return res


def test_rank_aggregation_is_max_time_and_summed_units(two_rank_result):
    step, e2e, units, pair = two_rank_result["agg"]
    assert step == 11.0 and e2e == 10.0 and units == 200.0 and pair == 2.0


def test_stripe_windows_partition_and_gather_to_the_full_matrix(two_rank_result, oracle_mod):
    import ssu_synth
    gathered = sorted(two_rank_result["gathered"], key=lambda g: g[0])
    assert gathered[0][0] == 0 and gathered[0][1] == gathered[1][0] and gathered[1][1] == 23
    stripes = np.concatenate([g[2] for g in gathered])
    tree = ssu_synth.random_binary_tree(80, 0.1, 5)
    table = ssu_synth.geometric_table(tree.tip_names(), 45, 0.15, 8.0, 6)
    full = oracle_mod.oracle_one_off(tree, table, "weighted_normalized_fp64")["stripes"]
    np.testing.assert_array_equal(stripes, full)


@pytest.mark.parametrize("n,world", [(6, 2), (7, 3), (2048, 8), (25000, 8), (5, 4)])
def test_stripe_window_covers_every_stripe_once(n, world):
    sys.path.insert(0, ROOT)
    import bench
    total = (n + 1) // 2
    windows = [bench.stripe_window(n, r, world) for r in range(world)]
    assert windows[0][0] == 0 and windows[-1][1] == total
    assert all(windows[i][1] == windows[i + 1][0] for i in range(world - 1))


def test_clock_sampler_returns_promptly_without_a_gpu():
    import time
    sys.path.insert(0, ROOT)
    import bench
    t0 = time.monotonic()
    s = bench.ClockSampler(0)
    s.start()
    clk = s.stop()
    assert time.monotonic() - t0 < 10
    assert clk is None or {"sm_mhz", "sm_max_mhz", "reasons", "samples"} <= set(clk)


def _reference_arm(env_extra, workload="100k-tips-25k-presence"):
    import json
    import subprocess
    env = dict(os.environ)
    env.update(env_extra)
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0", "--samples", "96", "--tips", "600", "--presence-samples", "96",
                          "--presence-tips", "600", "--workload", workload],
                         capture_output=True, text=True, env=env, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    return [json.loads(x) for x in out.stdout.splitlines() if x.startswith("{")]


@pytest.mark.parametrize("workload", ["100k-tips-25k-presence", "20k-tips-2048-samples"])
def test_reference_arm_prints_one_contract_line_on_rank_0(workload):
    lines = _reference_arm({"RANK": "0", "WORLD_SIZE": "1"}, workload)
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference" and d["metric"] == "pair-branch updates/s" and d["unit"] == "updates/s"
    assert d["value"] > 0 and d["higher_is_better"] is True and d["steps"] == 1 and d["warmup"] == 0
    assert d["cpu_baseline"]["kind"] in ("reference", "port") and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    sys.path.insert(0, ROOT)
    import bench
    expected = bench.PRESENCE_WORKLOAD if workload == "100k-tips-25k-presence" else bench.WEIGHTED_WORKLOAD
    assert d["config"]["workload"] == expected  # the same string as this arm's line


def test_reference_arm_other_ranks_exit_without_work():
    assert _reference_arm({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}) == []


def test_clock_lines_parse_with_throttle_reasons():
    sys.path.insert(0, ROOT)
    import bench
    text = ("0, 1965, 1965, 512.3, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active\n"
            "0, 1500, 1965, 998.7, 0x0000000000000004, Not Active, Not Active, Not Active, Active\n"
            "0, 1200, 1965, 700.0, 0x0000000000000008, Active, Not Active, Active, Not Active\n"
            "0, [N/A], 1965, 1.0, 0x0, Not Active, Not Active, Not Active, Not Active\n"
            "garbage\n")
    rows = bench.ClockSampler.parse_smi(text)
    assert [r[0] for r in rows] == [1965.0, 1500.0, 1200.0]
    assert all(r[1] == 1965.0 for r in rows)
    assert rows[0][2] == [] and rows[1][2] == ["sw_power_cap"]
    assert rows[2][2] == ["hw_slowdown", "sw_thermal_slowdown"]
