"""One matrix computed by two processes (gloo ranks on one GPU, no kernel of
one waits on the other's) on disjoint stripe windows through the product's
partial entry point (ssu_b200_partial_inmem_v3), each written to a partial
file (write_partial); rank 0 then reads the headers and merges the files
(merge_partial_to_mmap_matrix), as the reference's `ssu --mode partial`
then `--mode merge-partial` (src/su.cpp:347-399, ci/crawford_test.sh).  The
merged matrix equals the one-call matrix bit for bit."""
import os
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, outdir, method, out_q):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "unifrac-binaries_b200"))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=120))
    try:
        import bench
        import ssu_b200
        import ssu_synth
        tree = ssu_synth.random_binary_tree(1500, 0.05, 91)
        table = ssu_synth.lognormal_table(tree.tip_names(), 700, 0.03, 2.0, 1.5, 92)
        start, stop = bench.stripe_window(table.n_samples, rank, world)
        path = os.path.join(outdir, f"rank{rank}.partial")
        ssu_b200.partial_to_file(tree, table, method, start, stop, path)
        dist.barrier()
        if rank == 0:
            paths = [os.path.join(outdir, f"rank{r}.partial") for r in range(world)]
            merged, ids = ssu_b200.merge_partial_files(paths[::-1], mmap_dir=outdir)
            full, full_ids = ssu_b200.one_off_matrix(tree, table, method)
            out_q.put({"equal": bool(np.array_equal(merged, full)), "ids": ids == full_ids,
                       "windows": [bench.stripe_window(table.n_samples, r, world) for r in range(world)]})
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("method", ["weighted_normalized_fp64", "unweighted_fp64"])
def test_two_ranks_write_partials_and_rank_0_merges(tmp_path, method):
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, str(tmp_path), method, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert res["equal"] and res["ids"]
    (a0, a1), (b0, b1) = res["windows"]
    assert a0 == 0 and a1 == b0 and b1 == (700 + 1) // 2
