"""The multi-rank path of bench.py on the CPU: two ranks over gloo.

Replicas shard across ranks with no collective in the step; the only
collectives are the timing reductions.  These tests run them as two ranks:
  * the rank environment and the process group (bench.dist_env / dist_init);
  * max_over_ranks (the device time of the slowest rank) and sum_over_ranks
    (the work of all ranks), on rank-specific values;
  * the replica shard of each rank: rank r generates replicas r*R .. r*R+R-1,
    so the ranks hold different systems;
  * the reference arm under N > 1: ranks other than 0 exit at once, printing
    nothing.
"""
import json
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

WORLD = 2


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(WORLD), LOCAL_RANK=str(rank))
    try:
        import bench
        from md_nucleation_b200 import generate
        ws, r, local = bench.dist_env()
        dist = bench.dist_init(ws, local, "gloo")
        # rank r reports a device time of 10 + r ms and 100 * (r + 1) atom-steps
        t_max = bench.max_over_ranks(dist, 10.0 + r, "cpu")
        work = bench.sum_over_ranks(dist, 100.0 * (r + 1), "cpu")
        # the shard of this rank: replicas r*R .. r*R+R-1 (small versions)
        R = 2
        shard = [generate.config2_replica(r * R + i, scale=0.02) for i in range(R)]
        digest = [float(np.asarray(s.gas_x).sum()) for s in shard]
        dist.barrier()
        dist.destroy_process_group()
        q.put((r, ws, t_max, work, digest))
    except Exception as e:  # reported to the parent
        q.put((rank, "error", repr(e)))


def test_two_ranks_over_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, port, q)) for r in range(WORLD)]
    for p in procs:
        p.start()
    out = {}
    try:
        for _ in range(WORLD):
            item = q.get(timeout=240)
            assert item[1] != "error", item
            out[item[0]] = item
    finally:
        for p in procs:
            p.join(timeout=30)
            if p.is_alive():
                p.kill()
                p.join()
    assert sorted(out) == [0, 1]
    for r in range(WORLD):
        _, ws, t_max, work, _ = out[r]
        assert ws == WORLD
        assert t_max == 11.0          # the slowest rank's time, seen by every rank
        assert work == 300.0          # every rank's atom-steps
    # the two shards are different systems
    assert not np.allclose(out[0][4], out[1][4])


def test_reference_arm_other_ranks_exit_quietly(monkeypatch, capsys):
    import bench
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("LOCAL_RANK", "1")

    class Args:
        replicas, warmup, steps, ref_budget = 4, 3, 1, 1.0
    assert bench.run_reference(Args()) == 0
    assert capsys.readouterr().out == ""


def test_single_rank_needs_no_process_group(monkeypatch):
    import bench
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    ws, r, local = bench.dist_env()
    assert (ws, r, local) == (1, 0, 0)
    assert bench.dist_init(ws, local, "gloo") is None
    assert bench.max_over_ranks(None, 3.5, "cpu") == 3.5
    assert bench.sum_over_ranks(None, 7.0, "cpu") == 7.0
