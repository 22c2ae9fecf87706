"""Host dispatch of independent solves over ranks (lbm_b200.dispatch).

Single process: the shares are disjoint, cover every solve and stay balanced.
Two gloo ranks on the CPU (the same code path a two-GPU run takes for its
host plumbing): every rank derives the same assignment without exchanging
it, the max-over-ranks timing is the maximum, and a rank that leaves before
the barrier turns the other rank's barrier into an error instead of a hang.
"""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "jianhui-lbm_b200"))

from lbm_b200 import dispatch  # noqa: E402


def test_shard_partitions_and_balances():
    rng = np.random.default_rng(7)
    w = rng.lognormal(13, 1.2, size=64)
    for world in (1, 2, 3, 4, 8):
        shares = [dispatch.shard(w, world, r) for r in range(world)]
        flat = sorted(i for s in shares for i in s)
        assert flat == list(range(len(w)))
        loads = [w[s].sum() for s in shares]
        # longest-processing-time bound: the spread never exceeds the largest item
        assert max(loads) - min(loads) <= w.max() + 1e-6
    assert dispatch.shard([], 2, 1) == []
    with pytest.raises(ValueError):
        dispatch.shard(w, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir, leave_early):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, os.path.join(ROOT, "jianhui-lbm_b200"))
    from lbm_b200 import dispatch as D

    pg = D.init_process_group(timeout_s=20)
    w = [float(x) for x in np.random.default_rng(3).integers(1, 1000, size=37)]
    mine = D.shard(w, world, rank)
    gathered = [None] * world
    pg.all_gather_object(gathered, mine)
    tmax = D.max_over_ranks(pg, 1.5 + rank)
    if leave_early and rank == 1:
        os._exit(0)  # leaves between steps, with nothing in flight
    status = "ok"
    try:
        D.barrier(pg)
    except Exception as ex:  # the peer is gone
        status = "error: " + type(ex).__name__
    with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
        f.write(repr((gathered, tmax, status)))
    if status == "ok":
        pg.destroy_process_group()


def _run(world, leave_early, tmp_path):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, str(tmp_path), leave_early)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        if p.is_alive():
            p.kill()
            pytest.fail("a rank did not finish")
    import ast

    return {r: ast.literal_eval((tmp_path / f"rank{r}.txt").read_text())
            for r in range(world) if (tmp_path / f"rank{r}.txt").exists()}


def test_two_gloo_ranks_agree(tmp_path):
    res = _run(2, False, tmp_path)
    assert set(res) == {0, 1}
    g0, t0, s0 = res[0]
    g1, t1, s1 = res[1]
    assert g0 == g1
    assert sorted(g0[0] + g0[1]) == list(range(37)) and not set(g0[0]) & set(g0[1])
    assert t0 == t1 == 2.5
    assert s0 == s1 == "ok"


def test_rank_leaving_is_an_error_not_a_hang(tmp_path):
    res = _run(2, True, tmp_path)
    assert set(res) == {0}
    assert res[0][2].startswith("error")
