"""The multi-GPU path (replicas) on CPU: two gloo ranks, as torchrun would start them.

Each rank takes its round-robin share of the pair list (the rule of the CLI's --shard r/W
and of bench.py's per-rank pairs), the shares cover every pair exactly once, and the
whole-job throughput is all ranks' units over the slowest rank's time."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, pairs, out):
    import importlib.util
    import sys
    from pathlib import Path

    root = Path(__file__).resolve().parents[1] / "piv_xcorr2d_v1.0_b200"
    spec = importlib.util.spec_from_file_location("piv_b200_replicas", root / "replicas.py")
    R = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(R)
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    r, w, _ = R.init(backend="gloo", timeout_s=60)
    mine = R.shard(pairs, r, w)
    seconds = 1.0 + r  # rank 1 is the slow one
    thr = R.throughput(len(mine), seconds, w)
    import torch.distributed as dist

    gathered = [None] * w
    dist.all_gather_object(gathered, mine)
    R.finish(w)
    out.put((r, mine, thr, gathered))
    sys.exit(0)


def test_two_gloo_ranks_shard_and_time():
    pairs = list(range(1, 12))
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, pairs, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=90) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    (r0, m0, t0, g0), (r1, m1, t1, g1) = res
    assert m0 == pairs[0::2] and m1 == pairs[1::2]
    assert sorted(m0 + m1) == pairs and not set(m0) & set(m1)
    assert g0 == g1 == [m0, m1]
    assert t0 == pytest.approx(len(pairs) / 2.0) and t1 == t0


def test_shard_rule_matches_cli():
    import importlib.util
    from pathlib import Path

    root = Path(__file__).resolve().parents[1] / "piv_xcorr2d_v1.0_b200"
    spec = importlib.util.spec_from_file_location("piv_b200_replicas2", root / "replicas.py")
    R = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(R)
    assert R.shard([5, 6, 7, 8, 9], 1, 3) == [6, 9]
    with pytest.raises(ValueError):
        R.shard([1], 3, 3)
