"""Configuration 4 on several ranks (CPU, gloo, world size 2): each rank
takes a contiguous slice of the systems, no collective on the data path;
the per-system statuses are gathered in system order, the slices tile the
whole batch, and a rank that stops before the gather makes the others fail
with an error (a short process-group timeout) instead of hanging. The
device factorization itself is covered by the GPU tests on one GPU."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, count, mode, q):
    import datetime
    import torch.distributed as dist
    from opt_solver_b200.batch import gather_system_stats, shard
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=5))
    try:
        lo, hi = shard(count, rank, world)
        if mode == "drop" and rank == 1:
            q.put((rank, "left"))
            return
        # per-system stats as the engine reports them: (pos, neg, zero, 2x2, delays)
        T = np.arange(lo, hi) % 191 + 10
        stats = np.stack([16 * T + 12, 12 * T, 0 * T, T // 3, T // 2], axis=1)
        try:
            allst = gather_system_stats(stats, lo, count, world)
            q.put((rank, allst.tolist()))
        except Exception as exc:  # noqa: BLE001
            q.put((rank, f"error: {type(exc).__name__}"))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:  # noqa: BLE001
            pass


def _run(mode, count=1024, world=2):
    ctx = torch.multiprocessing.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, count, mode, q)) for r in range(world)]
    for p in ps:
        p.start()
    out = dict(q.get(timeout=120) for _ in range(world))
    for p in ps:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return out


def test_shard_tiles():
    from opt_solver_b200.batch import shard
    for world in (1, 2, 3, 8):
        cuts = [shard(1024, r, world) for r in range(world)]
        assert cuts[0][0] == 0 and cuts[-1][1] == 1024
        assert all(a[1] == b[0] for a, b in zip(cuts, cuts[1:]))


def test_two_ranks_gather_in_order():
    out = _run("ok")
    T = np.arange(1024) % 191 + 10
    want = np.stack([16 * T + 12, 12 * T, 0 * T, T // 3, T // 2], axis=1)
    for r in (0, 1):
        assert np.array_equal(np.asarray(out[r]), want)


def test_rank_leaving_is_an_error_not_a_hang():
    out = _run("drop")
    assert out[1] == "left"
    assert isinstance(out[0], str) and out[0].startswith("error")
