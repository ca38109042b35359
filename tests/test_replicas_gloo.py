"""Replica plumbing across ranks on CPU: two gloo processes, no GPU.

Covers what bench.py and multi-GPU candidate sweeps rely on: the maximum of
per-rank times, barriers, the candidate split (disjoint, covering) and the
gather of per-candidate results; and the failure path -- a rank that dies
between steps makes the survivor's next collective fail within the process
group's timeout instead of hanging.
"""
import importlib
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, mode, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    try:
        R = importlib.import_module("3d_fdtd_b200.replicas")
        r = R.Ranks("gloo", timeout_s=15)
        if mode == "plumbing":
            m = r.max(1.5 + rank)
            r.barrier()
            mine = r.shard(10)
            allres = r.gather_shards(10, {i: i * i for i in mine})
            q.put((rank, "ok", m, mine, allres))
            r.close()
        elif mode == "dead_rank":
            r.barrier()               # both ranks joined and finished a step
            if rank == 1:
                os._exit(3)           # leaves between steps, nothing in flight
            try:
                r.max(1.0)
                q.put((rank, "no error"))
            except Exception as e:    # noqa: BLE001 -- any collective error is the signal
                q.put((rank, "error", type(e).__name__))
    except Exception as e:            # noqa: BLE001
        q.put((rank, "exception", f"{type(e).__name__}: {e}"))


def _run(mode, world=2, timeout=120):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, mode, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = []
    try:
        for p in procs:
            p.join(timeout)
        while not q.empty():
            out.append(q.get(timeout=5))
    finally:
        for p in procs:
            if p.is_alive():
                p.kill()
                p.join(10)
    return sorted(out, key=lambda x: x[0]), [p.exitcode for p in procs]


def test_replica_plumbing_two_ranks():
    out, codes = _run("plumbing")
    assert codes == [0, 0], out
    assert [o[1] for o in out] == ["ok", "ok"], out
    for rank, _, m, mine, allres in out:
        assert m == 2.5                                   # max over ranks
        assert mine == list(range(rank, 10, 2))           # rank's candidates
        assert allres == [i * i for i in range(10)]       # every candidate, in order


def test_dead_rank_fails_collective_not_hang():
    out, codes = _run("dead_rank")
    assert codes[1] == 3
    assert len(out) == 1 and out[0][0] == 0, out
    assert out[0][1] == "error", out


def test_single_process_is_a_world_of_one(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    sys.path.insert(0, ROOT)
    R = importlib.import_module("3d_fdtd_b200.replicas")
    r = R.Ranks("gloo")
    assert (r.rank, r.world) == (0, 1)
    assert r.max(3.25) == 3.25
    assert r.shard(3) == [0, 1, 2]
    assert r.gather_shards(2, {0: "a", 1: "b"}) == ["a", "b"]
    with pytest.raises(RuntimeError):
        r.gather_shards(3, {0: "a"})
    r.barrier()
    r.close()
