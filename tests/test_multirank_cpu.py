"""The multi-GPU plumbing of bench.py on CPU: two ranks over gloo (the backend bench.py
picks without CUDA), the max-over-ranks and sum reductions that make its JSON line, the
barrier, and the work split (the Id-Vg workload replicated on every rank; the 64 diode
variants split so every variant is solved exactly once).  No GPU and no solver calls."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
    sys.path.insert(0, ROOT)
    import bench
    d = bench.Dist()
    mx = d.max(1.5 + rank)
    sm = d.sum(10 * (rank + 1))
    d.barrier()
    q.put((rank, d.backend, mx, sm, bench.shard(list(range(64)), d.rank, d.world), bench.sweep_order(2, d.rank)))
    d.close()


@pytest.mark.parametrize("world", [2])
def test_two_ranks_gloo(world):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    assert all(o[1] == "gloo" for o in out)
    assert all(o[2] == 1.5 + world - 1 for o in out)              # max over ranks
    assert all(o[3] == sum(10 * (r + 1) for r in range(world)) for o in out)
    units = [u for o in out for u in o[4]]
    assert sorted(units) == list(range(64))                        # every variant exactly once
    assert all(sorted(o[5]) == [0, 1] for o in out)                # both sweeps on every rank
    assert out[0][5] != out[1][5]                                  # rotated start


def test_shard_uneven():
    import bench
    parts = [bench.shard(range(10), r, 3) for r in range(3)]
    assert sorted(sum(parts, [])) == list(range(10))
    assert [len(p) for p in parts] == [4, 3, 3]
