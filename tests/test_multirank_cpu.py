"""The multi-GPU plumbing of bench.py on CPU: two ranks over gloo (the backend bench.py
picks without CUDA), the max-over-ranks and sum reductions that make its JSON line, the
barrier, the work split and the gather of the I-V arrays to rank 0.

Work split: the n-MOSFET family is replicated on every rank (independent jobs, weak
scaling); the FinFET's five drain-bias sweeps and the 64 diode variants are split so that
every unit is solved exactly once, balanced by node count (largest first, each to the least
loaded rank).  The gather is checked with synthetic per-rank current arrays: shape, order
and completeness of the family array rank 0 assembles.  No GPU and no solver calls; the
path is unmeasured on GPU hardware here (one GPU per run on this machine pool)."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _synthetic_currents(si, npts=24, nc=4):
    """What a rank's sweep `si` yields: per point (I per contact, Iflr per contact)."""
    return [([si * 1000.0 + q * 10.0 + c for c in range(nc)], [1e-18 * (c + 1) for c in range(nc)])
            for q in range(npts)]


def _rank_main(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
    sys.path.insert(0, ROOT)
    import bench
    from semiconductor_devices_simulator_b200 import devices as D
    d = bench.Dist()
    mx = d.max(1.5 + rank)
    sm = d.sum(10 * (rank + 1))
    d.barrier()
    var = D.diode_variants(64)
    nodes = [int(np.prod(v["n"])) for v in var]
    mine = bench.shard(list(range(64)), d.rank, d.world, weights=nodes)
    fin = bench.sweep_order(5, d.rank, d.world, replicate=False)
    mos = bench.sweep_order(2, d.rank, d.world, replicate=True)
    cur = {si: _synthetic_currents(si) for si in fin}
    iv = bench.gather_iv(d, cur, 5)
    q.put((rank, d.backend, mx, sm, mine, sum(nodes[i] for i in mine), fin, mos, iv))
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
    out.sort(key=lambda o: o[0])
    assert all(o[1] == "gloo" for o in out)
    assert all(o[2] == 1.5 + world - 1 for o in out)              # max over ranks
    assert all(o[3] == sum(10 * (r + 1) for r in range(world)) for o in out)
    # 64 diode variants: every one exactly once, node counts balanced within one variant
    units = [u for o in out for u in o[4]]
    assert sorted(units) == list(range(64))
    loads = [o[5] for o in out]
    assert max(loads) - min(loads) <= 72 ** 3
    # FinFET drain biases: split, every sweep once; n-MOSFET: both sweeps on every rank
    assert sorted(s for o in out for s in o[6]) == [0, 1, 2, 3, 4]
    assert all(sorted(o[7]) == [0, 1] for o in out)
    assert out[0][7] != out[1][7]                                  # rotated start
    # the gather: rank 0 holds the whole family (sweeps x points x contacts x 2) in sweep
    # order, every sweep solved once; the other ranks hold nothing
    arr, seen = out[0][8]
    assert out[1][8] is None
    assert arr.shape == (5, 24, 4, 2)
    assert seen == [1, 1, 1, 1, 1]
    for si in range(5):
        ref = np.asarray(_synthetic_currents(si), dtype=np.float64).transpose(0, 2, 1)
        assert np.array_equal(arr[si], ref)


def test_shard_uneven():
    import bench
    parts = [bench.shard(range(10), r, 3) for r in range(3)]
    assert sorted(sum(parts, [])) == list(range(10))
    assert sorted(len(p) for p in parts) == [3, 3, 4]


def test_shard_balances_node_counts():
    """Largest first to the least loaded rank: on weights 8, 7, 6, 5, 4 over two ranks the
    loads are 17 and 13 (a round robin in index order gives 18 and 12)."""
    import bench
    w = [8, 7, 6, 5, 4]
    parts = [bench.shard(range(5), r, 2, weights=w) for r in range(2)]
    assert sorted(sum(parts, [])) == list(range(5))
    assert sorted(sum(w[i] for i in p) for p in parts) == [13, 17]


def test_grid_shares_follow_gummel_iterations():
    """bench.balance_shares splits the SMs between concurrent sweeps in proportion to their
    Gummel iterations, never below a floor and never above the SM count in total, and
    clears the shares when switched off (a fake library records the calls)."""
    import bench

    class Lib:
        def __init__(self):
            self.cur, self.share = 0, {}

        def api3b_use(self, h):
            self.cur = h

        def api3b_set_share(self, b):
            self.share[self.cur] = b

    class W:
        def __init__(self, h, g):
            self.h, self.gummel = h, g
    lib = Lib()
    ws = [W(1, 129), W(2, 303)]
    sh = bench.balance_shares(lib, ws, 148)
    assert sh == [44, 103] and lib.share == {1: 44, 2: 103}
    ws5 = [W(q + 1, g) for q, g in enumerate([1, 1, 1, 1, 1000])]
    sh5 = bench.balance_shares(lib, ws5, 148)
    assert sum(sh5) <= 148 and min(sh5) >= 148 // 20 and sh5[4] == max(sh5)
    assert bench.balance_shares(lib, ws, 148, on=False) == [0, 0] and lib.share[1] == 0 and lib.share[2] == 0
    assert bench.balance_shares(lib, ws[:1], 148) == [0]


def test_worst_terminal_and_band():
    """bench.worst_terminal names the terminal with the largest relative distance among those
    above their floor, and measures every terminal in units of 1e-4 |I_ref| + Iflr."""
    import bench
    ref = {0: [([1e-6, 2e-14, 5e-20], [1e-15, 2.5e-15, 1e-15])]}
    cur = {0: [([1e-6 * (1 + 2e-5), 2e-14 + 8e-18, 7e-20], None)]}
    w, band = bench.worst_terminal(cur, ref)
    assert (w["sweep"], w["point"], w["contact"]) == (0, 0, 1)       # the 5e-20 A terminal is below its floor
    assert abs(w["rel"] - 4e-4) < 1e-12
    assert abs(band - max(2e-11 / (1e-10 + 1e-15), 8e-18 / (2e-18 + 2.5e-15))) < 1e-9
    assert bench.rel_dI(cur[0], ref[0]) == w["rel"]
    assert abs(bench.rel_dI(cur[0], ref[0], on=1e-9) - 2e-5) < 1e-15
