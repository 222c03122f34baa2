"""Grid shares of the persistent solves (api3b_set_share) and what they promise.

Two instances of the 60x40x30 n-MOSFET (72,000 nodes; a persistent solve wants ~35
blocks) are swept over the gate with shares of 12 and 20 blocks, first one after the
other, then both at once from two host threads (the way bench.py drives its sweeps):

* each instance's currents are bit-for-bit the same alone and concurrently: a solve's
  reductions follow its block count, not the timing of other instances;
* the two shares' currents agree within 1e-4 relative or the reference's round-off floor
  (both converged tightly), as any two launch shapes must.
"""
import os
import sys
import threading

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
sys.path.insert(0, HERE)

import make_golden as MG  # noqa: E402
import semiconductor_devices_simulator_b200 as S  # noqa: E402
from semiconductor_devices_simulator_b200 import devices as D  # noqa: E402
from test_gpu_sweep import check_currents  # noqa: E402

pytestmark = pytest.mark.gpu


def sweep(lib, h, share, out):
    lib.api3b_use(h)
    lib.api3b_set_precision(1)
    lib.api3b_set_share(share)
    w = D.nmosfet(lib, n=(60, 40, 30), vds=(1.0,), vg_max=0.5, dvg=0.1)
    lib.api3_set_solver(*MG.TIGHT_SOLVER)
    s = w.sweeps[0]
    assert D.start_sweep(lib, w, s)
    V, I, F, conv = D.run_sweep(lib, w, s)
    out[share] = (I, F, conv)
    lib.api3b_use(0)


def test_shares_are_reproducible_under_concurrency(monkeypatch):
    lib = S.load()
    for k, v in MG.TIGHT_ENV.items():
        monkeypatch.setenv(k, v)
    old = lib.api3b_set_persist(1, -1)
    hs = [lib.api3b_new(), lib.api3b_new()]
    try:
        alone = {}
        sweep(lib, hs[0], 12, alone)
        sweep(lib, hs[1], 20, alone)
        both = {}
        th = [threading.Thread(target=sweep, args=(lib, h, sh, both)) for h, sh in zip(hs, (12, 20))]
        for t in th:
            t.start()
        for t in th:
            t.join()
        for sh in (12, 20):
            assert alone[sh][2].all() and both[sh][2].all()
            np.testing.assert_array_equal(alone[sh][0], both[sh][0])
        check_currents(alone[12][0], alone[20][0], alone[20][1])
    finally:
        lib.api3b_use(0)
        for h in hs:
            lib.api3b_free(h)
        lib.api3b_set_persist(old, -1)
