"""The quadratic sweep predictor (api3b_set_pred_order(2)): a starting guess from the last
three sweep points' solutions instead of the reference's secant step from the last two
(semiconductor_3d.c:4018-4047).  Only the Gummel loop's start changes, so a sweep solved
with it reaches the same converged currents: checked on the small MOSFET's gate sweep,
converged tightly, against the secant-predictor sweep of this library and against the
reference core run live, every terminal within 1e-4 relative or its round-off floor.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
sys.path.insert(0, HERE)

import make_golden as MG  # noqa: E402
import semiconductor_devices_simulator_b200 as S  # noqa: E402
from test_gpu_iv_sweep import sweep2, tight_device  # noqa: E402
from test_gpu_sweep import check_currents, reference_lib  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture
def order():
    lib = S.load()
    old = lib.api3b_set_pred_order(-1)
    yield lib
    lib.api3b_set_pred_order(old)


def test_quadratic_predictor_reaches_the_same_currents(order, monkeypatch):
    lib = order
    out = {}
    for po in (1, 2):
        assert lib.api3b_set_pred_order(po) in (1, 2)
        tight_device(lib, "mos_small", monkeypatch)
        g0 = lib.api3_get_stat(3)
        V, I, F, C = sweep2(lib, 2, 0.0, 0.9, 10)          # the gate, 0.1 V steps
        out[po] = (V, I, F, C, lib.api3_get_stat(3) - g0)
    assert out[1][3].all() and out[2][3].all()
    np.testing.assert_array_equal(out[1][0], out[2][0])
    check_currents(out[2][1], out[1][1], out[1][2])
    ref = reference_lib()
    ref.api3_set_threads(os.cpu_count() or 1)
    tight_device(ref, "mos_small", monkeypatch)
    rV, rI, rF, rC = sweep2(ref, 2, 0.0, 0.9, 10)
    assert rC.all()
    check_currents(out[2][1], rI, rF)
    print(f"Gummel iterations: secant {out[1][4]}, quadratic {out[2][4]}")
