"""The large-device configuration's device - the vertical power cell (devices.power_cell:
n- drift 1e15 cm^-3 over an n+ substrate, Gaussian-diffused p-body wells, n+ sources, p+
taps, two 50 nm oxide gates at Vg = 10 V) - on a reduced 40x64x3 mesh, where the reference
core converges every drain step, against the reference's golden sweeps
(tests/golden/power_cell_small.npz, tests/golden/make_power_cell.py): the drain swept
0..50 V in 5 V steps.

* Both codes converged tightly, FP64 and refined: every terminal current within 1e-4
  relative or the reference's round-off floor, psi within 1e-6 V on every node.
* The production tolerances, FP64 and refined: every current within 1e-4, the floor, or
  twice the reference's own distance to its converged value.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
sys.path.insert(0, HERE)

import make_golden as MG  # noqa: E402
import make_power_cell as PC  # noqa: E402
import semiconductor_devices_simulator_b200 as S  # noqa: E402
from test_gpu_sweep import check_currents, PSI_TOL  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    return S.load()


@pytest.fixture(scope="module")
def gold():
    z = np.load(os.path.join(HERE, "golden", "power_cell_small.npz"))
    return {k: z[k] for k in z.files}


@pytest.fixture(params=[0, 1], ids=["fp64", "refined"])
def prec(lib, request):
    old = lib.api3b_set_precision(request.param)
    yield request.param
    lib.api3b_set_precision(old)


def test_power_cell_tight_matches_reference(lib, gold, prec, monkeypatch):
    for k, v in MG.TIGHT_ENV.items():
        monkeypatch.setenv(k, v)                  # read by api3_init, as the reference reads them
    w = PC.build(lib, MG.TIGHT_SOLVER)
    assert lib.api3b_get_precision() == prec
    r = PC.sweep(lib, w, "g")
    assert r["g_start_ok"] and r["g_conv"].all()
    np.testing.assert_allclose(r["g_V"], gold["swt_V"])
    check_currents(r["g_I"], gold["swt_I"], gold["swt_Iflr"])
    assert np.abs(r["g_psi"] - gold["swt_psi"]).max() <= PSI_TOL


def test_power_cell_default_matches_reference(lib, gold, prec):
    w = PC.build(lib)
    assert lib.api3b_get_precision() == prec
    r = PC.sweep(lib, w, "g")
    assert r["g_start_ok"] and r["g_conv"].all()
    own = 2.0 * np.abs(gold["sw_I"] - gold["swt_I"])
    check_currents(r["g_I"], gold["sw_I"], np.maximum(gold["sw_Iflr"], own))
