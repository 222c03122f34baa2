"""The tri-gate FinFET-like device (a Si fin wrapped by SiO2 and three metal gate electrodes
driven together, n+ source / drain, velocity-saturated mobility) against the reference core
run live on the same reduced mesh (32x32x24): Id-Vg sweeps at Vd = 0.05 and 1.0 V.

Converged tightly: psi within 1e-6 V, n and p within 1e-6 relative above 1e9 m^-3 wherever
the carrier is >= 1e-6 of the local charge scale (the fin has no body contact and is fully
depleted: its holes stay below that everywhere), every terminal current within 1e-6
relative or the reference's floor.  At the production tolerances, in both precisions: psi
within 1e-6 V and the currents within 1e-4 relative (or the floor)."""
import ctypes
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_golden as MG  # noqa: E402
import semiconductor_devices_simulator_b200 as S  # noqa: E402
from semiconductor_devices_simulator_b200 import abi, devices as D  # noqa: E402

pytestmark = pytest.mark.gpu

MESH = (32, 32, 24)


@pytest.fixture(scope="module")
def lib():
    return S.load()


def reference_lib():
    path = os.path.join(ROOT, "oracle", "_ref", "libsemisim_harness.so")
    if not os.path.exists(path):
        pytest.skip("reference core not built (make -C oracle)")
    ref = abi.bind(ctypes.CDLL(path))
    ref.api3_set_threads(os.cpu_count() or 1)
    return ref


def sweeps(L, tight):
    w = D.finfet(L, n=MESH, vds=(0.05, 1.0), dvg=0.1, solver=MG.TIGHT_SOLVER if tight else D.GUI_SOLVER)
    out = []
    for s in w.sweeps:
        ok0 = D.start_sweep(L, w, s)
        psi, nn, pp = [], [], []

        def grab(q, v):
            psi.append(D.field(L, 0, w.shape).ravel())
            nn.append(D.field(L, 1, w.shape).ravel())
            pp.append(D.field(L, 2, w.shape).ravel())
        V, I, F, conv = D.run_sweep(L, w, s, on_point=grab)
        out.append((ok0, I, F, conv, np.array(psi), np.array(nn), np.array(pp)))
    nd = np.abs(D.field(L, 14, w.shape).ravel())
    return out, nd


@pytest.mark.parametrize("tight", [1, 0], ids=["tight", "default"])
@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "refined"])
def test_finfet_sweeps_match_reference(lib, prec, tight, monkeypatch):
    for k, v in MG.TIGHT_ENV.items():
        if tight:
            monkeypatch.setenv(k, v)
        else:
            monkeypatch.delenv(k, raising=False)
    ref = reference_lib()
    old = lib.api3b_set_precision(prec)
    try:
        g, _ = sweeps(lib, tight)
    finally:
        lib.api3b_set_precision(old)
    r, nd = sweeps(ref, tight)
    for a, b in zip(g, r):
        assert a[0] and b[0] and a[3].all() and b[3].all()
        assert np.abs(a[4] - b[4]).max() <= 1e-6
        tol = np.maximum((1e-6 if tight else 1e-4) * np.abs(b[1]), b[2])
        assert (np.abs(a[1] - b[1]) <= tol).all(), f"currents\n{a[1]}\n{b[1]}"
        if tight:
            for x, y, o in ((a[5], b[5], b[6]), (a[6], b[6], b[5])):
                m = (y > 1e9) & (y >= 1e-6 * (y + o + nd))
                if m.any():                       # the fin has no body contact: its holes are trace
                    assert (np.abs(x[m] - y[m]) / y[m]).max() <= 1e-6
    # the device works as a transistor: the drain current rises by decades with the gate
    Id = np.abs(g[1][1][:, 1])
    assert Id[-1] > 100 * Id[0]
