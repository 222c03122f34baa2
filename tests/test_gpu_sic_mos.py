"""4H-SiC MOSFET channel physics against the reference core run live: Lombardi surface
mobility with the Coulomb term of the interface charge (models bit 4 with 4H-SiC), the
interface charge being the gate oxide's fixed charge (1e12 cm^-2) plus the charged states
of acceptor traps on the surface nodes; without and with incomplete ionisation (bit 9).
The small n-MOSFET geometry in 4H-SiC with a 20 nm oxide, gate swept 0..6 V at Vd = 0.5 V.

Converged tightly: drain current within 1e-6 relative or the floor, psi within 1e-6 V, the
interface-charge and trapped-charge maps (bulk_copy 34, 31) within 1e-9 of their peaks, the
display electron mobility (bulk_copy 10) within 1e-6: through the Coulomb term it depends on
the channel electron density, which the tight solve converges to that level (measured
2e-7)."""
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
from semiconductor_devices_simulator_b200.abi import dptr, iptr  # noqa: E402

pytestmark = pytest.mark.gpu


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


def run(L, models, monkeypatch):
    for k, v in MG.TIGHT_ENV.items():
        monkeypatch.setenv(k, v)
    n = (16, 12, 6)
    w = D.nmosfet(L, n=n, models=models, vds=(0.5,), vg_max=6.0, dvg=1.5, material=D.SIC, Nox=1e16,
                  tox=20e-9, solver=MG.TIGHT_SOLVER)
    k = np.arange(w.N)
    surf = np.ascontiguousarray(k[(k // n[0]) % n[1] == 0], np.int32)          # the y = 0 gate surface
    sid = L.api3_trap_species(-1, 0, 0.2, 1e-19, 1e-19)                        # acceptor 0.2 eV below Ec
    assert L.api3_trap_add(sid, len(surf), iptr(surf), dptr(np.full(len(surf), 1e24))) == 1
    s = w.sweeps[0]
    ok0 = D.start_sweep(L, w, s)
    V, I, F, conv = D.run_sweep(L, w, s)
    d = w.contacts["drain"]
    return (ok0, I[:, d], F[:, d], conv, D.field(L, 0, w.shape).ravel(), D.field(L, 34, w.shape).ravel(),
            D.field(L, 10, w.shape).ravel(), D.field(L, 31, w.shape).ravel())


@pytest.mark.parametrize("models", [7 | 16, 7 | 16 | 512], ids=["coulomb", "coulomb_incomplete"])
@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "refined"])
def test_sic_channel_matches_reference(lib, prec, models, monkeypatch):
    ref = reference_lib()
    old = lib.api3b_set_precision(prec)
    try:
        g = run(lib, models, monkeypatch)
    finally:
        lib.api3b_set_precision(old)
    r = run(ref, models, monkeypatch)
    assert g[0] and r[0] and g[3].all() and r[3].all()
    assert np.nanmax(r[5]) > 1e16                      # fixed plus trapped interface charge
    tol = np.maximum(1e-6 * np.abs(r[1]), r[2])
    assert (np.abs(g[1] - r[1]) <= tol).all(), f"currents\n{g[1]}\n{r[1]}"
    assert np.abs(g[4] - r[4]).max() <= 1e-6
    for q, rt in ((5, 1e-9), (6, 1e-6), (7, 1e-9)):
        a, b = g[q], r[q]
        assert np.array_equal(np.isnan(a), np.isnan(b))
        m = ~np.isnan(b)
        assert np.abs(a[m] - b[m]).max() <= rt * np.abs(b[m]).max(), f"map {q}"
