"""The ABI's C-side sweeps, api3_iv_sweep and api3_iv_sweep2 (semiconductor_3d.c:4933-4977),
against the reference core run live: the point loop inside the library (continuation per
point from the previous one, equilibrium first when there is no solution), the returned
voltages, current densities / currents and floors, the converged flags, and the
conventions - at most 400 points, at least 1, a stopped sweep marks every point NaN / -1,
the swept contact's voltage is restored afterwards.  Main.py binds both entries
(main.py:215-219).  Both codes converged tightly, so every current agrees within 1e-4
relative or the reference's round-off floor.
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
from semiconductor_devices_simulator_b200.abi import dptr, iptr  # noqa: E402
from test_gpu_sweep import reference_lib, check_currents  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def libs():
    ref = reference_lib()
    ref.api3_set_threads(os.cpu_count() or 1)
    return S.load(), ref


def tight_device(L, name, monkeypatch):
    for k, v in MG.TIGHT_ENV.items():
        monkeypatch.setenv(k, v)
    w, mat, bias = MG.build(L, name)
    L.api3_set_solver(*MG.TIGHT_SOLVER)
    return w


def sweep2(L, cid, v0, v1, n):
    nc = L.api3_get_ncon()
    m = max(1, min(n, 400))
    V = np.zeros(m); I = np.zeros((m, nc)); F = np.zeros((m, nc)); C = np.zeros(m, np.int32)
    L.api3_iv_sweep2(cid, v0, v1, n, dptr(V), dptr(I), dptr(F), iptr(C))
    return V, I, F, C


def sweep1(L, cid, v0, v1, n):
    m = max(1, min(n, 400))
    V = np.zeros(m); J = np.zeros(m); C = np.zeros(m, np.int32)
    L.api3_iv_sweep(cid, v0, v1, n, dptr(V), dptr(J), iptr(C))
    return V, J, C


@pytest.mark.parametrize("name", ["diode_small", "mos_small"])
def test_iv_sweep2_matches_reference(libs, name, monkeypatch):
    out = []
    for L in libs:
        tight_device(L, name, monkeypatch)
        cid = 0 if name == "diode_small" else 2           # the anode / the gate
        Vb = L.api3_get_contact_Vsolved(cid)
        out.append(sweep2(L, cid, 0.0, 0.6, 7) + (L.api3_get_contact_Vsolved(cid), Vb))
    (gV, gI, gF, gC, gVs, _), (rV, rI, rF, rC, rVs, _) = out
    assert gC.all() and rC.all()
    np.testing.assert_allclose(gV, rV, rtol=0, atol=1e-12)
    check_currents(gI, rI, rF)
    assert abs(gVs - rVs) <= 1e-12                         # the last point's solved voltage


@pytest.mark.parametrize("name", ["diode_small"])
def test_iv_sweep_matches_reference(libs, name, monkeypatch):
    out = []
    for L in libs:
        tight_device(L, name, monkeypatch)
        out.append(sweep1(L, 0, 0.0, 0.5, 6))
    (gV, gJ, gC), (rV, rJ, rC) = out
    assert gC.all() and rC.all()
    np.testing.assert_allclose(gV, rV, rtol=0, atol=1e-12)
    # current densities (A/m^2) of the swept contact: 1e-4 relative above the floor's density
    A = libs[1].api3_get_contact_A(0)
    floor = libs[1].api3_get_contact_Ifloor(0) / A
    assert (np.abs(gJ - rJ) <= np.maximum(1e-4 * np.abs(rJ), floor)).all(), (gJ, rJ)


def test_iv_sweep_conventions(libs, monkeypatch):
    """Stopped sweeps mark every point NaN / -1 without solving; the point count is
    clamped to 1 .. 400; the swept contact's set voltage is restored."""
    for L in libs:
        tight_device(L, "diode_small", monkeypatch)
        L.api3_set_contact_V(0, 0.123)
        L.api3_request_stop()
        try:
            V, I, F, C = sweep2(L, 0, 0.0, 0.3, 4)
            assert np.isnan(V).all() and np.isnan(I).all() and np.isnan(F).all() and (C == -1).all()
            V1, J1, C1 = sweep1(L, 0, 0.0, 0.3, 4)
            assert np.isnan(V1).all() and np.isnan(J1).all() and (C1 == -1).all()
        finally:
            L.api3_clear_stop()
        V, I, F, C = sweep2(L, 0, 0.2, 0.4, 0)            # Npts < 1 -> one point at Vs
        assert C[0] == 1 and abs(V[0] - 0.2) <= 1e-12
        # the sweep restores the contact's set voltage: a resolve now solves at 0.123 V
        assert L.api3_resolve() == 1
        assert abs(L.api3_get_contact_Vsolved(0) - 0.123) <= 1e-12
