"""Impact ionisation (models bit 8, Chynoweth law with the van Overstraeten - de Man
coefficients of silicon) against the reference core run live: a Si p+n diode (1e19 / 1e17
cm^-3, tau 1 ns so the generation-recombination leakage is far above the round-off floor)
swept in reverse to -11 V, where avalanche multiplication doubles the leakage.

Converged tightly (inner solves to round-off, Gummel tolerance 1e-12 V) psi agrees within
1e-6 V, the generation map (bulk_copy 33) within 1e-4 of its peak and the currents within
1e-4 relative (or the floor): the Gummel loop iterates the multiplication only until the
total generation changes by less than tol_ii = max(tol_c, 1e-4) of itself
(semiconductor_3d.c:3788-3831), so that is the resolution of an avalanche current in both
codes (measured: <= 6e-5).  At the production tolerances the reverse leakage - a generation
current carried by minority carriers - is converged only to ~1e-3 in either code (measured
with and without avalanche: up to 6e-4 apart), so a current may differ by 1e-3 relative or
the reference's own distance to its converged value."""
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

DIODE = dict(n=(40, 3, 3), NA=1e19, ND=1e17, xj=0.3e-6, mobility=None, tau=1e-9, vmax=-11.0, dv=-1.0)


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


def run(L, models, tight, monkeypatch):
    for k, v in MG.TIGHT_ENV.items():
        if tight:
            monkeypatch.setenv(k, v)
        else:
            monkeypatch.delenv(k, raising=False)
    kw = dict(DIODE, models=models)
    if tight:
        kw["solver"] = MG.TIGHT_SOLVER
    w = D.pn_diode(L, **kw)
    s = w.sweeps[0]
    ok0 = D.start_sweep(L, w, s)
    V, I, F, conv = D.run_sweep(L, w, s)
    return ok0, I[:, 0], F[:, 0], conv, D.field(L, 0, w.shape).ravel(), D.field(L, 33, w.shape).ravel()


@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "refined"])
def test_avalanche_multiplication_matches_reference(lib, prec, monkeypatch):
    ref = reference_lib()
    old = lib.api3b_set_precision(prec)
    try:
        g1 = run(lib, 7 | 256, 1, monkeypatch)
        g0 = run(lib, 7 | 256, 0, monkeypatch)
        plain = run(lib, 7, 1, monkeypatch)
    finally:
        lib.api3b_set_precision(old)
    r1 = run(ref, 7 | 256, 1, monkeypatch)
    r0 = run(ref, 7 | 256, 0, monkeypatch)
    for o in (g1, g0, r1, r0, plain):
        assert o[0] and o[3].all()
    # multiplication is real: the last point carries about twice the leakage without it
    assert abs(g1[1][-1]) > 1.5 * abs(plain[1][-1])
    tol = np.maximum(1e-4 * np.abs(r1[1]), r1[2])
    assert (np.abs(g1[1] - r1[1]) <= tol).all(), f"tight currents\n{g1[1]}\n{r1[1]}"
    assert np.abs(g1[4] - r1[4]).max() <= 1e-6
    assert np.abs(g1[5] - r1[5]).max() <= 1e-4 * np.abs(r1[5]).max()
    own = 2.0 * np.abs(r0[1] - r1[1])
    tol0 = np.maximum(np.maximum(1e-3 * np.abs(r0[1]), r0[2]), own)
    assert (np.abs(g0[1] - r0[1]) <= tol0).all(), f"default currents\n{g0[1]}\n{r0[1]}"
    assert np.abs(g0[4] - r0[4]).max() <= 1e-6
