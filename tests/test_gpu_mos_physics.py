"""Nanoscale MOS physics against the reference core run live on the small n-MOSFET (oxide
Robin face gate) swept in Vg at Vd = 0.5 V:

* Lombardi surface mobility (models bit 4: acoustic-phonon and surface-roughness scattering
  near an insulator or gate wall, weighted by D = exp(-d / 10 nm));
* MLDA quantum confinement (models bit 3: the carrier densities in front of the wall fall
  off as 1 - exp(-(z/lambda)^2), applied as band corrections qcn / qcp);
* both together.

Converged tightly: drain current within 1e-6 relative (or the floor), psi within 1e-6 V,
the display mobility maps (bulk_copy 10, 11) and quantum potentials (28, 29) within 1e-9 of
their peak; at the production tolerances the current within the reference's own distance
to its converged value or 1e-4."""
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
    kw = dict(n=(16, 12, 6), models=models, vds=(0.5,), vg_max=1.0, dvg=0.25)
    if tight:
        kw["solver"] = MG.TIGHT_SOLVER
    w = D.nmosfet(L, **kw)
    s = w.sweeps[0]
    ok0 = D.start_sweep(L, w, s)
    V, I, F, conv = D.run_sweep(L, w, s)
    d = w.contacts["drain"]
    return (ok0, I[:, d], F[:, d], conv, D.field(L, 0, w.shape).ravel(),
            D.field(L, 10, w.shape).ravel(), D.field(L, 11, w.shape).ravel(),
            D.field(L, 28, w.shape).ravel(), D.field(L, 29, w.shape).ravel())


@pytest.mark.parametrize("models", [7 | 16, 7 | 8, 7 | 8 | 16], ids=["lombardi", "mlda", "mlda_lombardi"])
@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "refined"])
def test_mos_physics_matches_reference(lib, prec, models, monkeypatch):
    ref = reference_lib()
    old = lib.api3b_set_precision(prec)
    try:
        g1 = run(lib, models, 1, monkeypatch)
        g0 = run(lib, models, 0, monkeypatch)
        plain = run(lib, 7, 1, monkeypatch)
    finally:
        lib.api3b_set_precision(old)
    r1 = run(ref, models, 1, monkeypatch)
    r0 = run(ref, models, 0, monkeypatch)
    for o in (g1, g0, r1, r0, plain):
        assert o[0] and o[3].all()
    # surface scattering and confinement both lower the on-state drain current
    assert abs(g1[1][-1]) < 0.97 * abs(plain[1][-1])
    tol = np.maximum(1e-6 * np.abs(r1[1]), r1[2])
    assert (np.abs(g1[1] - r1[1]) <= tol).all(), f"tight currents\n{g1[1]}\n{r1[1]}"
    assert np.abs(g1[4] - r1[4]).max() <= 1e-6
    for q in (5, 6, 7, 8):
        a, b = g1[q], r1[q]
        assert np.array_equal(np.isnan(a), np.isnan(b))
        m = ~np.isnan(b)
        assert np.abs(a[m] - b[m]).max() <= 1e-9 * max(np.abs(b[m]).max(), 1e-300), f"display map {q}"
    if models & 8:
        assert np.nanmax(np.abs(g1[7])) > 1e-3                  # a quantum potential of meV and more
    own = 2.0 * np.abs(r0[1] - r1[1])
    tol0 = np.maximum(np.maximum(1e-4 * np.abs(r0[1]), r0[2]), own)
    assert (np.abs(g0[1] - r0[1]) <= tol0).all(), f"default currents\n{g0[1]}\n{r0[1]}"
