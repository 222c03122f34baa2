"""Deep-level traps (api3_trap_species / api3_trap_add, Shockley-Read-Hall occupancy with
the trapped charge in Poisson) against the reference core run live: the small Si pn diode
with a mid-gap acceptor level (1e16 cm^-3) over its n side and a donor level 0.3 eV below
Ec (3e16 cm^-3) over its p side, two requests of the acceptor on one node (merged), swept
forward 0..0.6 V, where trap-assisted recombination dominates the current.

Converged tightly: currents within 1e-6 relative or the reference's floor, psi within
1e-6 V, the trapped-charge and trap-density maps (bulk_copy 31, 32) within 1e-9 of their
peaks, the number of compiled trap entries equal."""
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


def trapped_diode(L):
    n = (12, 6, 5)
    w = D.pn_diode(L, n=n, solver=MG.TIGHT_SOLVER, models=3)
    k = np.arange(w.N)
    i = k % n[0]
    sa = L.api3_trap_species(-1, 2, 0.0, 1e-19, 1e-19)          # mid-gap acceptor
    sd = L.api3_trap_species(1, 0, 0.3, 2e-20, 5e-20)           # donor 0.3 eV below Ec
    assert sa >= 0 and sd >= 0 and L.api3_trap_species(-1, 2, 0.0, 1e-19, 1e-19) == sa
    nn = np.ascontiguousarray(k[i >= n[0] // 2], np.int32)
    pp = np.ascontiguousarray(k[i < n[0] // 2], np.int32)
    assert L.api3_trap_add(sa, len(nn), iptr(nn), dptr(np.full(len(nn), 0.6e22))) == 1
    assert L.api3_trap_add(sa, len(nn), iptr(nn), dptr(np.full(len(nn), 0.4e22))) == 1   # merged
    assert L.api3_trap_add(sd, len(pp), iptr(pp), dptr(np.full(len(pp), 3e22))) == 1
    return w


def run(L, monkeypatch):
    for k, v in MG.TIGHT_ENV.items():
        monkeypatch.setenv(k, v)
    w = trapped_diode(L)
    s = w.sweeps[0]
    ok0 = D.start_sweep(L, w, s)
    V, I, F, conv = D.run_sweep(L, w, s)
    return (ok0, I, F, conv, D.field(L, 0, w.shape).ravel(), D.field(L, 31, w.shape).ravel(),
            D.field(L, 32, w.shape).ravel(), L.api3_n_trap_entries())


@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "refined"])
def test_traps_match_reference(lib, prec, monkeypatch):
    ref = reference_lib()
    old = lib.api3b_set_precision(prec)
    try:
        g = run(lib, monkeypatch)
    finally:
        lib.api3b_set_precision(old)
    r = run(ref, monkeypatch)
    assert g[0] and r[0] and g[3].all() and r[3].all()
    assert g[7] == r[7] and g[7] > 0
    tol = np.maximum(1e-6 * np.abs(r[1]), r[2])
    assert (np.abs(g[1] - r[1]) <= tol).all(), f"currents\n{g[1]}\n{r[1]}"
    assert np.abs(g[4] - r[4]).max() <= 1e-6
    for q in (5, 6):
        a, b = g[q], r[q]
        assert np.array_equal(np.isnan(a), np.isnan(b))
        m = ~np.isnan(b)
        assert np.abs(a[m] - b[m]).max() <= 1e-9 * np.abs(b[m]).max(), f"map {q}"
    assert np.nanmax(np.abs(r[5])) > 0
