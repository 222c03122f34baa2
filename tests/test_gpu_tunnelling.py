"""Gate tunnelling (models bit 5: Tsu-Esaki current with WKB transmission through the gate
stack, supply from the contact theorem) against the reference core run live:

* an n-Si MOS capacitor with a 1.5 nm SiO2 layer meshed at 0.5 nm under a metal gate
  electrode (paths through the insulator nodes to the Dirichlet gate), gate swept into
  accumulation: direct tunnelling of the accumulated electrons, 1e-11..1e-9 A (in inversion
  the reference's own solve of such a capacitor, whose minority carriers come only from
  generation, does not converge);
* the small n-MOSFET with a 1.2 nm SiO2 layer stack on its oxide Robin face gate
  (api3_set_gate_stack: one path per gate node).

Converged tightly: psi within 1e-6 V, every terminal current (the gate's is the tunnelling
current) within 1e-6 relative or the reference's floor; the number of paths equal; the
display map of the gate current density (bulk_copy 27) within 1e-9 of its peak."""
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


def moscap_thin(L, models):
    """n-Si (3e17 cm^-3) 40 nm deep under 1.5 nm of SiO2, metal gate (work function 4.1 eV)
    on the oxide, ohmic back contact; gate swept 0..1.6 V."""
    L.api3_init()
    ysi = D.graded_axis(40e-9, 24, 0.3e-9)[::-1]
    ysi = 40e-9 - ysi
    yox = 40e-9 + np.array([0.5e-9, 1.0e-9, 1.5e-9])
    ys = np.concatenate([ysi, yox])
    xs = np.linspace(0, 20e-9, 3)
    zs = np.linspace(0, 20e-9, 3)
    D._grid(L, xs, ys, zs)
    L.api3_set_solver(*MG.TIGHT_SOLVER)
    L.api3_set_models(models)
    si = L.api3_add_material(D.SI, 300.0)
    ox = L.api3_add_material(D.SIO2, 300.0)
    ny = len(ys)
    L.api3_set_region(0, 0, 0, 2, ny - 1, 2, si, 3e23, 0.0)
    L.api3_set_region(0, ny - 3, 0, 2, ny - 1, 2, ox, 0.0, 0.0)
    L.api3_clear_contacts()
    cb = L.api3_add_contact_ex(2, 0, 2, 0, 2, 0, 0, 0, 0.0, 0.0, 0.0, 0.0)
    cg = L.api3_add_contact_ex(3, 0, 2, 0, 2, 0, 0, 2, 0.0, 4.1, 0.0, 0.0)
    V = np.round(np.linspace(0.0, 1.6, 9), 12)
    return D.Workload("moscap_thin", (3, ny, 3), {"back": cb, "gate": cg},
                      [{"fixed": {"back": 0.0}, "swept": "gate", "V": V}])


def mosfet_stack(L, models):
    w = D.nmosfet(L, n=(16, 12, 6), models=models, vds=(0.5,), vg_max=1.0, dvg=0.25, solver=MG.TIGHT_SOLVER)
    ox = L.api3_add_material(D.SIO2, 300.0)
    mat = np.array([ox], np.int32)
    assert L.api3_set_gate_stack(w.contacts["gate"], 1, iptr(mat), dptr(np.array([1.2e-9]))) == 1
    return w


def run(L, build, models, monkeypatch):
    for k, v in MG.TIGHT_ENV.items():
        monkeypatch.setenv(k, v)
    w = build(L, models)
    s = w.sweeps[0]
    ok0 = D.start_sweep(L, w, s)
    V, I, F, conv = D.run_sweep(L, w, s)
    return ok0, I, F, conv, D.field(L, 0, w.shape).ravel(), D.field(L, 27, w.shape).ravel(), L.api3_get_ntp(-1), w


@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "refined"])
@pytest.mark.parametrize("device", ["moscap", "mosfet"])
def test_gate_tunnelling_matches_reference(lib, device, prec, monkeypatch):
    build = moscap_thin if device == "moscap" else mosfet_stack
    models = (1 | 32) if device == "moscap" else (7 | 32)
    ref = reference_lib()
    old = lib.api3b_set_precision(prec)
    try:
        g = run(lib, build, models, monkeypatch)
    finally:
        lib.api3b_set_precision(old)
    r = run(ref, build, models, monkeypatch)
    assert g[0] and r[0] and g[3].all() and r[3].all()
    assert g[6] == r[6] and g[6] > 0, (g[6], r[6])
    gate = g[7].contacts["gate"]
    assert np.abs(r[1][-1, gate]) > 1e3 * r[2][-1, gate]            # a real tunnelling current
    tol = np.maximum(1e-6 * np.abs(r[1]), r[2])
    assert (np.abs(g[1] - r[1]) <= tol).all(), f"currents\n{g[1]}\n{r[1]}"
    assert np.abs(g[4] - r[4]).max() <= 1e-6
    assert np.abs(g[5] - r[5]).max() <= 1e-9 * np.abs(r[5]).max()
