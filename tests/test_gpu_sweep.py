"""End-to-end parity of the GPU solve path with the reference core: whole bias sweeps
through the api3_* ABI (api3_solve, then api3_resolve per point), compared with the
reference's own sweeps.

Tolerances (the targets of the workload definition): psi within 1e-6 V; n and p within
1e-6 relative where above 1e3 cm^-3 (1e9 m^-3); terminal currents within 1e-4 relative,
or within the reference's own round-off floor Iflr where the current is below it.
"""
import ctypes
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_golden as MG  # noqa: E402
import semiconductor_devices_simulator_b200 as S  # noqa: E402
from semiconductor_devices_simulator_b200 import abi, devices as D  # noqa: E402

pytestmark = pytest.mark.gpu
NAMES = ["diode_small", "mos_small", "moscap_small"]
PSI_TOL = 1e-6
NP_RTOL, NP_FLOOR = 1e-6, 1e9
I_RTOL = 1e-4


def golden(name):
    z = np.load(os.path.join(HERE, "golden", name + ".npz"))
    return {k: z[k] for k in z.files}


@pytest.fixture(scope="module")
def lib():
    return S.load()


def sweep_fields(lib, w, s):
    ok0 = D.start_sweep(lib, w, s)
    psi, nn, pp = [], [], []

    def grab(q, v):
        psi.append(D.field(lib, 0, w.shape).ravel())
        nn.append(D.field(lib, 1, w.shape).ravel())
        pp.append(D.field(lib, 2, w.shape).ravel())
    V, I, F, conv = D.run_sweep(lib, w, s, on_point=grab)
    return ok0, V, I, F, conv, np.array(psi), np.array(nn), np.array(pp)


def check_fields(psi, n, p, rpsi, rn, rp, kind):
    semi = kind == 0
    dpsi = np.abs(psi - rpsi).max()
    assert dpsi <= PSI_TOL, f"psi differs by {dpsi:.3e} V"
    for a, b, lab in ((n, rn, "n"), (p, rp, "p")):
        m = (b > NP_FLOOR) & semi[None, :]
        rel = np.abs(a[m] - b[m]) / b[m]
        assert rel.max() <= NP_RTOL, f"{lab} differs by {rel.max():.3e} relative"


def check_currents(I, rI, rF):
    tol = np.maximum(I_RTOL * np.abs(rI), rF)
    err = np.abs(I - rI)
    bad = err > tol
    assert not bad.any(), f"currents differ: worst {err[bad].max():.3e} vs tol {tol[bad].min():.3e}\n{I}\n{rI}"


@pytest.mark.parametrize("name", NAMES)
def test_small_sweeps_match_reference(lib, name):
    g = golden(name)
    w, mat, bias = MG.build(lib, name)
    s = w.sweeps[0]
    ok0, V, I, F, conv, psi, n, p = sweep_fields(lib, w, s)
    assert ok0 and conv.all()
    np.testing.assert_allclose(V, g["sw0_V"])
    check_currents(I, g["sw0_I"], g["sw0_Iflr"])
    check_fields(psi, n, p, g["sw0_psi"], g["sw0_n"], g["sw0_p"], g["kind"])


def reference_lib():
    path = os.path.join(ROOT, "oracle", "_ref", "libsemisim_harness.so")
    if not os.path.exists(path):
        pytest.skip("reference core not built (make -C oracle)")
    return abi.bind(ctypes.CDLL(path))


def test_pn_diode_40cubed_matches_reference(lib):
    """The 40^3 Si pn diode sweep 0..0.6 V (13 points) on both libraries."""
    ref = reference_lib()
    ref.api3_set_threads(os.cpu_count() or 1)
    out = {}
    for tag, L in (("gpu", lib), ("ref", ref)):
        w = D.pn_diode(L)
        out[tag] = sweep_fields(L, w, w.sweeps[0])
    ok0, V, I, F, conv, psi, n, p = out["gpu"]
    rok0, rV, rI, rF, rconv, rpsi, rn, rp = out["ref"]
    assert ok0 and conv.all() and rconv.all()
    check_currents(I, rI, rF)
    check_fields(psi, n, p, rpsi, rn, rp, np.zeros(psi.shape[1], int))     # all nodes silicon
