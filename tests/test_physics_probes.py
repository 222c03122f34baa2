"""The host-side physics probes of the ABI (validate.py's checks of the tunnelling kernel,
MLDA, Lombardi and the Coulomb term) against the reference core, on the CPU: the same
material table set up through both libraries, the same arguments, the results equal to
1e-12 relative (the Tsu-Esaki integral to 1e-10).

api3_tun_eval (semiconductor_3d.c:4855-4868), api3_mlda_factor (:4869-4872),
api3_lombardi (:4894-4897), api3_coulomb_inv (:4878-4881), api3_set_surface_mobility
(:4885-4893)."""
import ctypes
import os

import numpy as np
import pytest

import semiconductor_devices_simulator_b200 as S
from semiconductor_devices_simulator_b200 import abi
from semiconductor_devices_simulator_b200.abi import dptr, iptr

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def libs():
    path = os.path.join(ROOT, "oracle", "_ref", "libsemisim_harness.so")
    if not os.path.exists(path):
        pytest.skip("reference core not built (make -C oracle)")
    ref = abi.bind(ctypes.CDLL(path))
    return S.load(), ref


def materials(L):
    """Si, SiO2, HfO2, 4H-SiC, GaN, GaAs at 300 K (material indices 0..5)."""
    L.api3_init()
    xs = np.linspace(0, 1e-7, 4)
    L.api3_set_grid_coords(4, 4, 4, dptr(xs), dptr(xs), dptr(xs))
    return [L.api3_add_material(i, 300.0) for i in (0, 8, 10, 4, 5, 2)]


def close(a, b, rtol):
    a, b = np.asarray(a, float), np.asarray(b, float)
    assert np.array_equal(np.isnan(a), np.isnan(b))
    m = ~np.isnan(b)
    err = np.abs(a[m] - b[m])
    assert np.all(err <= rtol * np.maximum(np.abs(b[m]), 1e-300)), (a, b)


def test_tunnelling_kernel_matches_reference(libs):
    out = {}
    for tag, L in zip(("gpu", "ref"), libs):
        mi = materials(L)
        res = []
        for stack in ([1], [2], [1, 2], [2, 1, 2]):
            mat = np.array([mi[q] for q in stack], np.int32)
            for tox in (1.0e-9, 1.5e-9, 2.5e-9):
                t = np.full(len(stack), tox / len(stack))
                for psi, Vg in ((0.0, 1.0), (0.3, -1.2), (0.9, 2.5), (0.5, 0.5)):
                    F = np.zeros(4)
                    J = L.api3_tun_eval(mi[0], len(stack), iptr(mat), dptr(t), psi, 0.0, 0.0, Vg, 4.1, dptr(F))
                    res.append([J, *F])
        # a semiconductor half cell first (the path form), and a rejected argument
        mat = np.array([mi[0], mi[1]], np.int32)
        t = np.array([0.5e-9, 1.2e-9])
        F = np.zeros(4)
        res.append([L.api3_tun_eval(mi[0], 2, iptr(mat), dptr(t), 0.4, 0.1, -0.1, 1.5, 0.0, dptr(F)), *F])
        res.append([L.api3_tun_eval(mi[0], 7, iptr(mat), dptr(t), 0.4, 0.1, -0.1, 1.5, 0.0, None), 0, 0, 0, 0])
        out[tag] = np.array(res)
    assert np.abs(out["ref"][:, 0]).max() > 0
    close(out["gpu"], out["ref"], 1e-10)


def test_mlda_lombardi_coulomb_match_reference(libs):
    out = {}
    for tag, L in zip(("gpu", "ref"), libs):
        mi = materials(L)
        v = []
        for m in (mi[0], mi[3], mi[4], mi[5]):
            for hole in (0, 1):
                for a, b in ((0.0, 0.5e-9), (0.2e-9, 0.3e-9), (1e-9, 3e-9), (5e-9, 5e-9), (2e-9, 1e-9)):
                    v.append(L.api3_mlda_factor(m, a, b, hole))
                for F in (1e3, 1e6, 5e7):
                    for Nt in (1e21, 1e24):
                        for Dw in (1.0, 0.3):
                            v.append(L.api3_lombardi(m, 0.1, F, Nt, Dw, hole))
            for F in (1e5, 3e7):
                for n in (1e22, 1e25):
                    v.append(L.api3_coulomb_inv(m, F, n, 1e15, 1e23))
        v.append(L.api3_mlda_factor(99, 0.0, 1e-9, 0))
        v.append(L.api3_lombardi(99, 0.07, 1e6, 1e22, 1.0, 0))
        assert L.api3_set_surface_mobility(mi[0], 2e14, 3e29, 50.0) == 1
        v.append(L.api3_lombardi(mi[0], 0.1, 1e7, 1e23, 1.0, 0))
        assert L.api3_set_surface_mobility(99, 1.0, 1.0, 1.0) == 0
        out[tag] = np.array(v)
    close(out["gpu"], out["ref"], 1e-12)
