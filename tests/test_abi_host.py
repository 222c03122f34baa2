"""Host-side checks of the solver library that need no GPU: it loads, exports every
entry point of the reference ABI (semiconductor_3d.c:4570-5353) plus the additive ones
the headers declare, records a device description, and refuses to solve without a GPU
instead of falling back to a CPU path."""
import ctypes
import os
import re

import numpy as np
import pytest

import semiconductor_devices_simulator_b200 as S
from semiconductor_devices_simulator_b200 import abi, devices as D
from semiconductor_devices_simulator_b200.abi import dptr, iptr

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    return S.load()


def exported(path):
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True).stdout
    return {ln.split()[-1] for ln in out.splitlines() if ln.strip()}


def declared():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", f)).read()
            names |= set(re.findall(r"\b(api3b?_\w+|b200x_\w+)\s*\(", txt))
    return names


def test_exports_every_reference_entry(lib):
    syms = exported(S.LIB_PATH)
    missing = set(abi.API3) - syms
    assert not missing, missing
    assert len(abi.API3) == 89


def test_exports_every_declared_entry(lib):
    syms = exported(S.LIB_PATH)
    decl = declared()
    assert decl, "no declarations found under include/"
    assert not (decl - syms), decl - syms


def test_setup_records_device_without_gpu(lib):
    w = D.nmosfet(lib, n=(16, 12, 6))
    assert lib.api3_get_Nx() == 16 and lib.api3_get_Ny() == 12 and lib.api3_get_Nz() == 6
    assert lib.api3_get_ncon() == 4
    assert abs(lib.api3_mat_ni(0) - 1.0673775147815666e16) < 1e4
    assert lib.api3_get_aa_depth() == 12
    assert lib.api3_add_material(99, 300.0) >= 0           # unknown id falls back to Si
    assert lib.api3_set_mesh_graph(0, 0, None, None, None, None, None, None) == 0
    assert np.isnan(lib.api3_get_phi(0))                     # nothing solved yet


def test_solve_without_gpu_fails_loudly(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    D.pn_diode(lib, n=(6, 4, 4))
    assert lib.api3_solve() == 0


def test_instances_are_independent(lib):
    h1 = lib.api3b_new()
    h2 = lib.api3b_new()
    assert h1 >= 1 and h2 == h1 + 1
    try:
        assert lib.api3b_use(h1) == 1
        D.pn_diode(lib, n=(6, 5, 4))
        assert lib.api3b_use(h2) == 1
        D.nmosfet(lib, n=(10, 8, 4))
        assert lib.api3b_current() == h2 and lib.api3_get_Nx() == 10
        assert lib.api3b_use(h1) == 1
        assert lib.api3_get_Nx() == 6 and lib.api3_get_ncon() == 2
        assert lib.api3b_use(0) == 1 and lib.api3b_current() == 0
        assert lib.api3b_use(9999) == 0
        # grid shares of the persistent solves belong to the instance
        lib.api3b_use(h1)
        assert lib.api3b_set_share(40) == 0
        lib.api3b_use(h2)
        assert lib.api3b_set_share(-1) == 0 and lib.api3b_set_share(100) == 0
        lib.api3b_use(h1)
        assert lib.api3b_set_share(-1) == 40 and lib.api3b_set_share(0) == 40
        assert lib.api3b_set_share(-1) == 0
        # the sweep predictor's order is library-wide: 1 secant, 2 quadratic
        old = lib.api3b_set_pred_order(2)
        assert old in (1, 2)
        assert lib.api3b_set_pred_order(0) == 2 and lib.api3b_set_pred_order(old) == 2
        assert lib.api3b_set_pred_order(-1) == old
    finally:
        lib.api3b_use(0)
        assert lib.api3b_free(h1) == 1 and lib.api3b_free(h2) == 1
        assert lib.api3b_free(h1) == 0


def test_reference_core_and_library_agree_on_setup(lib):
    """Contact areas and the material constants of both libraries after identical set-up
    (the reference core is the oracle; skipped when it has not been built)."""
    path = os.path.join(ROOT, "oracle", "_ref", "libsemisim_ref.so")
    if not os.path.exists(path):
        pytest.skip("reference core not built")
    ref = abi.bind(ctypes.CDLL(path))
    for L in (lib, ref):
        D.nmosfet(L, n=(16, 12, 6))
    for mi in range(1):
        assert lib.api3_mat_ni(mi) == ref.api3_mat_ni(mi)
        assert lib.api3_mat_Eg(mi) == ref.api3_mat_Eg(mi)


def test_mesh_graph_validation(lib):
    """api3_set_mesh_graph accepts a symmetric graph and refuses broken ones (no GPU needed);
    a tensor grid set afterwards leaves graph mode (semiconductor_3d.c:981-1041)."""
    xs = np.linspace(0, 1e-6, 4)
    rp, cj, h, ar, vol, pos = D.tensor_graph(xs, xs[:3], xs[:2], diag=0.2)
    N = len(vol)
    lib.api3_init()
    lib.api3_add_material(D.SI, 300.0)
    args = lambda rp_, cj_, h_: (N, len(cj_), iptr(rp_), iptr(cj_), dptr(h_), dptr(ar), dptr(vol), dptr(pos))
    assert lib.api3_set_mesh_graph(*args(rp, cj, h)) == 1
    assert lib.api3_is_graph() == 1 and lib.api3_get_Nx() == N and lib.api3_get_Ny() == 1
    bad = cj.copy(); bad[0] = 0                       # a self edge
    assert lib.api3_set_mesh_graph(*args(rp, bad, h)) == 0
    asym = cj.copy(); asym[0] = (cj[0] + 2) % N if (cj[0] + 2) % N != 0 else 3   # an edge without its reverse
    assert lib.api3_set_mesh_graph(*args(rp, asym, h)) == 0
    hz = h.copy(); hz[1] = 0.0
    assert lib.api3_set_mesh_graph(*args(rp, cj, hz)) == 0
    assert lib.api3_set_grid_coords(4, 3, 2, dptr(xs), dptr(xs[:3]), dptr(xs[:2])) == 1
    assert lib.api3_is_graph() == 0
