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
NAMES = ["diode_small", "mos_small", "moscap_small", "sic_small"]
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


@pytest.fixture(params=[0, 1], ids=["fp64", "refined"])
def prec(request, lib):
    """Linear-solve precision of the instance: 0 FP64 throughout, 1 FP32 inner solves
    refined in FP64 to the same stop rule."""
    old = lib.api3b_set_precision(request.param)
    yield request.param
    lib.api3b_set_precision(old)


@pytest.mark.parametrize("name", NAMES)
def test_small_sweeps_tight_match_reference(lib, name, prec, monkeypatch):
    """Both codes converged to the discrete solution (inner solves to round-off, Gummel
    tolerance 1e-12 V): every target holds on every node and terminal."""
    g = golden(name)
    for k, v in MG.TIGHT_ENV.items():
        monkeypatch.setenv(k, v)                 # read by api3_init, as the reference reads them
    w, mat, bias = MG.build(lib, name)
    assert lib.api3b_get_precision() == prec
    lib.api3_set_solver(*MG.TIGHT_SOLVER)
    s = w.sweeps[0]
    ok0, V, I, F, conv, psi, n, p = sweep_fields(lib, w, s)
    assert ok0 and conv.all()
    np.testing.assert_allclose(V, g["swt0_V"])
    check_currents(I, g["swt0_I"], g["swt0_Iflr"])
    check_fields(psi, n, p, g["swt0_psi"], g["swt0_n"], g["swt0_p"], g["kind"])


@pytest.mark.parametrize("name", NAMES)
def test_small_sweeps_default_match_reference(lib, name, prec):
    """Production tolerances (the GUI's solver tuple).  The reference then converges
    the quasi-Fermi level of a carrier only where it is >= 1e-3 of the local charge
    scale (its Gummel weight, semiconductor_3d.c:3136-3144), and its terminal currents
    only to its own tolerance: n, p are compared on those nodes, and a current may
    differ by the reference's own distance to its converged value."""
    g = golden(name)
    w, mat, bias = MG.build(lib, name)
    assert lib.api3b_get_precision() == prec
    s = w.sweeps[0]
    ok0, V, I, F, conv, psi, n, p = sweep_fields(lib, w, s)
    assert ok0 and conv.all()
    np.testing.assert_allclose(V, g["sw0_V"])
    own = 2.0 * np.abs(g["sw0_I"] - g["swt0_I"])
    check_currents(I, g["sw0_I"], np.maximum(g["sw0_Iflr"], own))
    dpsi = np.abs(psi - g["sw0_psi"]).max()
    assert dpsi <= PSI_TOL, f"psi differs by {dpsi:.3e} V"
    D_ = np.abs(g["Nd"] - g["Na"])
    free = (g["kind"] == 0) & (g["con"] == 0)
    for a, b, o, lab in ((n, g["sw0_n"], g["sw0_p"], "n"), (p, g["sw0_p"], g["sw0_n"], "p")):
        sig = free[None, :] & (b > NP_FLOOR) & (b >= 1e-3 * (b + o + D_[None, :]))
        if not sig.any():
            continue
        rel = np.abs(a[sig] - b[sig]) / b[sig]
        assert rel.max() <= NP_RTOL, f"{lab} differs by {rel.max():.3e} relative"


def test_concurrent_instances(lib):
    """Three devices solved at once from three host threads, one solver instance (and
    CUDA stream) each: every sweep still matches the reference."""
    import threading
    names = ["diode_small", "mos_small", "moscap_small"]
    hs = [lib.api3b_new() for _ in names]
    out = {}

    def work(name, h):
        lib.api3b_use(h)
        w, mat, bias = MG.build(lib, name)
        out[name] = sweep_fields(lib, w, w.sweeps[0])
        lib.api3b_use(0)

    th = [threading.Thread(target=work, args=(nm, h)) for nm, h in zip(names, hs)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    try:
        for name in names:
            g = golden(name)
            ok0, V, I, F, conv, psi, n, p = out[name]
            assert ok0 and conv.all(), name
            own = 2.0 * np.abs(g["sw0_I"] - g["swt0_I"])
            check_currents(I, g["sw0_I"], np.maximum(g["sw0_Iflr"], own))
            assert np.abs(psi - g["sw0_psi"]).max() <= PSI_TOL, name
    finally:
        for h in hs:
            lib.api3b_free(h)


def reference_lib():
    path = os.path.join(ROOT, "oracle", "_ref", "libsemisim_harness.so")
    if not os.path.exists(path):
        pytest.skip("reference core not built (make -C oracle)")
    return abi.bind(ctypes.CDLL(path))


def test_pn_diode_40cubed_matches_reference(lib, monkeypatch):
    """The 40^3 Si pn diode sweep 0..0.6 V (13 points) on both libraries, run live:
    converged tightly, every target on every node; at the production tolerances, the
    currents within the reference's own error bar (its distance to its converged value,
    or its round-off floor)."""
    ref = reference_lib()
    ref.api3_set_threads(os.cpu_count() or 1)
    out = {}
    for tight in (0, 1):
        for k, v in MG.TIGHT_ENV.items():
            if tight:
                monkeypatch.setenv(k, v)
            else:
                monkeypatch.delenv(k, raising=False)
        for tag, L in (("gpu", lib), ("ref", ref)):
            w = D.pn_diode(L)
            if tight:
                L.api3_set_solver(*MG.TIGHT_SOLVER)
            out[tag, tight] = sweep_fields(L, w, w.sweeps[0])
    allsi = np.zeros(out["gpu", 0][5].shape[1], int)           # every node silicon
    for tight in (0, 1):
        assert out["gpu", tight][0] and out["gpu", tight][4].all() and out["ref", tight][4].all()
    g1, r1 = out["gpu", 1], out["ref", 1]
    check_currents(g1[2], r1[2], r1[3])
    check_fields(g1[5], g1[6], g1[7], r1[5], r1[6], r1[7], allsi)
    g0, r0 = out["gpu", 0], out["ref", 0]
    check_currents(g0[2], r0[2], np.maximum(r0[3], 2.0 * np.abs(r0[2] - r1[2])))
    assert np.abs(g0[5] - r0[5]).max() <= PSI_TOL


@pytest.mark.parametrize("name", ["mos_small"])
def test_autotuned_shapes_keep_parity(lib, name):
    """Launch shapes picked by the autotuner (after the first solve) change no answer: the
    sweep still matches the reference within its error bar."""
    import ctypes
    g = golden(name)
    w, mat, bias = MG.build(lib, name)
    lib.api3b_set_precision(1)
    s = w.sweeps[0]
    try:
        assert D.start_sweep(lib, w, s)
        us = lib.api3b_autotune(1)
        r, gc, sm, zc = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        assert lib.api3b_tune_get(ctypes.byref(r), ctypes.byref(gc), ctypes.byref(sm), ctypes.byref(zc)) == 1
        assert zc.value in (65535, 296, 148)
        assert us > 0.0 and r.value in (2, 4, 8, 16, 32) and gc.value in (592, 1184, 1776) and sm.value in (0, 1024, 2048, 4096, 8192)
        ok0, V, I, F, conv, psi, n, p = sweep_fields(lib, w, s)
        assert ok0 and conv.all()
        own = 2.0 * np.abs(g["sw0_I"] - g["swt0_I"])
        check_currents(I, g["sw0_I"], np.maximum(g["sw0_Iflr"], own))
        assert np.abs(psi - g["sw0_psi"]).max() <= PSI_TOL
    finally:
        lib.api3b_autotune(0)
        lib.api3b_set_precision(-1)


def test_diode_variant_matches_reference(lib):
    """The smallest member of the 64-variant batch family (its own doping, junction depth
    and mesh), refined precision, against the reference core run live: the whole 0..0.7 V
    sweep at the production tolerances, currents within 1e-4 or the reference's floor."""
    ref = reference_lib()
    ref.api3_set_threads(os.cpu_count() or 1)
    var = min(D.diode_variants(64), key=lambda v: int(np.prod(v["n"])))
    out = {}
    for tag, L in (("gpu", lib), ("ref", ref)):
        w = D.diode_variant(L, var)
        if tag == "gpu":
            L.api3b_set_precision(1)
        try:
            out[tag] = sweep_fields(L, w, w.sweeps[0])
        finally:
            if tag == "gpu":
                L.api3b_set_precision(-1)
    g, r = out["gpu"], out["ref"]
    assert g[0] and g[4].all() and r[4].all()
    check_currents(g[2], r[2], r[3])
    assert np.abs(g[5] - r[5]).max() <= PSI_TOL


def test_resolve_batch_matches_sequential_resolves(lib):
    """Six bias vectors around an operating point of the small MOSFET (gate and drain
    perturbed both ways), solved at once by api3b_resolve_batch, give the currents of six
    sequential api3_resolve calls from the restored state (api3_set_state), to 1e-10."""
    import ctypes
    w, mat, bias = MG.build(lib, "mos_small")
    s = dict(w.sweeps[0])
    s["V"] = s["V"][:4]
    assert D.start_sweep(lib, w, s)
    D.run_sweep(lib, w, s)
    nc = lib.api3_get_ncon()
    base = np.array([lib.api3_get_contact_Vsolved(c) for c in range(nc)])
    N = w.N
    st = [np.zeros(N) for _ in range(3)]
    assert lib.api3_get_state(*(abi.dptr(a) for a in st))
    g, d = w.contacts["gate"], w.contacts["drain"]
    Vs = []
    for cid, dv in ((g, 0.01), (g, -0.01), (d, 0.02), (d, -0.02), (g, 0.03), (d, 0.05)):
        v = base.copy()
        v[cid] += dv
        Vs.append(v)
    Vs = np.ascontiguousarray(Vs)
    Ib = np.zeros((len(Vs), nc))
    conv = np.zeros(len(Vs), np.int32)
    try:
        nok = lib.api3b_resolve_batch(len(Vs), abi.dptr(Vs), abi.dptr(Ib), None,
                                      conv.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), 3)
        assert nok == len(Vs) and conv.all()
        # the source instance was not moved
        assert np.allclose([lib.api3_get_contact_Vsolved(c) for c in range(nc)], base)
        Iseq = np.zeros_like(Ib)
        for j, v in enumerate(Vs):
            for c in range(nc):
                lib.api3_set_contact_V(c, float(base[c]))
            assert lib.api3_set_state(*(abi.dptr(a) for a in st))
            for c in range(nc):
                lib.api3_set_contact_V(c, float(v[c]))
            assert lib.api3_resolve()
            Iseq[j] = [lib.api3_get_contact_I(c) for c in range(nc)]
        np.testing.assert_allclose(Ib, Iseq, rtol=1e-10, atol=1e-30)
    finally:
        lib.api3b_resolve_batch_free()
