"""Thermionic-emission metal contacts (models bit 6: image-force lowering; bit 7: barrier
tunnelling) against the reference core run live on the same inputs.

* Whole sweeps of n-Si Schottky diodes (1e16 cm^-3 forward and reverse with emission
  only; 1e18 cm^-3 forward and reverse with tunnelling) in both precisions.  Converged
  tightly (inner solves to round-off, Gummel tolerance 1e-12 V): psi within 1e-6 V, n, p
  within 1e-6 relative above 1e9 m^-3 wherever the carrier is >= 1e-6 of the local charge
  scale (the reverse-biased barrier's trace electrons, ~1e-10 of the doping, settle only to
  ~1e-4 in the reference itself), currents within 1e-6 relative or the reference's
  round-off floor Iflr (the V = 0 point carries ~1e-26 A of round-off).  At the
  production tolerances: psi within 1e-6 V and currents within 1e-4 relative or Iflr (the
  reference converges a trace carrier - the electrons in the depleted barrier region - only
  where it is >= 1e-6 of the local charge scale, so n is not compared there).
* The exchange terms themselves on one installed state: emission coefficients, image-force
  lowering, column tunnelling terms and the per-node band lowering after one te_update.
* Batched resolves with metal contacts equal sequential resolves from the restored state.
"""
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

PSI_TOL, NP_RTOL, NP_FLOOR, I_RTOL = 1e-6, 1e-6, 1e9, 1e-6
CASES = {
    "te_fwd": dict(ND=1e16, models=7 | 64),
    "te_rev": dict(ND=1e16, models=7 | 64, V=np.round(np.linspace(0, -1.0, 6), 12)),
    "tun_fwd": dict(ND=1e18, models=7 | 64 | 128),
    "tun_rev": dict(ND=1e18, models=7 | 64 | 128, V=np.round(np.linspace(0, -0.5, 6), 12)),
}


@pytest.fixture(scope="module")
def lib():
    return S.load()


HX_TE = {"hx_te_update": (None, []), "hx_rebuild_np": (None, []),
         "hx_set_qc": (None, [ctypes.POINTER(ctypes.c_double)] * 2),
         "hx_te": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int)] + [ctypes.POINTER(ctypes.c_double)] * 7)}


def reference_lib():
    path = os.path.join(ROOT, "oracle", "_ref", "libsemisim_harness.so")
    if not os.path.exists(path):
        pytest.skip("reference core not built (make -C oracle)")
    ref = abi.bind(ctypes.CDLL(path), HX_TE)
    ref.api3_set_threads(os.cpu_count() or 1)
    return ref


def sweep(L, kw, tight=False):
    kw = dict(kw)
    if tight:
        kw["solver"] = MG.TIGHT_SOLVER
    w = D.schottky_diode(L, **kw)
    s = w.sweeps[0]
    ok0 = D.start_sweep(L, w, s)
    psi, nn, pp = [], [], []

    def grab(q, v):
        psi.append(D.field(L, 0, w.shape).ravel())
        nn.append(D.field(L, 1, w.shape).ravel())
        pp.append(D.field(L, 2, w.shape).ravel())
    V, I, F, conv = D.run_sweep(L, w, s, on_point=grab)
    return ok0, I, F, conv, np.array(psi), np.array(nn), np.array(pp)


@pytest.mark.parametrize("tight", [1, 0], ids=["tight", "default"])
@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "refined"])
@pytest.mark.parametrize("case", sorted(CASES))
def test_schottky_sweep_matches_reference(lib, case, prec, tight, monkeypatch):
    for k, v in MG.TIGHT_ENV.items():
        if tight:
            monkeypatch.setenv(k, v)
        else:
            monkeypatch.delenv(k, raising=False)
    ref = reference_lib()
    old = lib.api3b_set_precision(prec)
    try:
        g = sweep(lib, CASES[case], tight)
    finally:
        lib.api3b_set_precision(old)
    r = sweep(ref, CASES[case], tight)
    assert g[0] and r[0] and g[3].all() and r[3].all()
    dpsi = np.abs(g[4] - r[4]).max()
    assert dpsi <= PSI_TOL, f"psi differs by {dpsi:.3e} V"
    if tight:
        ND = CASES[case]["ND"] * 1e6
        for a, b, o, lab in ((g[5], r[5], r[6], "n"), (g[6], r[6], r[5], "p")):
            m = (b > NP_FLOOR) & (b >= 1e-6 * (b + o + ND))
            rel = np.abs(a[m] - b[m]) / b[m]
            assert rel.max() <= NP_RTOL, f"{lab} differs by {rel.max():.3e} relative"
    tol = np.maximum((I_RTOL if tight else 1e-4) * np.abs(r[1]), r[2])
    err = np.abs(g[1] - r[1])
    assert (err <= tol).all(), f"currents\n{g[1]}\n{r[1]}"


def test_metal_exchange_terms_match_reference(lib):
    """One te_update on the same installed state: this library's solution at -0.3 V on the
    tunnelling diode and its image-force band, put into both libraries (api3_set_state, the
    band, n and p rebuilt from it)."""
    ref = reference_lib()
    kw = dict(CASES["tun_rev"])
    kw["V"] = np.array([0.0, -0.1, -0.2, -0.3])
    out = {}
    for tag, L in (("gpu", lib), ("ref", ref)):
        w = D.schottky_diode(L, **kw)
        s = w.sweeps[0]
        assert D.start_sweep(L, w, s)
        D.run_sweep(L, w, s)
        out[tag] = w
    N = out["gpu"].N
    st = [np.zeros(N) for _ in range(3)]
    assert lib.api3_get_state(*(dptr(a) for a in st)) == 1
    cnt = np.zeros(2, np.int32)
    qc = [np.zeros(N), np.zeros(N)]
    lib.b200x_te(iptr(cnt), None, None, None, None, None, dptr(qc[0]), dptr(qc[1]))
    assert ref.api3_set_state(*(dptr(a) for a in st)) == 1
    assert lib.api3_set_state(*(dptr(a) for a in st)) == 1
    ref.hx_set_qc(dptr(qc[0]), dptr(qc[1]))
    assert lib.b200x_set_qc(dptr(qc[0]), dptr(qc[1])) == 1
    ref.hx_rebuild_np()
    lib.b200x_rebuild_np()
    assert lib.b200x_te_update() == 1
    ref.hx_te_update()
    cnt = np.zeros(2, np.int32)
    rec = {}
    for tag, fn in (("gpu", lib.b200x_te), ("ref", ref.hx_te)):
        fn(iptr(cnt), None, None, None, None, None, None, None)
        nte, ntc = int(cnt[0]), int(cnt[1])
        a = [np.zeros(2 * nte), np.zeros(2 * nte), np.zeros(2 * ntc), np.zeros(2 * ntc), np.zeros(2 * ntc),
             np.zeros(N), np.zeros(N)]
        assert fn(iptr(cnt), *(dptr(x) for x in a)) == nte
        rec[tag] = (nte, ntc, a)
    assert rec["gpu"][:2] == rec["ref"][:2] and rec["gpu"][0] > 0
    g, r = rec["gpu"][2], rec["ref"][2]
    # the entry node's own column slot carries its emission terms in this library
    first = np.zeros(rec["gpu"][1], bool)
    names = ["te_K", "te_G", "tc_K", "tc_G", "tc_I", "qcn", "qcp"]
    for i, nm in enumerate(names):
        a, b = g[i].copy(), r[i]
        if nm in ("tc_K", "tc_G"):
            # entries start where the reference has zero in the column slot of the entry node
            z = (b.reshape(-1, 2) == 0).all(1) & (a.reshape(-1, 2) != 0).any(1)
            first |= z
            a = a.reshape(-1, 2)
            a[z] = 0.0
            a = a.ravel()
        scale = np.abs(b).max()
        err = np.abs(a - b).max()
        assert err <= 1e-10 * scale + 1e-300, f"{nm}: {err:.3e} of {scale:.3e}"
    assert first.any()


def test_batched_resolve_with_metal_contacts(lib):
    """Bias vectors around an operating point of the tunnelling diode, solved at once by
    api3b_resolve_batch, give the currents of sequential api3_resolve calls from the
    restored state, to the Gummel tolerance: the image-force band is part of the solver
    state that api3_set_state leaves alone (as in the reference), so a sequential resolve
    starts from the band of the previous resolve and a batched one from the operating
    point's (the worker copies carry it)."""
    kw = dict(CASES["tun_fwd"])
    kw["V"] = np.array([0.0, 0.1, 0.2])
    w = D.schottky_diode(lib, **kw)
    s = w.sweeps[0]
    assert D.start_sweep(lib, w, s)
    D.run_sweep(lib, w, s)
    nc = lib.api3_get_ncon()
    base = np.array([lib.api3_get_contact_Vsolved(c) for c in range(nc)])
    N = w.N
    st = [np.zeros(N) for _ in range(3)]
    assert lib.api3_get_state(*(dptr(a) for a in st))
    a = w.contacts["anode"]
    Vs = []
    for dv in (0.01, -0.01, 0.03, -0.05):
        v = base.copy()
        v[a] += dv
        Vs.append(v)
    Vs = np.ascontiguousarray(Vs)
    Ib = np.zeros((len(Vs), nc))
    conv = np.zeros(len(Vs), np.int32)
    try:
        assert lib.api3b_resolve_batch(len(Vs), dptr(Vs), dptr(Ib), None, iptr(conv), 2) == len(Vs)
    finally:
        lib.api3b_resolve_batch_free()
    for j, v in enumerate(Vs):
        assert lib.api3_set_state(*(dptr(x) for x in st))
        for c in range(nc):
            lib.api3_set_contact_V(c, float(v[c]))
        assert lib.api3_resolve()
        Iq = np.array([lib.api3_get_contact_I(c) for c in range(nc)])
        assert np.allclose(Ib[j], Iq, rtol=1e-5, atol=1e-22), (j, Ib[j], Iq)
