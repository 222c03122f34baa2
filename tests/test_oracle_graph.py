"""The CPU restatement of the general-mesh kernels (oracle/restate.py: poisson_eval_g,
upd_mob_g, cont_assemble_g) against the reference core's graph path, run live through the
oracle harness on graph devices at a converged bias with seeded perturbations: the Poisson
residual, diagonal and per-edge off-diagonals, the edge mobilities with velocity
saturation, both scaled Scharfetter-Gummel systems, the terminal fluxes, the
multigrid's Slotboom weights and Petrov-Galerkin coarse operators, and the floating-block
balance (on tensor and graph meshes).  Host only: no GPU needed."""
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
from oracle import restate as R  # noqa: E402
from semiconductor_devices_simulator_b200 import abi, devices as D  # noqa: E402
from semiconductor_devices_simulator_b200.abi import dptr, iptr  # noqa: E402

_IP, _DP = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
HXG = dict(MG.HX, hx_graph=(ctypes.c_int, [_IP, _IP, _IP, _DP, _DP, _DP]),
           hx_graph_vals=(ctypes.c_int, [_DP]), hx_graph_mob=(ctypes.c_int, [_DP, _DP]))

CASES = {
    # velocity saturation on, a Robin face gate, source / drain / body node lists
    "mosfet": (lambda L: D.graph_nmosfet(L, n=(16, 12, 4), models=4 | 1 | 2), {"gate": 0.8, "drain": 0.3}),
    # diagonal edges (no tensor product), constant-mobility-free Masetti silicon
    "diode_diag": (lambda L: D.graph_pn_diode(L, diag=0.3, models=7), {"anode": 0.4}),
}


def harness():
    path = os.path.join(ROOT, "oracle", "_ref", "libsemisim_harness.so")
    if not os.path.exists(path):
        pytest.skip("reference core not built (make -C oracle)")
    return abi.bind(ctypes.CDLL(path), HXG)


def state(lib, N):
    """Node state of a graph device (no face mobilities there)."""
    return {k: MG.get(lib, q, N) for k, q in (("phi", MG.W_PHI), ("phin", MG.W_PHIN), ("phip", MG.W_PHIP),
                                               ("n", MG.W_N), ("p", MG.W_P), ("mun", MG.W_MUN), ("mup", MG.W_MUP))}


def close(a, b, rtol, atol=0.0):
    a, b = np.asarray(a, float), np.asarray(b, float)
    err = np.abs(a - b)
    tol = atol + rtol * np.maximum(np.abs(a), np.abs(b))
    assert np.all(err <= tol), f"max err {err.max():.3e} (tol {tol[np.argmax(err - tol)]:.3e})"


@pytest.fixture(scope="module", params=sorted(CASES))
def dumped(request):
    lib = harness()
    build, bias = CASES[request.param]
    w = build(lib)
    lib.api3_set_verbose(0)
    for name, v in bias.items():
        lib.api3_set_contact_V(w.contacts[name], v)
    assert lib.api3_solve()
    rec = MG.device_record(lib, w)
    N = w.N
    E = lib.hx_graph(None, None, None, None, None, None)
    g_rp, g_cj, g_ue = np.zeros(N + 1, np.int32), np.zeros(E, np.int32), np.zeros(E, np.int32)
    g_h, g_ar, g_vol = np.zeros(E), np.zeros(E), np.zeros(N)
    lib.hx_graph(iptr(g_rp), iptr(g_cj), iptr(g_ue), dptr(g_h), dptr(g_ar), dptr(g_vol))
    pos = np.asarray(w.info["pos"], float)           # the builder's node positions
    crec = np.zeros((lib.api3_get_ncon(), 6))
    for c in range(crec.shape[0]):
        lib.hx_contact(c, dptr(crec[c]))
    lib.hx_mob0_init()
    lib.hx_apply_bc()
    st = state(lib, N)
    rng = np.random.default_rng(7)
    semi = rec["kind"] == 0
    free = semi & (rec["con"] == 0)
    phi = st["phi"] + np.where(rec["con"] == 0, rng.normal(0, 2e-3, N), 0.0)
    phin = st["phin"] + np.where(free, rng.normal(0, 5e-3, N), 0.0)
    phip = st["phip"] + np.where(free, rng.normal(0, 5e-3, N), 0.0)
    lib.hx_set(MG.W_PHI, dptr(phi)); lib.hx_set(MG.W_PHIN, dptr(phin)); lib.hx_set(MG.W_PHIP, dptr(phip))
    lib.hx_clamp_qf()
    lib.hx_rebuild_np()
    lib.hx_upd_mob()
    nue = lib.hx_graph_mob(None, None)
    mun, mup = np.zeros(nue), np.zeros(nue)
    lib.hx_graph_mob(dptr(mun), dptr(mup))
    ps = state(lib, N)
    out = {"mob": (mun, mup)}
    nc = lib.api3_get_ncon()
    I, S, In = np.zeros(nc), np.zeros(nc), np.zeros(nc)
    lib.hx_terminal_currents(dptr(I), dptr(S), dptr(In))
    out["cur"] = (I, S, In)
    F, A7, sc = np.zeros(N), np.zeros(7 * N), np.zeros(N)
    nrm = lib.hx_poisson_eval(dptr(ps["phi"]), 1, dptr(F), dptr(A7), dptr(sc))
    gv = np.zeros(E)
    lib.hx_graph_vals(dptr(gv))
    out["pois"] = (F, A7[:N].copy(), gv.copy(), sc, nrm)
    for hole in (0, 1):
        A7, rhs, sc, dsc = np.zeros(7 * N), np.zeros(N), np.zeros(N), np.zeros(N)
        lib.hx_cont_assemble(hole, dptr(A7), dptr(rhs), dptr(sc), dptr(dsc))
        lib.hx_graph_vals(dptr(gv))
        out[f"cont{hole}"] = (A7[:N].copy(), gv.copy(), rhs, sc, dsc)
    dev = dict(rec, **{k: ps[k] for k in ("phi", "phin", "phip", "n", "p", "mun", "mup")})
    dev.update(models=int(w.info["models"]), caxis=1, ref_mat=0, mat=np.zeros(N, np.int64),
               g_rp=g_rp, g_cj=g_cj, g_ue=g_ue, g_h=g_h, g_ar=g_ar, g_vol=g_vol, g_pos=pos,
               con_V=crec[:, 0], con_pm=crec[:, 1], con_tox=crec[:, 2], con_qox=crec[:, 3])
    return dev, out


def test_poisson_graph(dumped):
    dev, out = dumped
    F, dg, gval, sc, nrm = R.poisson_eval_g(dev, dev["phi"])
    Fr, dgr, gvr, scr, nrr = out["pois"]
    close(F, Fr, rtol=1e-11, atol=1e-12 * np.abs(Fr).max())
    close(dg, dgr, rtol=1e-12)
    close(gval, gvr, rtol=1e-12)
    close(sc, scr, rtol=1e-12)
    close(nrm, nrr, rtol=1e-9)


def test_edge_mobility_graph(dumped):
    dev, out = dumped
    mun, mup = R.upd_mob_g(dev)
    close(mun, out["mob"][0], rtol=1e-12)
    close(mup, out["mob"][1], rtol=1e-12)


@pytest.mark.parametrize("hole", [0, 1])
def test_cont_assemble_graph(dumped, hole):
    dev, out = dumped
    mun, mup = out["mob"]
    dg, gval, rhs, sc, dsc = R.cont_assemble_g(dev, hole, mun, mup)
    dgr, gvr, rhr, scr, dsr = out[f"cont{hole}"]
    close(dg, dgr, rtol=0.0)
    close(gval, gvr, rtol=1e-10, atol=1e-300)
    close(rhs, rhr, rtol=1e-10, atol=1e-12 * np.abs(rhr).max())
    close(sc, scr, rtol=1e-13)
    close(dsc, dsr, rtol=1e-10, atol=1e-300)


def test_terminal_currents_graph(dumped):
    dev, out = dumped
    mun, mup = out["mob"]
    I, S, In = R.terminal_currents_g(dev, len(out["cur"][0]), mun, mup)
    Ir, Sr, Inr = out["cur"]
    close(S, Sr, rtol=1e-12)
    # a contact's net current cancels between its in- and outflows: relative to its scale
    close(I, Ir, rtol=0.0, atol=1e-12 * Sr.max())
    close(In, Inr, rtol=0.0, atol=1e-12 * Sr.max())


HXM = dict(HXG, hx_mg_setup=(ctypes.c_int, [ctypes.c_int]),
           hx_gmg_level=(ctypes.c_int, [ctypes.c_int] + [_IP] * 5),
           hx_gmg_vals=(ctypes.c_int, [ctypes.c_int, _DP, _DP]))


@pytest.mark.parametrize("hole", [0, 1], ids=["electrons", "holes"])
def test_graph_multigrid_setup(hole):
    """The Slotboom weights and Petrov-Galerkin coarse operators of the graph multigrid,
    restated (gmg_weights_g, galerkin_g) from the assembled continuity system of a graph
    diode with diagonal edges and the reference's own hierarchy, equal the reference's
    coarse levels to 1e-13."""
    path = os.path.join(ROOT, "oracle", "_ref", "libsemisim_harness.so")
    if not os.path.exists(path):
        pytest.skip("reference core not built (make -C oracle)")
    lib = abi.bind(ctypes.CDLL(path), HXM)
    w = D.graph_pn_diode(lib, n=(24, 12, 8), diag=0.3)
    lib.api3_set_contact_V(w.contacts["anode"], 0.3)
    assert lib.api3_solve()
    N = w.N
    lib.hx_mob0_init(); lib.hx_apply_bc(); lib.hx_rebuild_np(); lib.hx_upd_mob()
    A7, rhs, sc, dsc = np.zeros(7 * N), np.zeros(N), np.zeros(N), np.zeros(N)
    lib.hx_cont_assemble(hole, dptr(A7), dptr(rhs), dptr(sc), dptr(dsc))
    E = lib.hx_graph(None, None, None, None, None, None)
    va0 = np.zeros(E)
    lib.hx_graph_vals(dptr(va0))
    dg0 = A7[:N].copy()
    qs = -1 if hole else 1
    nl = lib.hx_mg_setup(qs)
    assert nl >= 3
    levels = []
    for L in range(nl):
        n, nnz = np.zeros(1, np.int32), np.zeros(1, np.int32)
        lib.hx_gmg_level(L, iptr(n), iptr(nnz), None, None, None)
        rp, cj, agg = np.zeros(n[0] + 1, np.int32), np.zeros(max(nnz[0], 1), np.int32), np.zeros(n[0], np.int32)
        lib.hx_gmg_level(L, iptr(n), iptr(nnz), iptr(rp), iptr(cj), iptr(agg))
        va, dg = np.zeros(max(nnz[0], 1)), np.zeros(n[0])
        lib.hx_gmg_vals(L, dptr(va), dptr(dg))
        levels.append({"rp": rp, "cj": cj[:nnz[0]], "agg": agg, "va": va[:nnz[0]], "dg": dg})
    # level-0 reference potentials (ph0, semiconductor_3d.c:2085-2090), phi in units of VT
    kind, con = np.zeros(N, np.int32), np.zeros(N, np.int32)
    lib.hx_masks(iptr(kind), iptr(con), iptr(np.zeros(N, np.int32)))
    phin, phip = MG.get(lib, MG.W_PHIN, N), MG.get(lib, MG.W_PHIP, N)
    rec = np.zeros(128)
    lib.hx_mat(0, dptr(rec))
    VT = rec[R.MF["VT"]]
    fixed = (kind != 0) | (con != 0)
    ph0 = np.where(fixed, -1e300, phin / VT if qs > 0 else -phip / VT)
    pws = R.gmg_weights_g(levels, ph0)
    va, dg = va0, dg0
    for L in range(nl - 1):
        f, c = levels[L], levels[L + 1]
        cva, cdg = R.galerkin_g(f["rp"], f["cj"], va, dg, f["agg"], c["rp"], c["cj"], pws[L],
                                dsc if L == 0 else None)
        scale = np.abs(c["va"]).max()
        assert np.abs(cva - c["va"]).max() <= 1e-13 * scale, f"level {L + 1} couplings"
        assert np.allclose(cdg, c["dg"], rtol=1e-13, atol=0.0), f"level {L + 1} diagonal"
        va, dg = c["va"], c["dg"]


HXFF = dict(HXG, hx_float_fix=(ctypes.c_int, [ctypes.c_int, _DP]))


@pytest.mark.parametrize("graph", [1, 0], ids=["graph", "tensor"])
def test_float_fix_restated(graph):
    """The floating-block balance restated (float_fix, both mesh kinds) against the
    reference on the n base of a p+ n p+ bar contacted only at its ends: the electron
    system assembled at the equilibrium state with 0.3 V newly applied, a seeded solution
    vector; the same block fixed and the rescaled solution equal to 1e-12."""
    path = os.path.join(ROOT, "oracle", "_ref", "libsemisim_harness.so")
    if not os.path.exists(path):
        pytest.skip("reference core not built (make -C oracle)")
    lib = abi.bind(ctypes.CDLL(path), HXFF)
    w = D.floating_base_pnp(lib, graph=bool(graph))
    assert lib.api3_solve()
    lib.api3_set_contact_V(w.contacts["anode"], 0.3)
    N = w.N
    lib.hx_mob0_init(); lib.hx_apply_bc(); lib.hx_rebuild_np(); lib.hx_upd_mob()
    A7, rhs, sc, dsc = np.zeros(7 * N), np.zeros(N), np.zeros(N), np.zeros(N)
    lib.hx_cont_assemble(0, dptr(A7), dptr(rhs), dptr(sc), dptr(dsc))
    rec = MG.device_record(lib, w)
    dev = dict(rec, **state(lib, N))
    dev.update(models=7, caxis=1, ref_mat=0, mat=np.zeros(N, np.int64))
    if graph:
        E = lib.hx_graph(None, None, None, None, None, None)
        g_rp, g_cj, g_ue = np.zeros(N + 1, np.int32), np.zeros(E, np.int32), np.zeros(E, np.int32)
        g_h, g_ar, g_vol = np.zeros(E), np.zeros(E), np.zeros(N)
        lib.hx_graph(iptr(g_rp), iptr(g_cj), iptr(g_ue), dptr(g_h), dptr(g_ar), dptr(g_vol))
        dev.update(g_rp=g_rp, g_cj=g_cj, g_ue=g_ue, g_h=g_h, g_ar=g_ar, g_vol=g_vol)
        nue = lib.hx_graph_mob(None, None)
        mun, mup = np.zeros(nue), np.zeros(nue)
        lib.hx_graph_mob(dptr(mun), dptr(mup))
        nbrs, vol = R.neighbours_graph(dev, mun, mup)
    else:
        dev["fmu"] = np.array([MG.get(lib, 16 + q, N) for q in range(6)])
        nbrs, vol = R.neighbours_tensor(dev)
    sol0 = 1.0 + np.random.default_rng(11).normal(0, 0.02, N)
    nfix, u = R.float_fix(dev, 0, sol0, sc, nbrs, vol)
    sol = sol0.copy()
    nref = lib.hx_float_fix(0, dptr(sol))
    assert nref >= 1 and nfix == nref
    assert np.abs(u - sol).max() <= 1e-12 * np.abs(sol).max()


def test_graph_display_outputs_restated():
    """At a solved state of the graph diode with diagonal edges: the node current densities
    (bulk_copy 7-9 and the electron / hole parts 20-25) from the restated least-squares
    operator equal the reference's to 1e-8 of their peak.  A node's density is the difference
    of drift and diffusion fluxes ~1e6 times larger, and the reference is compiled with
    contractions (-ffast-math): one rounding of those terms is ~3e-9 of the peak here.  The
    largest field (api3_get_Emax) agrees to 1e-9."""
    path = os.path.join(ROOT, "oracle", "_ref", "libsemisim_harness.so")
    if not os.path.exists(path):
        pytest.skip("reference core not built (make -C oracle)")
    lib = abi.bind(ctypes.CDLL(path), HXG)
    w = D.graph_pn_diode(lib, diag=0.3, models=7)
    lib.api3_set_contact_V(w.contacts["anode"], 0.5)
    assert lib.api3_solve()
    N = w.N
    rec = MG.device_record(lib, w)
    dev = dict(rec, **state(lib, N))
    E = lib.hx_graph(None, None, None, None, None, None)
    g_rp, g_cj, g_ue = np.zeros(N + 1, np.int32), np.zeros(E, np.int32), np.zeros(E, np.int32)
    g_h, g_ar, g_vol = np.zeros(E), np.zeros(E), np.zeros(N)
    lib.hx_graph(iptr(g_rp), iptr(g_cj), iptr(g_ue), dptr(g_h), dptr(g_ar), dptr(g_vol))
    dev.update(models=7, caxis=1, ref_mat=0, mat=np.zeros(N, np.int64), g_rp=g_rp, g_cj=g_cj, g_ue=g_ue,
               g_h=g_h, g_ar=g_ar, g_vol=g_vol, g_pos=np.asarray(w.info["pos"], float))
    nue = lib.hx_graph_mob(None, None)
    mun, mup = np.zeros(nue), np.zeros(nue)
    lib.hx_graph_mob(dptr(mun), dptr(mup))
    for which, qs in ((0, (7, 8, 9)), (1, (20, 21, 22)), (2, (23, 24, 25))):
        J = R.graph_node_J(dev, mun, mup, which)
        ref = np.stack([D.field(lib, q, w.shape).ravel() for q in qs], axis=1)
        assert np.abs(J - ref).max() <= 1e-8 * np.abs(ref).max(), f"J part {which}"
    g = R.graph_grad(dev, dev["phi"], R.graph_lsq(dev))
    emax = np.sqrt(np.max(np.sum(g * g, axis=1)))
    assert abs(emax - lib.api3_get_Emax()) <= 1e-9 * lib.api3_get_Emax()


def test_graph_impact_ionisation_restated():
    """Impact-ionisation generation on a graph (models bit 8): the Si p+n diode of the
    avalanche tests given as a graph, solved at -8 V; the restated generation (least-squares
    node currents and field, the Chynoweth law with the van Overstraeten - de Man
    coefficients) equals the reference's ii_update at the same state to 1e-7 of its peak."""
    path = os.path.join(ROOT, "oracle", "_ref", "libsemisim_harness.so")
    if not os.path.exists(path):
        pytest.skip("reference core not built (make -C oracle)")
    lib = abi.bind(ctypes.CDLL(path), dict(HXG, hx_ii_update=(ctypes.c_int, [_DP])))
    w = D.graph_pn_diode(lib, n=(40, 3, 3), NA=1e19, ND=1e17, xj=0.3e-6, tau=1e-9, models=7 | 256)
    lib.api3_set_contact_V(w.contacts["anode"], -8.0)
    assert lib.api3_solve()
    N = w.N
    rec = MG.device_record(lib, w)
    dev = dict(rec, **state(lib, N))
    E = lib.hx_graph(None, None, None, None, None, None)
    g_rp, g_cj, g_ue = np.zeros(N + 1, np.int32), np.zeros(E, np.int32), np.zeros(E, np.int32)
    g_h, g_ar, g_vol = np.zeros(E), np.zeros(E), np.zeros(N)
    lib.hx_graph(iptr(g_rp), iptr(g_cj), iptr(g_ue), dptr(g_h), dptr(g_ar), dptr(g_vol))
    dev.update(models=7 | 256, caxis=1, ref_mat=0, mat=np.zeros(N, np.int64), g_rp=g_rp, g_cj=g_cj, g_ue=g_ue,
               g_h=g_h, g_ar=g_ar, g_vol=g_vol, g_pos=np.asarray(w.info["pos"], float))
    nue = lib.hx_graph_mob(None, None)
    mun, mup = np.zeros(nue), np.zeros(nue)
    lib.hx_graph_mob(dptr(mun), dptr(mup))
    gref = np.zeros(N)
    lib.hx_ii_update(dptr(gref))
    g = R.graph_ii(dev, mun, mup)
    assert gref.max() > 0
    assert np.abs(g - gref).max() <= 1e-7 * gref.max()
