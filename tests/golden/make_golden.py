"""Generate the golden vectors of the parity tests from the reference core itself.

Runs the oracle harness (oracle/harness.c: the unmodified reference core
semiconductor_3d.c #included, plus dump hooks) on small seeded devices and writes one
.npz per device into this folder:

  diode_small   Si pn diode 12x6x5, models 0, constant mobility (the 40^3 workload's
                physics at a size the oracle finishes at once)
  mos_small     n-MOSFET 16x12x6 with an oxide Robin face gate, models 7 (band-gap
                narrowing, tau(N), velocity saturation)
  moscap_small  Si / SiO2 stack 8x10x4 with a metal gate electrode on the oxide and a
                Schottky back contact (insulator and metal node kinds)
  sic_small     4H-SiC pn diode 14x5x4 (p+ 1e18 / n 1e16 cm^-3), models 519: band-gap
                narrowing, tau(N), velocity saturation and incomplete ionisation of the
                nitrogen donors and aluminium acceptors; anode swept 0..2.8 V

Each file holds the prepared device (masks, geometry, materials, contacts), a
converged state and, at a perturbed state, the outputs of the per-node kernels
(poisson_eval, upd_mob_ref, cont_assemble, cont_update, terminal_currents), the
multigrid hierarchy of the electron system (level shapes, Galerkin operators,
Slotboom weights, restriction / prolongation of a seeded vector) and the bias sweep
end to end (psi, n, p per point and every terminal current with its floor).

Usage (needs the reference checkout and `make -C oracle`):
    python tests/golden/make_golden.py
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from semiconductor_devices_simulator_b200 import abi, devices as D   # noqa: E402
from semiconductor_devices_simulator_b200.abi import dptr, iptr       # noqa: E402

_I, _D, _L = ctypes.c_int, ctypes.c_double, ctypes.c_long
_DP, _IP, _LP = ctypes.POINTER(_D), ctypes.POINTER(_I), ctypes.POINTER(_L)
HX = {
    "hx_N": (_L, []), "hx_prepare": (_I, []), "hx_equilibrium": (_I, []), "hx_nlev": (_I, []),
    "hx_cref": (_D, []), "hx_masks": (None, [_IP, _IP, _IP]), "hx_rob": (_I, [_LP, _DP, _IP]),
    "hx_contact_area": (None, [_DP]), "hx_contact": (_I, [_I, _DP]), "hx_get": (_I, [_I, _DP]), "hx_set": (_I, [_I, _DP]),
    "hx_poisson_eval": (_D, [_DP, _I, _DP, _DP, _DP]), "hx_apply_bc": (None, []),
    "hx_rebuild_np": (None, []), "hx_mob0_init": (None, []), "hx_upd_mob": (None, []),
    "hx_clamp_qf": (None, []), "hx_vlo": (_D, []), "hx_vhi": (_D, []),
    "hx_cont_assemble": (None, [_I, _DP, _DP, _DP, _DP]),
    "hx_cont_update": (_D, [_I, _DP, _D, _D, _DP]),
    "hx_float_fix": (_I, [_I, _DP]),
    "hx_terminal_currents": (None, [_DP, _DP, _DP]),
    "hx_mg_setup": (_I, [_I]), "hx_mg_level": (_I, [_I, _IP, _DP, _DP, _DP]),
    "hx_mg_matvec": (_I, [_I, _DP, _DP]), "hx_mg_restrict": (_I, [_I, _DP, _DP]),
    "hx_mg_prolong": (_I, [_I, _DP, _DP]), "hx_bicg_floor": (_D, [_DP, _DP]),
    "hx_B": (_D, [_D]), "hx_mat": (_I, [_I, _DP]), "hx_ion": (_I, [_DP]),
}
W_PHI, W_PHIN, W_PHIP, W_N, W_P, W_MUN, W_MUP, W_BGN, W_EPS, W_ND, W_NA, W_NF = range(12)


def load_harness():
    path = os.path.join(ROOT, "oracle", "_ref", "libsemisim_harness.so")
    lib = abi.bind(ctypes.CDLL(path), HX)
    return lib


def get(lib, which, N):
    a = np.zeros(N)
    assert lib.hx_get(which, dptr(a))
    return a


def device_record(lib, w):
    """Prepared device description in the restatement's layout (oracle/restate.py)."""
    assert lib.hx_prepare(), "prepare failed"
    N = int(lib.hx_N())
    kind = np.zeros(N, np.int32); con = np.zeros(N, np.int32); gate = np.zeros(N, np.int32)
    lib.hx_masks(iptr(kind), iptr(con), iptr(gate))
    nrob = lib.hx_rob(None, None, None)
    rk = np.zeros(max(nrob, 1), np.int64); rA = np.zeros(max(nrob, 1)); rc = np.zeros(max(nrob, 1), np.int32)
    lib.hx_rob(rk.ctypes.data_as(_LP), dptr(rA), iptr(rc))
    nc = lib.api3_get_ncon()
    area = np.zeros(nc)
    lib.hx_contact_area(dptr(area))
    mats = []
    for mi in range(16):
        rec = np.zeros(128)
        m = lib.hx_mat(mi, dptr(rec))
        if m == 0:
            break
        mats.append(rec[:m])
    Nx, Ny, Nz = w.shape
    xs = np.array([lib.api3_get_xs(i) for i in range(Nx)])
    ys = np.array([lib.api3_get_ys(i) for i in range(Ny)])
    zs = np.array([lib.api3_get_zs(i) for i in range(Nz)])
    # material index per node: recovered from eps and the Nd/Na layout is not unique,
    # so the builders' material ids are passed explicitly
    rec = dict(dims=np.array(w.shape), xs=xs, ys=ys, zs=zs, kind=kind, con=con, gate=gate,
               rob_k=rk[:nrob], rob_A=rA[:nrob], rob_c=rc[:nrob], con_A=area,
               mats=np.array(mats), Cref=lib.hx_cref(),
               Nd=get(lib, W_ND, N), Na=get(lib, W_NA, N), Nf=get(lib, W_NF, N),
               bgn=get(lib, W_BGN, N), eps=get(lib, W_EPS, N))
    nw = lib.hx_ion(None)
    if nw:                                   # incomplete-ionisation constants, (N, 4)
        ion = np.zeros(nw * N)
        lib.hx_ion(dptr(ion))
        rec["ion"] = ion.reshape(N, nw)
    return rec


def state(lib, N):
    return dict(phi=get(lib, W_PHI, N), phin=get(lib, W_PHIN, N), phip=get(lib, W_PHIP, N),
                n=get(lib, W_N, N), p=get(lib, W_P, N), mun=get(lib, W_MUN, N), mup=get(lib, W_MUP, N),
                fmu=np.array([get(lib, 16 + q, N) for q in range(6)]))


# Tight tolerances: inner solves to round-off and a Gummel tolerance of 1e-12 V, so the
# sweep converges to the discrete solution itself (trace carriers included).  The
# environment knobs are the reference's own (semiconductor_3d.c:4578-4581).
TIGHT_ENV = {"SEMISIM_BRTOL": "1e-12", "SEMISIM_PCGRTOL": "1e-10"}
TIGHT_SOLVER = (2000, 1000, 500, 1e-12, 1e-9, 1.0, 1.0)


def sweep_record(lib, w, tag=""):
    """End-to-end: api3_solve at the first point of every sweep, then api3_resolve per
    point; keys sw<tag><sweep>_* (tag "" default tolerances, "t" tight)."""
    out = {}
    for si, s in enumerate(w.sweeps):
        si = f"{tag}{si}"
        ok0 = D.start_sweep(lib, w, s)
        psi, nn, pp, qn, qp = [], [], [], [], []

        def grab(q, v):
            psi.append(D.field(lib, 0, w.shape).ravel()); nn.append(D.field(lib, 1, w.shape).ravel())
            pp.append(D.field(lib, 2, w.shape).ravel()); qn.append(D.field(lib, 15, w.shape).ravel())
            qp.append(D.field(lib, 16, w.shape).ravel())
        V, I, F, conv = D.run_sweep(lib, w, s, on_point=grab)
        out[f"sw{si}_V"] = V; out[f"sw{si}_I"] = I; out[f"sw{si}_Iflr"] = F
        out[f"sw{si}_conv"] = conv; out[f"sw{si}_start_ok"] = np.array(ok0)
        out[f"sw{si}_psi"] = np.array(psi); out[f"sw{si}_n"] = np.array(nn); out[f"sw{si}_p"] = np.array(pp)
        out[f"sw{si}_phin"] = np.array(qn); out[f"sw{si}_phip"] = np.array(qp)
        out[f"sw{si}_swept"] = np.array(w.contacts[s["swept"]])
        fixed = np.array([[w.contacts[k], v] for k, v in s["fixed"].items()])
        out[f"sw{si}_fixed"] = fixed
    return out


def kernels(lib, w, rec, mat_idx, bias, seed):
    """Per-node kernel outputs at a converged bias with seeded perturbations."""
    N = w.N
    rng = np.random.default_rng(seed)
    for cid, v in bias.items():
        lib.api3_set_contact_V(cid, v)
    ok = lib.api3_solve()
    out = {"kern_solve_ok": np.array(ok), "kern_bias": np.array(sorted(bias.items()))}
    crec = np.zeros((lib.api3_get_ncon(), 6))
    for c in range(crec.shape[0]):
        lib.hx_contact(c, dptr(crec[c]))
    out.update(con_V=crec[:, 0].copy(), con_pm=crec[:, 1].copy(), con_tox=crec[:, 2].copy(),
               con_qox=crec[:, 3].copy(), con_bc=crec[:, 4].astype(np.int32), con_face=crec[:, 5].astype(np.int32))
    lib.hx_mob0_init()          # node mobility back to the low-field values (mob_display overwrote it)
    lib.hx_apply_bc()
    st = state(lib, N)
    out.update({"conv_" + k: v for k, v in st.items()})
    # perturbed state: quasi-Fermi potentials and psi moved by seeded noise
    semi = rec["kind"] == 0
    free = semi & (rec["con"] == 0)
    phi = st["phi"] + np.where(rec["con"] == 0, rng.normal(0, 2e-3, N), 0.0)
    phin = st["phin"] + np.where(free, rng.normal(0, 5e-3, N), 0.0)
    phip = st["phip"] + np.where(free, rng.normal(0, 5e-3, N), 0.0)
    lib.hx_set(W_PHI, dptr(phi)); lib.hx_set(W_PHIN, dptr(phin)); lib.hx_set(W_PHIP, dptr(phip))
    lib.hx_clamp_qf()
    lib.hx_rebuild_np()
    lib.hx_upd_mob()
    ps = state(lib, N)
    out.update({"pert_" + k: v for k, v in ps.items()})
    out["vlo"] = np.array(lib.hx_vlo()); out["vhi"] = np.array(lib.hx_vhi())
    F = np.zeros(N); A7 = np.zeros(7 * N); sc = np.zeros(N)
    out["pois_norm"] = np.array(lib.hx_poisson_eval(dptr(ps["phi"]), 1, dptr(F), dptr(A7), dptr(sc)))
    out["pois_F"] = F.copy(); out["pois_A"] = A7.reshape(7, N).copy(); out["pois_sc"] = sc.copy()
    nc = lib.api3_get_ncon()
    I = np.zeros(nc); S = np.zeros(nc); In = np.zeros(nc)
    lib.hx_terminal_currents(dptr(I), dptr(S), dptr(In))
    out["cur_I"] = I; out["cur_S"] = S; out["cur_In"] = In
    for hole, tag in ((0, "n"), (1, "p")):
        A7 = np.zeros(7 * N); rhs = np.zeros(N); sc = np.zeros(N); dsc = np.zeros(N)
        lib.hx_cont_assemble(hole, dptr(A7), dptr(rhs), dptr(sc), dptr(dsc))
        out[f"cont{tag}_A"] = A7.reshape(7, N).copy(); out[f"cont{tag}_rhs"] = rhs
        out[f"cont{tag}_sc"] = sc; out[f"cont{tag}_dsc"] = dsc
        x = 1.0 + rng.normal(0, 0.05, N)
        out[f"cont{tag}_x"] = x
        out[f"cont{tag}_floor"] = np.array(lib.hx_bicg_floor(dptr(rhs), dptr(x)))
        if hole == 0:
            # multigrid hierarchy of the electron system (Slotboom weights, weighted Galerkin)
            nl = lib.hx_mg_setup(1)
            out["mg_nlev"] = np.array(nl)
            for L in range(nl):
                dims = np.zeros(6, np.int32)
                lib.hx_mg_level(L, iptr(dims), None, None, None)
                NL = int(dims[0] * dims[1] * dims[2])
                A7L = np.zeros(7 * NL); pw = np.zeros(NL); ph = np.zeros(NL)
                lib.hx_mg_level(L, iptr(dims), dptr(A7L), dptr(pw), dptr(ph))
                out[f"mg{L}_dims"] = dims.copy(); out[f"mg{L}_A"] = A7L.reshape(7, NL)
                out[f"mg{L}_pw"] = pw; out[f"mg{L}_ph"] = ph
                if L < nl - 1:
                    r = rng.normal(0, 1, NL)
                    dn = np.zeros(6, np.int32); lib.hx_mg_level(L + 1, iptr(dn), None, None, None)
                    NC = int(dn[0] * dn[1] * dn[2])
                    bc = np.zeros(NC); lib.hx_mg_restrict(L, dptr(r), dptr(bc))
                    xc = rng.normal(0, 1, NC); xf = np.zeros(NL)
                    lib.hx_mg_prolong(L, dptr(xc), dptr(xf))
                    out[f"mg{L}_r"] = r; out[f"mg{L}_rc"] = bc; out[f"mg{L}_xc"] = xc; out[f"mg{L}_xf"] = xf
            y = np.zeros(N); lib.hx_mg_matvec(0, dptr(x), dptr(y)); out["contn_Ax"] = y
        sol = 1.0 + rng.normal(0, 0.02, N)
        dq = np.zeros(N)
        out[f"cont{tag}_sol"] = sol
        out[f"cont{tag}_dmax"] = np.array(lib.hx_cont_update(hole, dptr(sol), lib.hx_vlo(), lib.hx_vhi(), dptr(dq)))
        out[f"cont{tag}_dq"] = dq
        after = state(lib, N)
        out[f"cont{tag}_qf"] = after["phip" if hole else "phin"]
        out[f"cont{tag}_car"] = after["p" if hole else "n"]
        # restore the perturbed state for the other carrier
        lib.hx_set(W_PHIN, dptr(ps["phin"])); lib.hx_set(W_PHIP, dptr(ps["phip"]))
        lib.hx_set(W_N, dptr(ps["n"])); lib.hx_set(W_P, dptr(ps["p"]))
    out["mat"] = mat_idx
    return out


def build(lib, name):
    if name == "diode_small":
        w = D.pn_diode(lib, n=(12, 6, 5))
        mat = np.zeros(w.N, np.int32)
        bias = {w.contacts["anode"]: 0.45, w.contacts["cathode"]: 0.0}
    elif name == "mos_small":
        w = D.nmosfet(lib, n=(16, 12, 6), models=7, vds=(0.5,), vg_max=1.0, dvg=0.25)
        mat = np.zeros(w.N, np.int32)
        bias = {w.contacts["gate"]: 0.8, w.contacts["drain"]: 0.5}
    elif name == "sic_small":
        w = D.pn_diode(lib, n=(14, 5, 4), NA=1e18, ND=1e16, material=D.SIC, mobility=None, tau=None,
                       models=519, vmax=2.8, dv=0.4)
        mat = np.zeros(w.N, np.int32)
        bias = {w.contacts["anode"]: 2.6, w.contacts["cathode"]: 0.0}
    elif name == "moscap_small":
        w = moscap(lib)
        mat = w.info.pop("mat")
        bias = {w.contacts["gate"]: 0.7}
    else:
        raise ValueError(name)
    return w, mat, bias


def moscap(lib, n=(8, 10, 4)):
    """p-Si under a SiO2 layer, metal gate electrode on the oxide (bc 2 on insulator
    nodes: Dirichlet), Schottky back contact (bc 1); gate swept 0..1 V."""
    lib.api3_init()
    xs = np.linspace(0, 40e-9, n[0]); ys = np.linspace(0, 60e-9, n[1]); zs = np.linspace(0, 20e-9, n[2])
    D._grid(lib, xs, ys, zs)
    lib.api3_set_solver(*D.GUI_SOLVER)
    lib.api3_set_models(1)
    si = lib.api3_add_material(D.SI, 300.0)
    ox = lib.api3_add_material(D.SIO2, 300.0)
    lib.api3_set_region(0, 0, 0, n[0] - 1, n[1] - 1, n[2] - 1, si, 0.0, 3e23)
    lib.api3_set_region(0, n[1] - 3, 0, n[0] - 1, n[1] - 1, n[2] - 1, ox, 0.0, 0.0)
    lib.api3_clear_contacts()
    cb = lib.api3_add_contact_ex(2, 0, n[0] - 1, 0, n[2] - 1, 0, 0, 1, 0.0, 4.9, 0.0, 0.0)
    cg = lib.api3_add_contact_ex(3, 0, n[0] - 1, 0, n[2] - 1, 0, 0, 2, 0.0, 4.6, 0.0, 0.0)
    mat = np.zeros(n[0] * n[1] * n[2], np.int32).reshape(n[2], n[1], n[0])
    mat[:, n[1] - 3:, :] = 1
    V = np.round(np.linspace(0.0, 1.0, 5), 12)
    return D.Workload("moscap", n, {"back": cb, "gate": cg},
                      [{"fixed": {"back": 0.0}, "swept": "gate", "V": V}], {"mat": mat.ravel()})


def main(names=("diode_small", "mos_small", "moscap_small", "sic_small")):
    lib = load_harness()
    lib.api3_set_threads(1)          # fixed thread count: the chunked ILU depends on it
    for name in names:
        w, mat, bias = build(lib, name)
        rec = device_record(lib, w)
        rec["models"] = np.array(w.info.get("models", 1))
        rec["caxis"] = np.array(1)
        rec["ref_mat"] = np.array(0)
        out = dict(rec)
        out.update(kernels(lib, w, rec, mat, bias, seed=1234))
        w, mat, bias = build(lib, name)              # fresh device for the sweep
        out.update(sweep_record(lib, w))
        os.environ.update(TIGHT_ENV)                 # read by api3_init
        w, mat, bias = build(lib, name)
        lib.api3_set_solver(*TIGHT_SOLVER)
        out.update(sweep_record(lib, w, "t"))
        for k in TIGHT_ENV:
            del os.environ[k]
        out["threads"] = np.array(1)
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **out)
        print(f"{name}: {w.shape} -> {os.path.relpath(path, ROOT)} ({os.path.getsize(path)//1024} KiB)")


if __name__ == "__main__":
    main(tuple(sys.argv[1:]) or ("diode_small", "mos_small", "moscap_small", "sic_small"))
