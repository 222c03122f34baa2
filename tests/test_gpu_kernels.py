"""Kernel-level parity of the CUDA solve path against the reference.

Every device kernel runs through the library's b200x_* hooks on the same seeded state
the golden vectors were dumped at (tests/golden/*.npz, from the reference core), and on
top of that against the numpy restatement (oracle/restate.py).  FP64 throughout, except
the refined linear solves (FP32 inner solves refined in FP64), which are held to the
reference's FP64 stop rule; the tolerances are stated per quantity.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_golden as MG  # noqa: E402
from oracle import restate as R  # noqa: E402
import semiconductor_devices_simulator_b200 as S  # noqa: E402
from semiconductor_devices_simulator_b200.abi import dptr, iptr  # noqa: E402

pytestmark = pytest.mark.gpu
NAMES = ["diode_small", "mos_small", "moscap_small", "sic_small"]


def golden(name):
    z = np.load(os.path.join(HERE, "golden", name + ".npz"))
    return {k: z[k] for k in z.files}


def close(a, b, rtol, atol=0.0, what=""):
    a, b = np.asarray(a, float), np.asarray(b, float)
    err = np.abs(a - b)
    tol = atol + rtol * np.maximum(np.abs(a), np.abs(b))
    bad = ~(err <= tol)
    assert not bad.any(), f"{what}: {bad.sum()} mismatches, worst {err.max():.3e} (tol {tol.ravel()[np.argmax(err)]:.3e})"


@pytest.fixture(scope="module")
def lib():
    return S.load()


def setup(lib, name):
    g = golden(name)
    w, mat, bias = MG.build(lib, name)
    for cid, v in g["kern_bias"]:
        lib.api3_set_contact_V(int(cid), float(v))
    assert lib.b200x_prepare() == 1
    return g, w


def put(lib, which, a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    assert lib.b200x_set(which, dptr(a)) == 1


def get(lib, which, N):
    a = np.zeros(N)
    assert lib.b200x_get(which, dptr(a)) == 1
    return a


def load_state(lib, g, prefix):
    put(lib, S.ST_PHI, g[prefix + "phi"]); put(lib, S.ST_PHIN, g[prefix + "phin"])
    put(lib, S.ST_PHIP, g[prefix + "phip"]); put(lib, S.ST_N, g[prefix + "n"]); put(lib, S.ST_P, g[prefix + "p"])
    for q in range(6):
        put(lib, S.ST_FMU + q, g[prefix + "fmu"][q])


@pytest.mark.parametrize("name", NAMES)
def test_prepare_masks(lib, name):
    g, w = setup(lib, name)
    N = w.N
    kind = np.zeros(N, np.int32); con = np.zeros(N, np.int32); gate = np.zeros(N, np.int32); robA = np.zeros(N)
    assert lib.b200x_masks(iptr(kind), iptr(con), iptr(gate), dptr(robA)) == 1
    np.testing.assert_array_equal(kind, g["kind"])
    np.testing.assert_array_equal(con, g["con"])
    np.testing.assert_array_equal(gate, g["gate"])
    ref = np.zeros(N)
    ref[g["rob_k"].astype(int)] = g["rob_A"]
    close(robA, ref, 1e-15, what="Robin areas")
    for c in range(len(g["con_A"])):
        close(lib.api3_get_contact_A(c), g["con_A"][c], 1e-14, what=f"contact {c} area")
    close(lib.api3_get_Cref(), g["Cref"], 1e-15, what="Cref")
    # low-field node mobility of the semiconductor nodes
    semi = g["kind"] == 0
    close(get(lib, S.ST_MU0N, N)[semi], g["pert_mun"][semi], 1e-14, what="mu0n")
    close(get(lib, S.ST_MU0P, N)[semi], g["pert_mup"][semi], 1e-14, what="mu0p")


@pytest.mark.parametrize("name", NAMES)
def test_poisson_eval(lib, name):
    g, w = setup(lib, name)
    N = w.N
    load_state(lib, g, "pert_")
    F = np.zeros(N); A7 = np.zeros(7 * N); sc = np.zeros(N)
    nrm = lib.b200x_poisson(dptr(np.ascontiguousarray(g["pert_phi"])), dptr(F), dptr(A7), dptr(sc))
    scale = np.abs(g["pois_F"]).max()
    close(F, g["pois_F"], 1e-11, 1e-12 * scale, "F")
    close(A7.reshape(7, N), g["pois_A"], 1e-12, what="Jacobian")
    close(sc, g["pois_sc"], 1e-12, what="sc")
    close(nrm, g["pois_norm"], 1e-9, what="norm")


@pytest.mark.parametrize("name", NAMES)
def test_face_mobility(lib, name):
    g, w = setup(lib, name)
    N = w.N
    load_state(lib, g, "pert_")
    lib.b200x_upd_mob()
    fmu = np.array([get(lib, S.ST_FMU + q, N) for q in range(6)])
    close(fmu, g["pert_fmu"], 1e-12, what="face mobility")


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("hole", [0, 1])
def test_cont_assemble_update(lib, name, hole):
    g, w = setup(lib, name)
    N = w.N
    t = "p" if hole else "n"
    load_state(lib, g, "pert_")
    A7 = np.zeros(7 * N); rhs = np.zeros(N); sc = np.zeros(N); dsc = np.zeros(N)
    lib.b200x_cont_assemble(hole, dptr(A7), dptr(rhs), dptr(sc), dptr(dsc))
    close(A7.reshape(7, N), g[f"cont{t}_A"], 1e-10, 1e-300, "A")
    close(rhs, g[f"cont{t}_rhs"], 1e-10, 1e-12 * np.abs(g[f"cont{t}_rhs"]).max(), "rhs")
    close(sc, g[f"cont{t}_sc"], 1e-13, what="sc")
    close(dsc, g[f"cont{t}_dsc"], 1e-10, 1e-300, "dsc")
    dq = np.zeros(N)
    dmax = lib.b200x_cont_update(hole, dptr(np.ascontiguousarray(g[f"cont{t}_sol"])), float(g["vlo"]),
                                 float(g["vhi"]), dptr(dq))
    close(dq, g[f"cont{t}_dq"], 1e-9, 1e-15, "dq")
    close(dmax, g[f"cont{t}_dmax"], 1e-9, 1e-15, "dmax")
    close(get(lib, S.ST_PHIP if hole else S.ST_PHIN, N), g[f"cont{t}_qf"], 1e-12, 1e-15, "qf")
    close(get(lib, S.ST_P if hole else S.ST_N, N), g[f"cont{t}_car"], 1e-11, 1e-300, "carrier")


@pytest.mark.parametrize("name", NAMES)
def test_terminal_currents(lib, name):
    g, w = setup(lib, name)
    load_state(lib, g, "pert_")
    nc = len(g["cur_I"])
    I = np.zeros(nc); Sv = np.zeros(nc); In = np.zeros(nc)
    lib.b200x_currents(dptr(I), dptr(Sv), dptr(In))
    close(Sv, g["cur_S"], 1e-12, what="S")
    close(I, g["cur_I"], 1e-9, 1e-13 * np.abs(g["cur_S"]).max(), "I")
    close(In, g["cur_In"], 1e-9, 1e-13 * np.abs(g["cur_S"]).max(), "In")


@pytest.mark.parametrize("name", NAMES)
def test_multigrid_hierarchy(lib, name):
    g, w = setup(lib, name)
    N = w.N
    load_state(lib, g, "pert_")
    lib.b200x_cont_assemble(0, None, None, None, None)
    nl = lib.b200x_mg_setup(1)
    assert nl == int(g["mg_nlev"])
    for L in range(nl):
        dims = np.zeros(6, np.int32)
        lib.b200x_mg_level(L, iptr(dims), None, None)
        np.testing.assert_array_equal(dims[:3], g[f"mg{L}_dims"][:3])
        NL = int(np.prod(dims[:3]))
        A7 = np.zeros(7 * NL); pw = np.zeros(NL)
        lib.b200x_mg_level(L, iptr(dims), dptr(A7), dptr(pw))
        close(A7.reshape(7, NL), g[f"mg{L}_A"], 1e-10, 1e-300, f"level {L} operator")
        if L < nl - 1:
            close(pw, g[f"mg{L}_pw"], 1e-13, what=f"level {L} weights")


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("hole", [0, 1])
def test_bicgstab_solves_continuity(lib, name, hole):
    """The MG-preconditioned BiCGSTAB reaches the reference's stopping rule
    ||b - A x|| <= max(rtol ||r0||, atol floor) on the reference's own system."""
    g, w = setup(lib, name)
    N = w.N
    t = "p" if hole else "n"
    load_state(lib, g, "pert_")
    lib.b200x_cont_assemble(hole, None, None, None, None)
    sol = np.zeros(N); rn = np.zeros(1); r0 = np.zeros(1)
    rtol, atol = 1e-6, 2e-14
    its = lib.b200x_bicgstab(1000, rtol, atol, -1 if hole else 1, None, dptr(sol), dptr(rn), dptr(r0))
    A, b = g[f"cont{t}_A"], g[f"cont{t}_rhs"]
    dims = tuple(int(v) for v in g["dims"])
    res = np.linalg.norm(b - R.matvec(A, dims, sol))
    r00 = np.linalg.norm(b - R.matvec(A, dims, np.ones(N)))
    tgt = max(rtol * r00, atol * R.bicg_floor(A, dims, b, np.ones(N)))
    assert its < 200
    assert res <= 1.5 * tgt + 1e-300, (res, tgt, its)


@pytest.mark.parametrize("name", NAMES)
def test_pcg_solves_poisson(lib, name):
    g, w = setup(lib, name)
    N = w.N
    load_state(lib, g, "pert_")
    F = np.zeros(N)
    lib.b200x_poisson(dptr(np.ascontiguousarray(g["pert_phi"])), dptr(F), None, None)
    sol = np.zeros(N)
    its = lib.b200x_pcg(2000, 1e-8, dptr(sol))
    A = g["pois_A"]
    dims = tuple(int(v) for v in g["dims"])
    res = np.linalg.norm(g["pois_F"] - R.matvec(A, dims, sol))
    assert its < 100
    assert res <= 1e-5 * np.linalg.norm(g["pois_F"]), (res, its)


@pytest.fixture
def refined(lib):
    old = lib.api3b_set_precision(1)
    yield
    lib.api3b_set_precision(old)


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("hole", [0, 1])
@pytest.mark.parametrize("rtol", [1e-4, 1e-10])
def test_refined_bicgstab_meets_fp64_stop_rule(lib, refined, name, hole, rtol):
    """FP32 Krylov / multigrid inner solves refined in FP64: the FP64 residual of the
    result meets the reference's FP64 rule ||b - A x|| <= max(rtol ||r0||, atol floor),
    also far below FP32 round-off (rtol 1e-10)."""
    g, w = setup(lib, name)
    N = w.N
    t = "p" if hole else "n"
    load_state(lib, g, "pert_")
    lib.b200x_cont_assemble(hole, None, None, None, None)
    sol = np.zeros(N); rn = np.zeros(1); r0 = np.zeros(1)
    atol = 2e-14
    s0, f0 = ir_stats(lib)
    its = lib.b200x_bicgstab(1000, rtol, atol, -1 if hole else 1, None, dptr(sol), dptr(rn), dptr(r0))
    A, b = g[f"cont{t}_A"], g[f"cont{t}_rhs"]
    dims = tuple(int(v) for v in g["dims"])
    res = np.linalg.norm(b - R.matvec(A, dims, sol))
    r00 = np.linalg.norm(b - R.matvec(A, dims, np.ones(N)))
    tgt = max(rtol * r00, atol * R.bicg_floor(A, dims, b, np.ones(N)))
    assert its < 400
    assert res <= 1.5 * tgt + 1e-300, (res, tgt, its)
    close(r0[0], r00, 1e-9, what="initial residual")


def ir_stats(lib):
    from ctypes import c_longlong, byref
    a, b = c_longlong(0), c_longlong(0)
    lib.b200x_ir_stats(byref(a), byref(b))
    return a.value, b.value


@pytest.mark.parametrize("name", NAMES)
def test_refined_pcg_matches_fp64(lib, refined, name):
    """FP32 PCG (the Newton-Poisson correction; the Newton loop's FP64 residual refines
    it) reaches the same relative stop rule as the FP64 solve, and its correction agrees
    with the FP64 one to that tolerance."""
    g, w = setup(lib, name)
    N = w.N
    load_state(lib, g, "pert_")
    F = np.zeros(N)
    lib.b200x_poisson(dptr(np.ascontiguousarray(g["pert_phi"])), dptr(F), None, None)
    sol32 = np.zeros(N)
    its32 = lib.b200x_pcg(2000, 1e-5, dptr(sol32))
    lib.api3b_set_precision(0)
    sol64 = np.zeros(N)
    its64 = lib.b200x_pcg(2000, 1e-5, dptr(sol64))
    lib.api3b_set_precision(1)
    A = g["pois_A"]
    dims = tuple(int(v) for v in g["dims"])
    nF = np.linalg.norm(g["pois_F"])
    res32 = np.linalg.norm(g["pois_F"] - R.matvec(A, dims, sol32))
    res64 = np.linalg.norm(g["pois_F"] - R.matvec(A, dims, sol64))
    assert its32 <= its64 + 3, (its32, its64)
    assert res32 <= 1e-3 * nF and res64 <= 1e-3 * nF, (res32, res64, nF)
    assert np.abs(sol32 - sol64).max() <= 1e-3 * np.abs(sol64).max()


def test_ionisation_constants(lib):
    """The device's incomplete-ionisation constants of the 4H-SiC diode (level constants
    of the nitrogen sites and the aluminium acceptor from the host, the neutral majority
    density from the device's Newton on the neutrality condition) against the reference's."""
    g, w = setup(lib, "sic_small")
    N = w.N
    assert lib.b200x_ion(None) == 4
    x = np.zeros(4 * N)
    assert lib.b200x_ion(dptr(x)) == 4
    x = x.reshape(N, 4)
    close(x[:, :3], g["ion"][:, :3], 1e-14, what="level constants")
    close(x[:, 3], g["ion"][:, 3], 1e-11, what="neutral majority density")
    g2, w2 = setup(lib, "diode_small")
    assert lib.b200x_ion(None) == 0
