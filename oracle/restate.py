"""CPU restatement of the reference solve path's per-node kernels (oracle; test
infrastructure only - never imported by the product library or timed as it).

Each function restates one routine of the reference core semiconductor_3d.c in
vectorised numpy and cites the lines it follows.  The parity tests pin these
restatements against golden vectors dumped from the reference itself
(tests/golden/make_golden.py, oracle/harness.c) and then use them as the checker for
the CUDA kernels on seeded inputs.

A device is a dict of numpy arrays (the golden fixture layout):
  dims (Nx,Ny,Nz); xs, ys, zs; kind, con, gate (int, per node); mat (int per node);
  Nd, Na, Nf, bgn (per node); phi, phin, phip, n, p, mun, mup (state); fmu (6,N);
  mats: (n_mats, F) records in the field order MAT_FIELDS; models; caxis; rob_k,
  rob_A, rob_c; con_V, con_tox, con_qox, con_pm (per contact); Cref; ref_mat.
Node index k = i + Nx*(j + Ny*l) (semiconductor_3d.c:114).
"""
import numpy as np

Q = 1.602176634e-19            # semiconductor_3d.c:95-99
KB = 1.380649e-23
EPS0 = 8.8541878128e-12
EPS_OX = 3.9 * EPS0
LN_MIN, LN_MAX, NFLOOR = -230.0, 150.0, 1e-100   # semiconductor_3d.c:108-110
K_SEMI, K_INS, K_METAL = 0, 1, 2
PH_NONE = -1e300

# field order of the material records written by oracle/harness.c (hx_mat)
MAT_FIELDS = ["T", "VT", "Eg", "chi", "eps_r", "Nc", "Nv", "ni",
              "mu_n_max", "mu_p_max", "mu_n_min", "mu_p_min", "Nref_n", "Nref_p", "alpha_n", "alpha_p",
              "mt_min", "mt_max_n", "mt_max_p", "mt_Nref", "mt_alpha", "mas_on",
              "vsat_n", "vsat_p", "beta_n", "beta_p", "tau_n0", "tau_p0", "Cn", "Cp", "Brad", "tau_Nref",
              "bgn_E", "bgn_N", "bgn_C", "lnc", "lnv", "insulator", "ani_n", "ani_p",
              "ion_on", "ion_w0", "ion_w1", "ion_Ed0", "ion_Ed1", "ion_ad0", "ion_ad1",
              "ion_gd", "ion_Ea", "ion_aa", "ion_ga",
              "ii_on", "ii_a00", "ii_a01", "ii_a10", "ii_a11", "ii_b00", "ii_b01", "ii_b10", "ii_b11",
              "ii_E00", "ii_E01", "ii_m0", "ii_m1", "ii_g"]
MF = {n: i for i, n in enumerate(MAT_FIELDS)}


def matp(dev, name):
    """Per-node value of material field `name`."""
    return dev["mats"][dev["mat"], MF[name]]


# ------------------------------------------------------------------ scalar physics
def bernoulli(x):
    """B(x) = x/(e^x-1): series below 1e-6, limits beyond +-700 (semiconductor_3d.c:670-675)."""
    x = np.asarray(x, dtype=np.float64)
    out = np.empty_like(x)
    small = np.abs(x) < 1e-6
    big = x > 700.0
    neg = x < -700.0
    mid = ~(small | big | neg)
    out[small] = 1.0 - x[small] / 2.0 + x[small] ** 2 / 12.0
    out[big] = 0.0
    out[neg] = -x[neg]
    with np.errstate(over="ignore", divide="ignore", invalid="ignore"):
        out[mid] = x[mid] / np.expm1(x[mid])
    return out


def clampe(e):
    """semiconductor_3d.c:677"""
    return np.clip(e, LN_MIN, LN_MAX)


def lncK(dev):
    """ln of the electron effective density incl. band-gap narrowing (semiconductor_3d.c:736)."""
    return matp(dev, "lnc") + dev["bgn"]


def lnvK(dev):
    """semiconductor_3d.c:737"""
    return matp(dev, "lnv") + dev["bgn"]


def niK(dev):
    """semiconductor_3d.c:738 (no quantum correction in scope)"""
    return matp(dev, "ni") * np.exp(dev["bgn"])


def nK(dev, psi, qn):
    """semiconductor_3d.c:739-741"""
    with np.errstate(over="ignore", invalid="ignore"):
        return np.exp(clampe(lncK(dev) + (psi - qn) / matp(dev, "VT")))


def pK(dev, psi, qp):
    """semiconductor_3d.c:742-744"""
    with np.errstate(over="ignore", invalid="ignore"):
        return np.exp(clampe(lnvK(dev) + (qp - psi) / matp(dev, "VT")))


# ------------------------------------------------------------------ incomplete ionisation
def _ion_fields(dev):
    return dev["mats"].shape[1] > MF["ion_ga"]


def ion_consts(dev):
    """Per-node ionisation constants (semiconductor_3d.c:1472-1510): N_c/g_D e^(-dE_s/kT)
    of the two donor sites, N_v/g_A e^(-dE_A/kT), dE = dE0 - alpha N^(1/3) clamped at 0,
    and the neutral majority density |n - p| at the neutral potential; None when models
    bit 9 is off or no semiconductor material has level data."""
    if not (dev["models"] & 512) or not _ion_fields(dev):
        return None
    mats = dev["mats"]
    if not np.any((mats[:, MF["ion_on"]] != 0) & (mats[:, MF["insulator"]] == 0)):
        return None
    N = len(dev["Nd"])
    x = np.zeros((N, 4))
    on = (dev["kind"] == K_SEMI) & (matp(dev, "ion_on") != 0)
    VT = matp(dev, "VT")
    Nd, Na = dev["Nd"], dev["Na"]
    cd = np.cbrt(Nd)
    for s_ in range(2):
        E = np.maximum(matp(dev, f"ion_Ed{s_}") - matp(dev, f"ion_ad{s_}") * cd, 0.0)
        x[:, s_] = np.where(on & (Nd > 0), matp(dev, "Nc") / matp(dev, "ion_gd") * np.exp(-E / VT), 0.0)
    E = np.maximum(matp(dev, "ion_Ea") - matp(dev, "ion_aa") * np.cbrt(Na), 0.0)
    x[:, 2] = np.where(on & (Na > 0), matp(dev, "Nv") / matp(dev, "ion_ga") * np.exp(-E / VT), 0.0)
    d2 = dict(dev)
    d2["ion"] = x
    io = ion_node(d2)
    psi = neutral_psi(d2, 0.0)
    n, p = nK(d2, psi, 0.0), pK(d2, psi, 0.0)
    x[:, 3] = np.where(io, np.abs(n - p), 0.0)
    return x


def ion_node(dev):
    """semiconductor_3d.c:755-757"""
    x = dev.get("ion")
    if x is None:
        return np.zeros(len(dev["Nd"]), bool)
    return ((x[:, 0] > 0) & (dev["Nd"] > 0)) | ((x[:, 2] > 0) & (dev["Na"] > 0))


def ion_eval(dev, n, p):
    """Ionised donor / acceptor densities and their psi-derivatives at fixed quasi-Fermi
    potentials (semiconductor_3d.c:758-777); fully ionised where no constants apply."""
    Nd, Na = dev["Nd"], dev["Na"]
    x = dev.get("ion")
    if x is None:
        z = np.zeros_like(Nd)
        return Nd.copy(), z, Na.copy(), z.copy()
    VT = matp(dev, "VT")
    e = dev["bgn"]
    w0, w1 = matp(dev, "ion_w0"), matp(dev, "ion_w1")
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        ne = np.where(e != 0, n * np.exp(-e), n)
        don = (Nd > 0) & (x[:, 0] > 0)
        a = ne / np.where(don, x[:, 0], 1.0)
        f = w0 / (1 + a)
        df = -w0 * a / ((1 + a) * (1 + a))
        two = don & (w1 > 0) & (x[:, 1] > 0)
        b = ne / np.where(two, x[:, 1], 1.0)
        f = np.where(two, f + w1 / (1 + b), f)
        df = np.where(two, df - w1 * b / ((1 + b) * (1 + b)), df)
        Np = np.where(don, Nd * f, Nd)
        dNp = np.where(don, Nd * df / VT, 0.0)
        pe = np.where(e != 0, p * np.exp(-e), p)
        acc = (Na > 0) & (x[:, 2] > 0)
        c = pe / np.where(acc, x[:, 2], 1.0)
        Nm = np.where(acc, Na / (1 + c), Na)
        dNm = np.where(acc, Na * c / ((1 + c) * (1 + c) * VT), 0.0)
    return Np, dNp, Nm, dNm


def neutral_psi(dev, V):
    """Neutral potential with both quasi-Fermi levels at V (semiconductor_3d.c:1782-1805):
    closed form, then on incompletely ionised nodes the safeguarded Newton on
    p - n + N_D+ - N_A- + Nf = 0 (no traps in scope), each node stopping on its own."""
    VT = matp(dev, "VT")
    D = dev["Nd"] - dev["Na"]
    with np.errstate(divide="ignore", invalid="ignore"):
        psi = V + VT * (np.arcsinh(D / (2.0 * niK(dev))) - 0.5 * (lncK(dev) - lnvK(dev)))
    act = ion_node(dev).copy()
    if not act.any():
        return psi
    Eg = matp(dev, "Eg")
    lo, hi = psi - Eg - 1.0, psi + Eg + 1.0
    for _ in range(200):
        if not act.any():
            break
        n, p = nK(dev, psi, V), pK(dev, psi, V)
        Np, dNp, Nm, dNm = ion_eval(dev, n, p)
        g = p - n + Np - Nm + dev["Nf"]
        dg = -(n + p) / VT + dNp - dNm
        lo = np.where(act & (g > 0), psi, lo)
        hi = np.where(act & ~(g > 0), psi, hi)
        with np.errstate(divide="ignore", invalid="ignore"):
            nx = np.where(dg < 0, psi - g / dg, 0.5 * (lo + hi))
        nx = np.where((nx > lo) & (nx < hi), nx, 0.5 * (lo + hi))
        done = np.abs(nx - psi) < 1e-13 * (1.0 + np.abs(psi))
        psi = np.where(act, nx, psi)
        act = act & ~done
    return psi


def tauf(dev):
    """SRH lifetime doping factor (semiconductor_3d.c:787-791)."""
    tn = matp(dev, "tau_Nref")
    f = 1.0 / (1.0 + (dev["Nd"] + dev["Na"]) / np.where(tn > 0, tn, 1.0))
    on = (dev["models"] & 2) != 0
    return np.where(on & (tn > 0), f, 1.0)


def recomb(dev, n, p):
    """SRH + Auger + radiative with derivatives (semiconductor_3d.c:686-697)."""
    ni = niK(dev)
    tf = tauf(dev)
    tp0, tn0 = matp(dev, "tau_p0"), matp(dev, "tau_n0")
    Cn, Cp, Br = matp(dev, "Cn"), matp(dev, "Cp"), matp(dev, "Brad")
    ni2 = ni * ni
    np_ = n * p - ni2
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        den = tf * (tp0 * (n + ni) + tn0 * (p + ni)) + 1e-300
        Rs = np_ / den
        dsn = (p * den - np_ * tf * tp0) / (den * den)
        dsp = (n * den - np_ * tf * tn0) / (den * den)
        Au = Cn * n + Cp * p
        R = Rs + Au * np_ + Br * np_
        dRn = dsn + Cn * np_ + Au * p + Br * p
        dRp = dsp + Cp * np_ + Au * n + Br * n
    return R, dRn, dRp


def mob_hf(mu0, E, vsat, beta):
    """Caughey-Thomas saturation (semiconductor_3d.c:664-668)."""
    r = mu0 * np.abs(E) / vsat
    with np.errstate(over="ignore", divide="ignore", invalid="ignore"):
        s = mu0 / np.power(1.0 + np.power(r, beta), 1.0 / beta)
    return np.where(r < 1e-12, mu0, s)


def heat_field(dq, dps, h):
    """Harmonic-mean driving field (semiconductor_3d.c:2882-2886)."""
    a, b = np.abs(dq), np.abs(dps)
    with np.errstate(divide="ignore", invalid="ignore"):
        F = 2.0 * a * b / ((a + b) * h)
    return np.where(dq * dps <= 0.0, 0.0, F)


# ------------------------------------------------------------------ geometry
def fv_len(c):
    """Finite-volume lengths with half cells on the faces (semiconductor_3d.c:700-705)."""
    c = np.asarray(c, float)
    N = len(c)
    L = np.empty(N)
    if N < 2:
        return np.ones(N)
    L[0] = 0.5 * (c[1] - c[0])
    L[-1] = 0.5 * (c[-1] - c[-2])
    L[1:-1] = 0.5 * (c[2:] - c[:-2])
    return L


class Grid:
    """Neighbour bookkeeping of nbr() (semiconductor_3d.c:709-719) as per-direction
    index / validity / spacing / area arrays over the flattened nodes."""

    def __init__(self, dev):
        Nx, Ny, Nz = (int(v) for v in dev["dims"])
        self.Nx, self.Ny, self.Nz = Nx, Ny, Nz
        self.N = Nx * Ny * Nz
        xs, ys, zs = (np.asarray(dev[a], float) for a in ("xs", "ys", "zs"))
        Lx, Ly, Lz = fv_len(xs), fv_len(ys), fv_len(zs)
        l, j, i = np.meshgrid(np.arange(Nz), np.arange(Ny), np.arange(Nx), indexing="ij")
        i, j, l = i.ravel(), j.ravel(), l.ravel()
        self.i, self.j, self.l = i, j, l
        k = np.arange(self.N)
        self.vol = Lx[i] * Ly[j] * Lz[l]
        self.valid, self.kb, self.h, self.ar = [], [], [], []
        for d in range(6):
            ax, up = d // 2, d % 2
            idx = (i, j, l)[ax]
            nmax = (Nx, Ny, Nz)[ax]
            st = (1, Nx, Nx * Ny)[ax]
            c = (xs, ys, zs)[ax]
            if up:
                v = idx < nmax - 1
                kb = np.where(v, k + st, k)
                h = np.where(v, c[np.minimum(idx + 1, nmax - 1)] - c[idx], 1.0)
            else:
                v = idx > 0
                kb = np.where(v, k - st, k)
                h = np.where(v, c[idx] - c[np.maximum(idx - 1, 0)], 1.0)
            ar = (Ly[j] * Lz[l], Lx[i] * Lz[l], Lx[i] * Ly[j])[ax]
            self.valid.append(v)
            self.kb.append(kb)
            self.h.append(h)
            self.ar.append(ar)


# ------------------------------------------------------------------ Poisson
def poisson_eval(dev, phi, g=None):
    """F, 7-point Jacobian (c,xm,xp,ym,yp,zm,zp), sc and ||F/sc|| (semiconductor_3d.c:2732-2789)."""
    g = g or Grid(dev)
    N = g.N
    kind, con = dev["kind"], dev["con"]
    isdir = con != 0
    eps = matp(dev, "eps_r") * EPS0
    F = np.zeros(N)
    dg = np.zeros(N)
    off = np.zeros((6, N))
    for d in range(6):
        v, kb = g.valid[d], g.kb[d]
        ek, eb = eps, eps[kb]
        cf = np.where(v, (2.0 * ek * eb / (ek + eb)) * g.ar[d] / g.h[d], 0.0)
        F += cf * (phi[kb] - phi)
        dg += cf
        off[d] = np.where(v & ~isdir[kb], -cf, 0.0)
    semi = kind == K_SEMI
    n = nK(dev, phi, dev["phin"])
    p = pK(dev, phi, dev["phip"])
    VT = matp(dev, "VT")
    Np, dNp, Nm, dNm = ion_eval(dev, n, p)          # the doping itself where fully ionised
    F += np.where(semi, g.vol * Q * (p - n + Np - Nm + dev["Nf"]), g.vol * Q * dev["Nf"])
    dg += np.where(semi, g.vol * Q * ((n + p) / VT - dNp + dNm), 0.0)
    A = np.vstack([dg[None, :], off])
    sc = dg.copy()
    F[isdir] = 0.0
    A[:, isdir] = 0.0
    A[0, isdir] = 1.0
    sc[isdir] = 1.0
    for r in range(len(dev["rob_k"])):
        k, c = int(dev["rob_k"][r]), int(dev["rob_c"][r])
        tox = dev["con_tox"][c] if dev["con_tox"][c] > 0 else 10e-9
        Cox = EPS_OX / tox
        pm = dev["con_pm"][c] if dev["con_pm"][c] > 0 else dev["Cref"]
        VG = dev["con_V"][c] + dev["Cref"] - pm
        F[k] += dev["rob_A"][r] * (Cox * (VG - phi[k]) + dev["con_qox"][c])
        A[0, k] += Cox * dev["rob_A"][r]
        sc[k] = A[0, k]
    return F, A, sc, float(np.sqrt(np.sum((F / sc) ** 2)))


# ------------------------------------------------------------------ mobility
def upd_mob(dev, g=None):
    """Face mobilities fmu[6][N] from node mobility and the potentials
    (semiconductor_3d.c:2962-3006; Lombardi/Coulomb branches out of scope)."""
    g = g or Grid(dev)
    kind = dev["kind"]
    semi = kind == K_SEMI
    fmu = np.zeros((6, g.N))
    sat = (dev["models"] & 4) != 0
    for ax in range(3):
        d = 2 * ax + 1
        v, kb, h = g.valid[d], g.kb[d], g.h[d]
        ok = semi & v & semi[kb]
        mn = 0.5 * (dev["mun"] + dev["mun"][kb])
        mp = 0.5 * (dev["mup"] + dev["mup"][kb])
        if ax == dev["caxis"]:
            an, ap = matp(dev, "ani_n"), matp(dev, "ani_p")
            mn = np.where(an > 0, mn * an, mn)
            mp = np.where(ap > 0, mp * ap, mp)
        if sat:
            dps = dev["phi"][kb] - dev["phi"]
            Fn = heat_field(dev["phin"][kb] - dev["phin"], dps, h)
            Fp = heat_field(dev["phip"][kb] - dev["phip"], dps, h)
            mn = mob_hf(mn, Fn, matp(dev, "vsat_n"), matp(dev, "beta_n"))
            mp = mob_hf(mp, Fp, matp(dev, "vsat_p"), matp(dev, "beta_p"))
        fmu[ax] = np.where(ok, mn, 0.0)
        fmu[3 + ax] = np.where(ok, mp, 0.0)
    return fmu


# ------------------------------------------------------------------ continuity
def car_fix(dev):
    """Contact nodes keep fixed carrier densities (semiconductor_3d.c:796-799; no
    thermionic-emission contacts in scope)."""
    return dev["con"] != 0


def cont_assemble(dev, hole, g=None):
    """Scaled SG system for u = c/s: A (7,N), rhs, sc, dsc (semiconductor_3d.c:3067-3106)."""
    g = g or Grid(dev)
    N = g.N
    kind = dev["kind"]
    semi = kind == K_SEMI
    fix = car_fix(dev)
    car = dev["p"] if hole else dev["n"]
    VT = matp(dev, "VT")
    lc = lnvK(dev) if hole else lncK(dev)
    sk = np.maximum(car, NFLOOR)
    dg = np.zeros(N)
    b = np.zeros(N)
    off = np.zeros((6, N))
    fmu = dev["fmu"]
    for d in range(6):
        v, kb, h, ar = g.valid[d], g.kb[d], g.h[d], g.ar[d]
        ok = v & semi[kb]
        dl = lc[kb] - lc
        D = (dev["phi"][kb] - dev["phi"]) / VT + (-dl if hole else dl)
        kl = np.minimum(np.arange(N), kb)
        gg = ar * fmu[(3 if hole else 0) + d // 2][kl] * VT / h
        self_ = gg * (bernoulli(D) if hole else bernoulli(-D))
        nb = gg * (bernoulli(-D) if hole else bernoulli(D))
        dg += np.where(ok, self_, 0.0)
        b += np.where(ok & fix[kb], nb * car[kb], 0.0)
        off[d] = np.where(ok & ~fix[kb], -nb * np.maximum(car[kb], NFLOOR), 0.0)
    R, dRn, dRp = recomb(dev, dev["n"], dev["p"])
    dR = np.maximum(dRp if hole else dRn, 0.0)
    dg += g.vol * dR
    b += g.vol * (dR * car - R)
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        w = 1.0 / (dg * sk)
    A = np.vstack([np.ones((1, N)), off * w])
    rhs = b * w
    sc = sk.copy()
    dsc = dg * sk
    ident = ~semi | fix
    A[:, ident] = 0.0
    A[0, ident] = 1.0
    rhs[ident] = np.where(semi[ident], 1.0, 0.0)
    sc[ident] = np.where(semi[ident], car[ident], 0.0)
    dsc[ident] = 0.0
    return A, rhs, sc, dsc


def cont_update(dev, hole, sol, sc, lo, hi):
    """u -> carrier and quasi-Fermi potential, weighted max |dq| (semiconductor_3d.c:3112-3146).
    Returns (qf_new, car_new, dq, dmax); other carrier taken from dev."""
    semi = dev["kind"] == K_SEMI
    act = semi & ~car_fix(dev)
    u = np.where(~(sol > 1e-30), 1e-30, np.minimum(sol, 1e30))
    c = sc * u
    VT = matp(dev, "VT")
    with np.errstate(divide="ignore", invalid="ignore"):
        if hole:
            qn = dev["phi"] + VT * (np.log(c) - lnvK(dev))
        else:
            qn = dev["phi"] - VT * (np.log(c) - lncK(dev))
    qn = np.clip(qn, lo, hi)
    qf_old = dev["phip"] if hole else dev["phin"]
    ch = qn - qf_old
    cn = pK(dev, dev["phi"], qn) if hole else nK(dev, dev["phi"], qn)
    qf = np.where(act, qn, qf_old)
    car = np.where(act, cn, dev["p"] if hole else dev["n"])
    dq = np.where(act, ch, 0.0)
    nn = dev["n"] if hole else car
    pp = car if hole else dev["p"]
    scale = nn + pp + np.abs(dev["Nd"] - dev["Na"])
    with np.errstate(divide="ignore", invalid="ignore"):
        r = np.where(scale > 0, cn / scale, 0.0)
    wgt = np.where(r >= 1e-3, 1.0, r * 1e3)
    a = np.where(act & (r > 1e-6), wgt * np.abs(ch), 0.0)
    return qf, car, dq, float(a.max() if a.size else 0.0)


def terminal_currents(dev, ncon, g=None):
    """Contact fluxes I, scales S and electron parts In (semiconductor_3d.c:2843-2854,
    3598-3623)."""
    g = g or Grid(dev)
    N = g.N
    kind, con = dev["kind"], dev["con"]
    semi = kind == K_SEMI
    I = np.zeros(ncon)
    S = np.zeros(ncon)
    In = np.zeros(ncon)
    VT = matp(dev, "VT")
    lc, lv = lncK(dev), lnvK(dev)
    for d in range(6):
        v, kb, h, ar = g.valid[d], g.kb[d], g.h[d], g.ar[d]
        ok = (con != 0) & semi & v & semi[kb] & (con[kb] != con)
        if not ok.any():
            continue
        k = np.nonzero(ok)[0]
        b = kb[k]
        dps = (dev["phi"][b] - dev["phi"][k]) / VT[k]
        Dn = dps + (lc[b] - lc[k])
        Dp = dps - (lv[b] - lv[k])
        kl = np.minimum(k, b)
        gn = Q * ar[k] * dev["fmu"][d // 2][kl] * VT[k] / h[k]
        gp = Q * ar[k] * dev["fmu"][3 + d // 2][kl] * VT[k] / h[k]
        a1 = gn * dev["n"][b] * bernoulli(Dn)
        a2 = gn * dev["n"][k] * bernoulli(-Dn)
        b1 = gp * dev["p"][k] * bernoulli(Dp)
        b2 = gp * dev["p"][b] * bernoulli(-Dp)
        c = con[k] - 1
        np.add.at(I, c, (a1 - a2) + (b1 - b2))
        np.add.at(S, c, (a1 + a2) + (b1 + b2))
        np.add.at(In, c, a1 - a2)
    return I, S, In


# ------------------------------------------------------------------ linear algebra
def matvec(A, dims, x):
    """7-point stencil product (semiconductor_3d.c:1975-1993)."""
    Nx, Ny, Nz = dims
    X = x.reshape(Nz, Ny, Nx)
    Y = (A[0] * x).reshape(Nz, Ny, Nx).copy()
    C = [a.reshape(Nz, Ny, Nx) for a in A]
    Y[:, :, 1:] += C[1][:, :, 1:] * X[:, :, :-1]
    Y[:, :, :-1] += C[2][:, :, :-1] * X[:, :, 1:]
    Y[:, 1:, :] += C[3][:, 1:, :] * X[:, :-1, :]
    Y[:, :-1, :] += C[4][:, :-1, :] * X[:, 1:, :]
    Y[1:, :, :] += C[5][1:, :, :] * X[:-1, :, :]
    Y[:-1, :, :] += C[6][:-1, :, :] * X[1:, :, :]
    return Y.ravel()


def bicg_floor(A, dims, b, x):
    """sqrt(sum_a (sum_b |A_ab x_b| + |b_a|)^2) (semiconductor_3d.c:2244-2268)."""
    absA = [np.abs(a) for a in A]
    s = matvec(absA, dims, np.abs(x)) + np.abs(b)
    return float(np.sqrt(np.sum(s * s)))


def mg_dims(dims):
    """Level shapes and coarsening flags of the 2x2x2 aggregation (semiconductor_3d.c:1894-1921)."""
    levs = [(tuple(int(v) for v in dims), None)]
    while len(levs) < 24:
        (Nx, Ny, Nz), _ = levs[-1]
        if Nx * Ny * Nz <= 64:
            break
        cx, cy, cz = Nx > 2, Ny > 2, Nz > 2
        if not (cx or cy or cz):
            break
        levs[-1] = ((Nx, Ny, Nz), (cx, cy, cz))
        levs.append((((Nx + 1) // 2 if cx else Nx, (Ny + 1) // 2 if cy else Ny,
                      (Nz + 1) // 2 if cz else Nz), None))
    return levs


def _parent(dims, cflags):
    """Coarse index of every fine node (2x2x2 aggregates)."""
    Nx, Ny, Nz = dims
    cx, cy, cz = cflags
    Cx = (Nx + 1) // 2 if cx else Nx
    Cy = (Ny + 1) // 2 if cy else Ny
    l, j, i = np.meshgrid(np.arange(Nz), np.arange(Ny), np.arange(Nx), indexing="ij")
    I = i >> 1 if cx else i
    J = j >> 1 if cy else j
    L = l >> 1 if cz else l
    return (I + Cx * (J + Cy * L)).ravel()


def mg_weights(levs, ph0):
    """Slotboom prolongation weights (semiconductor_3d.c:2092-2117). ph0: level-0
    reference potential per node in units of VT (PH_NONE where none), or None for
    plain aggregation.  Returns the list of pw per fine level."""
    pws = []
    ph = ph0
    for L in range(len(levs) - 1):
        dims, cf = levs[L]
        N = int(np.prod(dims))
        if ph0 is None:
            pws.append(np.ones(N))
            continue
        par = _parent(dims, cf)
        Nc = int(np.prod(levs[L + 1][0]))
        mx = np.full(Nc, PH_NONE)
        np.maximum.at(mx, par, ph)
        e = np.where(ph <= 0.5 * PH_NONE, -800.0, ph - mx[par])
        pws.append(np.where(e < -700.0, 0.0, np.exp(np.maximum(e, -700.0))))
        ph = mx
    return pws


def galerkin(A, dims, cf, pw, w=None):
    """Coarse 7-point operator P^T W A P (semiconductor_3d.c:2003-2027)."""
    Nx, Ny, Nz = dims
    N = Nx * Ny * Nz
    par = _parent(dims, cf)
    cx, cy, cz = cf
    Cdims = ((Nx + 1) // 2 if cx else Nx, (Ny + 1) // 2 if cy else Ny, (Nz + 1) // 2 if cz else Nz)
    Nc = int(np.prod(Cdims))
    wk = np.ones(N) if w is None else w
    l, j, i = np.meshgrid(np.arange(Nz), np.arange(Ny), np.arange(Nx), indexing="ij")
    i, j, l = i.ravel(), j.ravel(), l.ravel()
    k = np.arange(N)
    Ac = np.zeros((7, Nc))
    np.add.at(Ac[0], par, wk * A[0] * pw)
    strides = (1, Nx, Nx * Ny)
    idxs = (i, j, l)
    ns = (Nx, Ny, Nz)
    for d in range(6):
        ax, up = d // 2, d % 2
        v = idxs[ax] < ns[ax] - 1 if up else idxs[ax] > 0
        kb = np.where(v, k + strides[ax] if up else k - strides[ax], k)
        a = np.where(v, wk * A[1 + d] * pw[kb], 0.0)
        same = par[kb] == par
        np.add.at(Ac[0], par, np.where(v & same, a, 0.0))
        np.add.at(Ac[1 + d], par, np.where(v & ~same, a, 0.0))
    zero = np.all(Ac == 0.0, axis=0)
    Ac[0, zero] = 1.0
    return Ac, Cdims


def restrict(dims, cf, r, w=None):
    """Aggregate sums (semiconductor_3d.c:2028-2037)."""
    par = _parent(dims, cf)
    Nx, Ny, Nz = dims
    cx, cy, cz = cf
    Nc = ((Nx + 1) // 2 if cx else Nx) * ((Ny + 1) // 2 if cy else Ny) * ((Nz + 1) // 2 if cz else Nz)
    out = np.zeros(Nc)
    np.add.at(out, par, r if w is None else w * r)
    return out


def prolong_add(dims, cf, pw, xc, x, alpha=1.0):
    """x += alpha pw P xc (semiconductor_3d.c:2038-2048)."""
    return x + alpha * pw * xc[_parent(dims, cf)]


def ph0(dev, qsign):
    """Level-0 reference potential / VT of the Slotboom weights (semiconductor_3d.c:2085-2090)."""
    if qsign == 0:
        return None
    VT = dev["mats"][dev["ref_mat"], MF["VT"]]
    val = dev["phin"] / VT if qsign > 0 else -dev["phip"] / VT
    none = (dev["kind"] != K_SEMI) | car_fix(dev)
    return np.where(none, PH_NONE, val)


# ------------------------------------------------------------------ general (graph) meshes
def graph_rows(dev):
    """Row index of every directed edge of the CSR graph."""
    return np.repeat(np.arange(len(dev["g_rp"]) - 1), np.diff(dev["g_rp"]))


def poisson_eval_g(dev, phi):
    """F, diagonal, off-diagonals per directed edge, sc and ||F/sc|| of the Poisson system on
    a graph (poisson_core_g, semiconductor_3d.c:4181-4217, with the Robin gates of
    poisson_eval, :2732-2789).  Edge terms are summed row by row in CSR order."""
    rp, cj, h, ar = dev["g_rp"], dev["g_cj"], dev["g_h"], dev["g_ar"]
    N = len(rp) - 1
    row = graph_rows(dev)
    kind, con = dev["kind"], dev["con"]
    isdir = con != 0
    eps = matp(dev, "eps_r") * EPS0
    ek, eb = eps[row], eps[cj]
    cf = (2.0 * ek * eb / (ek + eb)) * ar / h
    F = np.zeros(N)
    dg = np.zeros(N)
    for k in range(N):                               # CSR order within a row, as the reference sums
        acc = 0.0
        d = 0.0
        for e in range(rp[k], rp[k + 1]):
            acc += cf[e] * (phi[cj[e]] - phi[k])
            d += cf[e]
        F[k] = acc
        dg[k] = d
    gval = np.where(isdir[cj], 0.0, -cf)
    vol = dev["g_vol"]
    semi = kind == K_SEMI
    n = nK(dev, phi, dev["phin"])
    p = pK(dev, phi, dev["phip"])
    VT = matp(dev, "VT")
    Np, dNp, Nm, dNm = ion_eval(dev, n, p)
    F += np.where(semi, vol * Q * (p - n + Np - Nm + dev["Nf"]), vol * Q * dev["Nf"])
    dg += np.where(semi, vol * Q * ((n + p) / VT - dNp + dNm), 0.0)
    sc = dg.copy()
    F[isdir] = 0.0
    dg[isdir] = 1.0
    sc[isdir] = 1.0
    gval[isdir[row]] = 0.0
    for r in range(len(dev["rob_k"])):
        k, c = int(dev["rob_k"][r]), int(dev["rob_c"][r])
        tox = dev["con_tox"][c] if dev["con_tox"][c] > 0 else 10e-9
        Cox = EPS_OX / tox
        pm = dev["con_pm"][c] if dev["con_pm"][c] > 0 else dev["Cref"]
        VG = dev["con_V"][c] + dev["Cref"] - pm
        F[k] += dev["rob_A"][r] * (Cox * (VG - phi[k]) + dev["con_qox"][c])
        dg[k] += Cox * dev["rob_A"][r]
        sc[k] = dg[k]
    return F, dg, gval, sc, float(np.sqrt(np.sum((F / sc) ** 2)))


def upd_mob_g(dev):
    """Edge mobilities per undirected edge (upd_mob_ref_g, semiconductor_3d.c:4241-4293):
    the mean of the node low-field mobilities projected on the edge for a hexagonal crystal,
    velocity saturation with the harmonic-mean driving field (models bit 2); no surface
    model or metal contacts in scope here."""
    rp, cj, ue, h = dev["g_rp"], dev["g_cj"], dev["g_ue"], dev["g_h"]
    row = graph_rows(dev)
    semi = dev["kind"] == K_SEMI
    nue = int(ue.max()) + 1 if len(ue) else 0
    mun, mup = np.zeros(nue), np.zeros(nue)
    up = cj > row                                    # each undirected edge once, from its lower node
    k, kp, e_ue, hh = row[up], cj[up], ue[up], h[up]
    mn = 0.5 * (dev["mun"][k] + dev["mun"][kp])
    mp = 0.5 * (dev["mup"][k] + dev["mup"][kp])
    pos = dev["g_pos"].reshape(-1, 3)
    ax = int(dev["caxis"])
    for which, mu in (("ani_n", mn), ("ani_p", mp)):
        a = matp(dev, which)[k]
        if ax >= 0:
            dv = pos[kp] - pos[k]
            L2 = np.sum(dv * dv, axis=1)
            f = np.where((a > 0) & (a != 1.0) & (L2 > 0), 1.0 + (a - 1.0) * dv[:, ax] ** 2 / np.where(L2 > 0, L2, 1.0), 1.0)
            mu *= f
    if dev["models"] & 4:
        dps = dev["phi"][kp] - dev["phi"][k]
        Fn = heat_field(dev["phin"][kp] - dev["phin"][k], dps, hh)
        Fp = heat_field(dev["phip"][kp] - dev["phip"][k], dps, hh)
        sn = mob_hf(mn, Fn, matp(dev, "vsat_n")[k], matp(dev, "beta_n")[k])
        sp = mob_hf(mp, Fp, matp(dev, "vsat_p")[k], matp(dev, "beta_p")[k])
        mn = mn + 1.0 * (sn - mn)
        mp = mp + 1.0 * (sp - mp)
    ok = semi[k] & semi[kp]
    mun[e_ue] = np.where(ok, mn, 0.0)
    mup[e_ue] = np.where(ok, mp, 0.0)
    return mun, mup


def cont_assemble_g(dev, hole, gmu_n, gmu_p):
    """Scaled Scharfetter-Gummel system for u = c/s on a graph: diagonal, off-diagonals per
    directed edge, rhs, sc, dsc (cont_assemble_g, semiconductor_3d.c:4314-4351)."""
    rp, cj, ue, h, ar = dev["g_rp"], dev["g_cj"], dev["g_ue"], dev["g_h"], dev["g_ar"]
    N = len(rp) - 1
    row = graph_rows(dev)
    semi = dev["kind"] == K_SEMI
    fix = car_fix(dev)
    car = dev["p"] if hole else dev["n"]
    VT = matp(dev, "VT")
    lc = lnvK(dev) if hole else lncK(dev)
    mu = gmu_p if hole else gmu_n
    ok = semi[row] & semi[cj]
    dl = lc[cj] - lc[row]
    D = (dev["phi"][cj] - dev["phi"][row]) / VT[row] + (-dl if hole else dl)
    g = ar * mu[ue] * VT[row] / h
    self_ = g * (bernoulli(D) if hole else bernoulli(-D))
    nb = g * (bernoulli(-D) if hole else bernoulli(D))
    gval = np.where(ok & ~fix[cj], -nb * np.maximum(car[cj], NFLOOR), 0.0)
    dg = np.zeros(N)
    b = np.zeros(N)
    for k in range(N):                               # CSR order within a row
        d = 0.0
        bb = 0.0
        for e in range(rp[k], rp[k + 1]):
            if not ok[e]:
                continue
            d += self_[e]
            if fix[cj[e]]:
                bb += nb[e] * car[cj[e]]
        dg[k] = d
        b[k] = bb
    R, dRn, dRp = recomb(dev, dev["n"], dev["p"])
    dR = np.maximum(dRp if hole else dRn, 0.0)
    vol = dev["g_vol"]
    dg += vol * dR
    b += vol * (dR * car - R)
    sk = np.maximum(car, NFLOOR)
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        w = 1.0 / (dg * sk)
    gval = gval * w[row]
    rhs = b * w
    diag = np.ones(N)
    sc = sk.copy()
    dsc = dg * sk
    ident = ~semi | fix
    gval[ident[row]] = 0.0
    rhs[ident] = np.where(semi[ident], 1.0, 0.0)
    sc[ident] = np.where(semi[ident], car[ident], 0.0)
    dsc[ident] = 0.0
    return diag, gval, rhs, sc, dsc


def terminal_currents_g(dev, ncon, gmu_n, gmu_p):
    """Contact fluxes I, scales S and electron parts In on a graph: the Scharfetter-Gummel
    flux of every edge from a contact's semiconductor node to a semiconductor node outside
    that contact (terminal_flux_g and face_flux_g, semiconductor_3d.c:4219-4229, 4414-4426;
    no metal contacts in scope), summed per contact in CSR order."""
    cj, ue, h, ar = dev["g_cj"], dev["g_ue"], dev["g_h"], dev["g_ar"]
    row = graph_rows(dev)
    con = dev["con"]
    semi = dev["kind"] == K_SEMI
    ok = (con[row] != 0) & semi[row] & semi[cj] & (con[cj] != con[row])
    I, S, In = np.zeros(ncon), np.zeros(ncon), np.zeros(ncon)
    e = np.nonzero(ok)[0]
    ka, kb = row[e], cj[e]
    VT = matp(dev, "VT")[ka]
    lc, lv = lncK(dev), lnvK(dev)
    dps = (dev["phi"][kb] - dev["phi"][ka]) / VT
    Dn = dps + (lc[kb] - lc[ka])
    Dp = dps - (lv[kb] - lv[ka])
    gn = Q * ar[e] * gmu_n[ue[e]] * VT / h[e]
    gp = Q * ar[e] * gmu_p[ue[e]] * VT / h[e]
    a1 = gn * dev["n"][kb] * bernoulli(Dn)
    a2 = gn * dev["n"][ka] * bernoulli(-Dn)
    b1 = gp * dev["p"][ka] * bernoulli(Dp)
    b2 = gp * dev["p"][kb] * bernoulli(-Dp)
    c = con[ka] - 1
    np.add.at(I, c, (a1 - a2) + (b1 - b2))
    np.add.at(S, c, (a1 + a2) + (b1 + b2))
    np.add.at(In, c, a1 - a2)
    return I, S, In


def gmg_weights_g(levels, ph0):
    """Slotboom prolongation weights of every graph level towards the next (g_weights,
    semiconductor_3d.c:2621-2642): per aggregate the largest reference potential of its
    members (ph, in units of VT; PH_NONE for contact and non-semiconductor nodes), and
    pw = exp(ph - max) per member (0 below e^-700).  levels[L] holds "agg" (the aggregate
    of every node of level L) for L below the coarsest; ph0 is level 0's potential.
    Returns pw per level below the coarsest."""
    PH_NONE = -1e300
    pws = []
    ph = np.asarray(ph0, float)
    for L in range(len(levels) - 1):
        agg = levels[L]["agg"]
        na = int(agg.max()) + 1
        mx = np.full(na, PH_NONE)
        np.maximum.at(mx, agg, ph)
        e = np.where(ph <= 0.5 * PH_NONE, -800.0, ph - mx[agg])
        with np.errstate(over="ignore", invalid="ignore"):
            pw = np.where(e < -700.0, 0.0, np.exp(np.maximum(e, -745.0)))
        pws.append(pw)
        ph = mx
    return pws


def galerkin_g(rp, cj, va, dg, agg, crp, ccj, pw, w=None):
    """Coarse operator of a graph level (g_galerkin, semiconductor_3d.c:2575-2594): row I of
    the coarse level sums, over the aggregate's members i in ascending order and their
    entries in CSR order, w_i a_ij pw_j into the coarse entry (I, agg[j]) (into the
    diagonal when agg[j] == I), plus w_i a_ii pw_i; a row with nothing but zeros becomes an
    identity row.  Returns the coarse couplings in the coarse CSR order and the diagonal."""
    nc = len(crp) - 1
    cva = np.zeros(len(ccj))
    cdg = np.zeros(nc)
    pos = {}
    for I in range(nc):
        for s in range(crp[I], crp[I + 1]):
            pos[(I, int(ccj[s]))] = s
    members = [[] for _ in range(nc)]
    for i in range(len(agg)):
        members[int(agg[i])].append(i)
    for I in range(nc):
        cc = 0.0
        for i in members[I]:
            wi = 1.0 if w is None else w[i]
            cc += wi * dg[i] * pw[i]
            for e in range(rp[i], rp[i + 1]):
                a = wi * va[e] * pw[cj[e]]
                J = int(agg[cj[e]])
                if J == I:
                    cc += a
                else:
                    cva[pos[(I, J)]] += a
        zero = cc == 0.0 and not np.any(cva[crp[I]:crp[I + 1]] != 0.0)
        cdg[I] = 1.0 if zero else cc
    return cva, cdg


def neighbours_tensor(dev, g=None):
    """Per node, its neighbours in the reference's direction order with area / length and
    the face mobilities of the edge (nbr() and fmu, semiconductor_3d.c:709-719, 256)."""
    g = g or Grid(dev)
    out = [[] for _ in range(g.N)]
    for d in range(6):
        for k in np.nonzero(g.valid[d])[0]:
            kb = int(g.kb[d][k])
            kl = min(int(k), kb)
            out[k].append((kb, g.ar[d][k] / g.h[d][k], dev["fmu"][d // 2][kl], dev["fmu"][3 + d // 2][kl]))
    return out, g.vol


def neighbours_graph(dev, gmu_n, gmu_p):
    """Per node, its graph neighbours in CSR order with dual area / length and the edge
    mobilities."""
    rp, cj, ue, h, ar = dev["g_rp"], dev["g_cj"], dev["g_ue"], dev["g_h"], dev["g_ar"]
    out = [[(int(cj[e]), ar[e] / h[e], gmu_n[ue[e]], gmu_p[ue[e]]) for e in range(rp[k], rp[k + 1])]
           for k in range(len(rp) - 1)]
    return out, dev["g_vol"]


def float_fix(dev, hole, sol, sc, nbrs, vol):
    """Balance of every floating majority block (float_fix / float_fix_g,
    semiconductor_3d.c:3159-3228, 4353-4412; no incomplete ionisation, traps or exchange
    terms in scope).  A block is a breadth-first set of majority, quasi-neutral
    semiconductor nodes (c = s u >= the other carrier, c and s >= |Nd - Na| / 2, c > 10 n_i)
    found in node order; a block touching a contact is anchored.  Otherwise u is scaled by
    lambda solving lambda Aout - Bin + sum vol R(lambda c) = 0 (Newton in ln lambda, steps
    clipped to +-2, 60 at most).  Returns (blocks fixed, u)."""
    N = len(sol)
    u = np.array(sol, float)
    s = np.asarray(sc, float)
    semi = dev["kind"] == K_SEMI
    con = dev["con"]
    car = dev["p"] if hole else dev["n"]
    oth = dev["n"] if hole else dev["p"]
    dnet = np.abs(dev["Nd"] - dev["Na"])
    ni = niK(dev)
    VT = matp(dev, "VT")
    lc, lv = lncK(dev), lnvK(dev)

    def maj(k):
        c = s[k] * u[k]
        return (semi[k] and not con[k] and c >= oth[k] and c >= 0.5 * dnet[k] and s[k] >= 0.5 * dnet[k]
                and c > 10.0 * ni[k])
    lab = np.zeros(N, int)
    nfix = blk = 0
    for k0 in range(N):
        if lab[k0] or not maj(k0):
            continue
        blk += 1
        q = [k0]
        lab[k0] = blk
        anch = False
        head = 0
        while head < len(q):
            k = q[head]
            head += 1
            for kb, _, _, _ in nbrs[k]:
                if not semi[kb]:
                    continue
                if con[kb]:
                    anch = True
                    continue
                if not lab[kb] and maj(kb):
                    lab[kb] = blk
                    q.append(kb)
        if anch:
            continue
        Aout = Bin = 0.0
        for k in q:
            for kb, arh, mn, mp in nbrs[k]:
                if not semi[kb] or lab[kb] == blk:
                    continue
                D = (dev["phi"][kb] - dev["phi"][k]) / VT[k] + (-(lv[kb] - lv[k]) if hole else (lc[kb] - lc[k]))
                gg = arh * (mp if hole else mn) * VT[k]
                Bp, Bm = bernoulli(np.array([D, -D]))
                self_, nb = (gg * Bp, gg * Bm) if hole else (gg * Bm, gg * Bp)
                cb = car[kb] if con[kb] else s[kb] * u[kb]
                Aout += self_ * s[k] * u[k]
                Bin += nb * cb
        qa = np.array(q)
        sl = 0.0
        for _ in range(60):
            lam = np.exp(sl)
            G, dG = lam * Aout - Bin, lam * Aout
            c = lam * s[qa] * u[qa]
            nn, pp = dev["n"].copy(), dev["p"].copy()
            if hole:
                pp[qa] = c
            else:
                nn[qa] = c
            R, dRn, dRp = recomb(dev, nn, pp)
            for t, k in enumerate(q):
                G += vol[k] * R[k]
                dG += vol[k] * (dRp[k] if hole else dRn[k]) * c[t]
            if not dG > 0.0:
                break
            ds = min(max(-G / dG, -2.0), 2.0)
            sl += ds
            if abs(ds) < 1e-13:
                break
        if sl == sl and 1e-15 < abs(sl) < 200.0:
            u[qa] *= np.exp(sl)
            nfix += 1
    return nfix, u


def graph_lsq(dev):
    """Inverse least-squares matrices M^-1 of every semiconductor node (g_lsq_setup,
    semiconductor_3d.c:2682-2700): M = sum over semiconductor neighbours w dr dr^T,
    w = 1 / |dr|^2, regularised by 1e-6 of its trace; symmetric, stored xx xy xz yy yz zz."""
    rp, cj = dev["g_rp"], dev["g_cj"]
    pos = dev["g_pos"].reshape(-1, 3)
    semi = dev["kind"] == K_SEMI
    N = len(rp) - 1
    out = np.zeros((N, 6))
    for k in range(N):
        if not semi[k]:
            continue
        m = np.zeros(6)
        for e in range(rp[k], rp[k + 1]):
            b = cj[e]
            if not semi[b]:
                continue
            dx, dy, dz = pos[b] - pos[k]
            w = 1.0 / (dx * dx + dy * dy + dz * dz + 1e-40)
            m += w * np.array([dx * dx, dx * dy, dx * dz, dy * dy, dy * dz, dz * dz])
        eps = 1e-6 * (m[0] + m[3] + m[5]) + 1e-30
        M = np.array([[m[0] + eps, m[1], m[2]], [m[1], m[3] + eps, m[4]], [m[2], m[4], m[5] + eps]])
        if abs(np.linalg.det(M)) > 0:
            Mi = np.linalg.inv(M)
            out[k] = [Mi[0, 0], Mi[0, 1], Mi[0, 2], Mi[1, 1], Mi[1, 2], Mi[2, 2]]
    return out


def graph_grad(dev, fld, lsq):
    """Least-squares gradient of a node field over the semiconductor neighbours (g_grad,
    semiconductor_3d.c:2702-2714)."""
    rp, cj = dev["g_rp"], dev["g_cj"]
    pos = dev["g_pos"].reshape(-1, 3)
    semi = dev["kind"] == K_SEMI
    N = len(rp) - 1
    g = np.zeros((N, 3))
    for k in range(N):
        if not semi[k]:
            continue
        r = np.zeros(3)
        for e in range(rp[k], rp[k + 1]):
            b = cj[e]
            if not semi[b]:
                continue
            d = pos[b] - pos[k]
            r += (fld[b] - fld[k]) / (d @ d + 1e-40) * d
        m = lsq[k]
        g[k] = [m[0] * r[0] + m[1] * r[1] + m[2] * r[2], m[1] * r[0] + m[3] * r[1] + m[4] * r[2],
                m[2] * r[0] + m[4] * r[1] + m[5] * r[2]]
    return g


def graph_node_J(dev, gmu_n, gmu_p, which=0):
    """Node current density by least squares from the edge fluxes (g_node_J,
    semiconductor_3d.c:4428-4452): J = (sum_e A_e t t^T)^-1 sum_e A_e t j_e over the
    semiconductor neighbours, t the unit edge vector, j_e the flux density; which 0 total,
    1 electrons, 2 holes."""
    rp, cj, ue, h, ar = dev["g_rp"], dev["g_cj"], dev["g_ue"], dev["g_h"], dev["g_ar"]
    pos = dev["g_pos"].reshape(-1, 3)
    semi = dev["kind"] == K_SEMI
    N = len(rp) - 1
    VT = matp(dev, "VT")
    lc, lv = lncK(dev), lnvK(dev)
    J = np.zeros((N, 3))
    for k in range(N):
        if not semi[k]:
            continue
        M = [0.0] * 6                                # xx xy xz yy yz zz, summed as the reference
        r = [0.0, 0.0, 0.0]
        for e in range(rp[k], rp[k + 1]):
            b = cj[e]
            if not semi[b]:
                continue
            t = (pos[b] - pos[k]) / h[e]
            dps = (dev["phi"][b] - dev["phi"][k]) / VT[k]
            Dn, Dp = dps + (lc[b] - lc[k]), dps - (lv[b] - lv[k])
            gn, gp = Q * ar[e] * gmu_n[ue[e]] * VT[k] / h[e], Q * ar[e] * gmu_p[ue[e]] * VT[k] / h[e]
            Bn = bernoulli(np.array([Dn, -Dn]))
            Bp = bernoulli(np.array([Dp, -Dp]))
            Jn = gn * dev["n"][b] * Bn[0] - gn * dev["n"][k] * Bn[1]
            Jp = gp * dev["p"][k] * Bp[0] - gp * dev["p"][b] * Bp[1]
            j = (Jn if which == 1 else (Jp if which == 2 else Jn + Jp)) / (ar[e] if ar[e] > 0 else 1e-300)
            w = ar[e]
            M[0] += w * t[0] * t[0]; M[1] += w * t[0] * t[1]; M[2] += w * t[0] * t[2]
            M[3] += w * t[1] * t[1]; M[4] += w * t[1] * t[2]; M[5] += w * t[2] * t[2]
            r[0] += w * t[0] * j; r[1] += w * t[1] * j; r[2] += w * t[2] * j
        eps = 1e-6 * (M[0] + M[3] + M[5]) + 1e-300
        a, b, c, dd, ee, f = M[0] + eps, M[1], M[2], M[3] + eps, M[4], M[5] + eps
        A, Bq, Cc = dd * f - ee * ee, -(b * f - c * ee), b * ee - c * dd           # cofactors
        Dq, E, F = a * f - c * c, -(a * ee - b * c), a * dd - b * b
        det = a * A + b * Bq + c * Cc
        if abs(det) > 0:
            J[k] = [(A * r[0] + Bq * r[1] + Cc * r[2]) / det, (Bq * r[0] + Dq * r[1] + E * r[2]) / det,
                    (Cc * r[0] + E * r[1] + F * r[2]) / det]
    return J


def ii_alpha(dev, F, c):
    """Impact-ionisation coefficient of carrier c (0 electrons, 1 holes) at field F, per node
    (ii_alpha, semiconductor_3d.c:4478-4485): g a exp(-(g b / F)^m) with (a, b) below / above
    E0, nothing below 1e5 V/m or beyond an exponent of 700."""
    F = np.asarray(F, float)
    g = matp(dev, "ii_g")
    E0 = matp(dev, f"ii_E0{c}")
    hi = F >= E0
    a = np.where(hi, matp(dev, f"ii_a{c}1"), matp(dev, f"ii_a{c}0"))
    b = np.where(hi, matp(dev, f"ii_b{c}1"), matp(dev, f"ii_b{c}0"))
    m = matp(dev, f"ii_m{c}")
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        x = g * b / F
        x = np.where(m != 1.0, x ** m, x)
        out = np.where((F > 1e5) & (x <= 700.0), g * a * np.exp(-np.minimum(x, 700.0)), 0.0)
    return out


def graph_ii(dev, gmu_n, gmu_p):
    """Impact-ionisation pair generation of every node on a graph (ii_update,
    semiconductor_3d.c:4486-4523): G = sum over carriers alpha(F) |J| / q over the control
    volume, J the carrier's least-squares node current density, F = |E.J| / |J| with E the
    least-squares field; contact nodes and materials without data generate nothing."""
    Jn = graph_node_J(dev, gmu_n, gmu_p, 1)
    Jp = graph_node_J(dev, gmu_n, gmu_p, 2)
    E = -graph_grad(dev, dev["phi"], graph_lsq(dev))
    G = np.zeros(len(E))
    for c, J in ((0, Jn), (1, Jp)):
        jj = np.sqrt(np.sum(J * J, axis=1))
        with np.errstate(divide="ignore", invalid="ignore"):
            F = np.where(jj > 0, np.abs(np.sum(E * J, axis=1)) / np.where(jj > 0, jj, 1.0), 0.0)
        G += np.where(jj > 0, ii_alpha(dev, F, c) * jj, 0.0)
    on = (dev["kind"] == K_SEMI) & (dev["con"] == 0) & (matp(dev, "ii_on") != 0)
    return np.where(on, G / Q * dev["g_vol"], 0.0)
