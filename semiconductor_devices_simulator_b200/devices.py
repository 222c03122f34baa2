"""Synthetic device builders for the benchmark and parity workloads.

Every builder drives a library through the ``api3_*`` ABI only (the calls main.py's
``setup_device`` makes, main.py:3286-3361), so the same builder sets up the B200 solver
library and the reference core identically.  Sizes, doping and biases follow the
workload definitions:

* ``pn_diode``   Si abrupt pn diode, 1x1x1 um, uniform tensor mesh (40^3 by default),
                 N_A 1e17 cm^-3 for x < 0.5 um, N_D 1e17 cm^-3 for x >= 0.5 um, 300 K,
                 constant mobility 1350 / 480 cm^2/Vs, tau_n = tau_p = 1e-7 s, ohmic
                 contacts on x = 0 (anode) and x = L (cathode), models = 0.
* ``nmosfet``    n-MOSFET on a 120x80x60 mesh: p-body 1e17 cm^-3, Gaussian n+ source /
                 drain (peak 1e20 cm^-3, sigma 20 nm), 2 nm SiO2 gate oxide as the oxide
                 Robin condition of a face gate (tox = 2 nm, eps_r 3.9), velocity
                 saturation (models = 4), Id-Vg sweep 0..1.2 V in 0.05 V steps at
                 Vd = 0.05 V and 1.0 V.
* ``diode_variant``  the batched pn-diode family: node counts between 32^3 and 72^3,
                 doping log-uniform in [1e15, 1e18] cm^-3, junction depth in
                 [0.2, 0.8] um, from a recorded seed.

Concentrations are given in cm^-3 and converted to m^-3 at the ABI, as main.py does.
"""
import ctypes
import numpy as np

from .abi import dptr, iptr

SI, SIC, SIO2 = 0, 4, 8             # material ids of semiconductor_3d.c:431, :513, :600
GUI_SOLVER = (2000, 1000, 500, 1e-8, 1e-6, 1.0, 1.0)   # main.py:3286 default tuple


class Workload:
    """What a builder set up: mesh shape, contact ids and the bias sweep(s)."""

    def __init__(self, name, shape, contacts, sweeps, info=None):
        self.name = name
        self.shape = tuple(shape)                # (Nx, Ny, Nz)
        self.contacts = dict(contacts)           # label -> contact id
        self.sweeps = sweeps                     # list of dicts: {"fixed": {label: V}, "swept": label, "V": array}
        self.info = dict(info or {})

    @property
    def N(self):
        return int(np.prod(self.shape))

    @property
    def points(self):
        return int(sum(len(s["V"]) for s in self.sweeps))


def _grid(lib, xs, ys, zs):
    xs, ys, zs = (np.ascontiguousarray(a, dtype=np.float64) for a in (xs, ys, zs))
    ok = lib.api3_set_grid_coords(len(xs), len(ys), len(zs), dptr(xs), dptr(ys), dptr(zs))
    if not ok:
        raise MemoryError("api3_set_grid_coords failed")
    return xs, ys, zs


def pn_diode(lib, n=(40, 40, 40), L=(1e-6, 1e-6, 1e-6), NA=1e17, ND=1e17, xj=0.5e-6,
             mobility=(1350.0, 480.0), tau=1e-7, models=0, solver=GUI_SOLVER, vmax=0.6,
             dv=0.05, material=None):
    """Abrupt pn diode (silicon unless `material` names another reference material id);
    the anode (x = 0, p side) is swept 0..vmax."""
    lib.api3_init()
    xs = np.linspace(0.0, L[0], n[0])
    ys = np.linspace(0.0, L[1], n[1])
    zs = np.linspace(0.0, L[2], n[2])
    _grid(lib, xs, ys, zs)
    lib.api3_set_solver(*solver)
    lib.api3_set_models(models)
    si = lib.api3_add_material(SI if material is None else material, 300.0)
    if mobility is not None:
        if not lib.api3_set_mat_mobility(si, mobility[0] * 1e-4, mobility[1] * 1e-4):
            raise RuntimeError("api3_set_mat_mobility failed")
    if tau is not None:
        lib.api3_set_mat_tau(si, tau, tau)
    ij = int(np.searchsorted(xs, xj, side="left"))          # first node with x >= xj
    lib.api3_set_region(0, 0, 0, ij - 1, n[1] - 1, n[2] - 1, si, 0.0, NA * 1e6)
    lib.api3_set_region(ij, 0, 0, n[0] - 1, n[1] - 1, n[2] - 1, si, ND * 1e6, 0.0)
    lib.api3_clear_contacts()
    ca = lib.api3_add_contact_ex(0, 0, n[1] - 1, 0, n[2] - 1, 0, 0, 0, 0.0, 0.0, 0.0, 0.0)
    cc = lib.api3_add_contact_ex(1, 0, n[1] - 1, 0, n[2] - 1, 0, 0, 0, 0.0, 0.0, 0.0, 0.0)
    npts = int(round(vmax / dv)) + 1
    V = np.round(np.linspace(0.0, vmax, npts), 12)
    return Workload("pn_diode", n, {"anode": ca, "cathode": cc},
                    [{"fixed": {"cathode": 0.0}, "swept": "anode", "V": V}],
                    {"NA_cm3": NA, "ND_cm3": ND, "xj_m": xj, "models": models, "L_m": L})


def schottky_diode(lib, n=(40, 3, 3), L=1e-6, ND=1e16, phi_m=4.8, models=7 | 64, h0=2e-9,
                   solver=GUI_SOLVER, V=None):
    """n-Si Schottky diode: a metal face contact (bc 1, work function phi_m eV) on x = 0
    over uniform donors ND (cm^-3), ohmic cathode on x = L, mesh graded from h0 at the
    metal; `models` 7 | 64 switches on thermionic emission with image-force lowering, | 128
    barrier tunnelling.  The metal (anode) is swept over V (default 0..0.4 V)."""
    lib.api3_init()
    xs = graded_axis(L, n[0], h0)
    ys = np.linspace(0.0, 0.2e-6, n[1])
    zs = np.linspace(0.0, 0.2e-6, n[2])
    _grid(lib, xs, ys, zs)
    lib.api3_set_solver(*solver)
    lib.api3_set_models(models)
    si = lib.api3_add_material(SI, 300.0)
    lib.api3_set_region(0, 0, 0, n[0] - 1, n[1] - 1, n[2] - 1, si, ND * 1e6, 0.0)
    lib.api3_clear_contacts()
    ca = lib.api3_add_contact_ex(0, 0, n[1] - 1, 0, n[2] - 1, 0, 0, 1, 0.0, phi_m, 0.0, 0.0)
    cc = lib.api3_add_contact_ex(1, 0, n[1] - 1, 0, n[2] - 1, 0, 0, 0, 0.0, 0.0, 0.0, 0.0)
    if V is None:
        V = np.round(np.linspace(0.0, 0.4, 9), 12)
    return Workload("schottky", n, {"anode": ca, "cathode": cc},
                    [{"fixed": {"cathode": 0.0}, "swept": "anode", "V": np.asarray(V, float)}],
                    {"ND_cm3": ND, "phi_m": phi_m, "models": models})


def fv_len(c):
    """Box-method cell lengths of a coordinate axis (half the distance to each neighbour)."""
    c = np.asarray(c, float)
    L = np.empty_like(c)
    L[0] = 0.5 * (c[1] - c[0])
    L[-1] = 0.5 * (c[-1] - c[-2])
    L[1:-1] = 0.5 * (c[2:] - c[:-2])
    return L


def tensor_graph(xs, ys, zs, diag=0.0):
    """A tensor mesh as a general box-method graph (api3_set_mesh_graph): node k = i + Nx (j +
    Ny l), edges to the six axis neighbours with their spacing and dual face area, control
    volumes Lx Ly Lz, positions.  diag > 0 adds the two diagonals of every x-y cell face pair
    (i, j) - (i+1, j+1) and (i+1, j) - (i, j+1) with a dual area of diag times the smaller
    axis face: a graph that is no tensor product, on which both solvers must still agree.
    Returns (rp, cj, h, ar, vol, pos) as numpy arrays."""
    Nx, Ny, Nz = len(xs), len(ys), len(zs)
    Lx, Ly, Lz = fv_len(xs), fv_len(ys), fv_len(zs)
    N = Nx * Ny * Nz
    nb = [[] for _ in range(N)]
    for l in range(Nz):
        for j in range(Ny):
            for i in range(Nx):
                k = i + Nx * (j + Ny * l)
                for di, dj, dl in ((-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)):
                    ii, jj, ll = i + di, j + dj, l + dl
                    if not (0 <= ii < Nx and 0 <= jj < Ny and 0 <= ll < Nz):
                        continue
                    kb = ii + Nx * (jj + Ny * ll)
                    if di:
                        h, a = abs(xs[ii] - xs[i]), Ly[j] * Lz[l]
                    elif dj:
                        h, a = abs(ys[jj] - ys[j]), Lx[i] * Lz[l]
                    else:
                        h, a = abs(zs[ll] - zs[l]), Lx[i] * Ly[j]
                    nb[k].append((kb, h, a))
                if diag > 0.0:
                    for di, dj in ((-1, -1), (1, 1), (-1, 1), (1, -1)):
                        ii, jj = i + di, j + dj
                        if not (0 <= ii < Nx and 0 <= jj < Ny):
                            continue
                        kb = ii + Nx * (jj + Ny * l)
                        h = float(np.hypot(xs[ii] - xs[i], ys[jj] - ys[j]))
                        a = diag * min(Ly[min(j, jj)], Lx[min(i, ii)]) * Lz[l]
                        nb[k].append((kb, h, a))
    rp = np.zeros(N + 1, np.int32)
    for k in range(N):
        rp[k + 1] = rp[k] + len(nb[k])
    cj = np.array([b for row in nb for b, _, _ in row], np.int32)
    h = np.array([x for row in nb for _, x, _ in row], float)
    ar = np.array([a for row in nb for _, _, a in row], float)
    vol = np.array([Lx[i] * Ly[j] * Lz[l] for l in range(Nz) for j in range(Ny) for i in range(Nx)])
    pos = np.array([[xs[i], ys[j], zs[l]] for l in range(Nz) for j in range(Ny) for i in range(Nx)]).ravel()
    return rp, cj, h, ar, vol, pos


def graph_pn_diode(lib, n=(12, 6, 5), L=(1e-6, 1e-6, 1e-6), NA=1e17, ND=1e17, xj=0.5e-6, models=7,
                   solver=GUI_SOLVER, vmax=0.6, dv=0.1, diag=0.0, graph=True, mobility=None, tau=None):
    """The abrupt Si pn diode on a general (graph) mesh built from its tensor mesh
    (tensor_graph, optional diagonal edges), contacts as node lists on the x = 0 and x = L
    planes with their face areas; graph=False sets up the same diode on the tensor grid."""
    lib.api3_init()
    xs = np.linspace(0.0, L[0], n[0]); ys = np.linspace(0.0, L[1], n[1]); zs = np.linspace(0.0, L[2], n[2])
    Nx, Ny, Nz = n
    N = Nx * Ny * Nz
    si = None
    if graph:
        rp, cj, h, ar, vol, pos = tensor_graph(xs, ys, zs, diag)
        si = lib.api3_add_material(SI, 300.0)
        if not lib.api3_set_mesh_graph(N, len(cj), iptr(rp), iptr(cj), dptr(h), dptr(ar), dptr(vol), dptr(pos)):
            raise RuntimeError("api3_set_mesh_graph rejected the graph")
    else:
        _grid(lib, xs, ys, zs)
        si = lib.api3_add_material(SI, 300.0)
    lib.api3_set_solver(*solver)
    lib.api3_set_models(models)
    if mobility is not None:
        if not lib.api3_set_mat_mobility(si, mobility[0] * 1e-4, mobility[1] * 1e-4):
            raise RuntimeError("api3_set_mat_mobility failed")
    if tau is not None:
        lib.api3_set_mat_tau(si, tau, tau)
    i = np.arange(N) % Nx
    x = xs[i]
    Nd = np.where(x >= xj, ND * 1e6, 0.0)
    Na = np.where(x < xj, NA * 1e6, 0.0)
    mat = np.full(N, si, np.int32)
    lib.api3_set_node_data(iptr(mat), dptr(np.ascontiguousarray(Nd)), dptr(np.ascontiguousarray(Na)), None)
    lib.api3_clear_contacts()
    ca = lib.api3_add_contact_ex(0, 0, Ny - 1, 0, Nz - 1, 0, 0, 0, 0.0, 0.0, 0.0, 0.0)
    cc = lib.api3_add_contact_ex(1, 0, Ny - 1, 0, Nz - 1, 0, 0, 0, 0.0, 0.0, 0.0, 0.0)
    if graph:
        Ly, Lz = fv_len(ys), fv_len(zs)
        k = np.arange(N)
        j, l = (k // Nx) % Ny, k // (Nx * Ny)
        for cid, plane in ((ca, 0), (cc, Nx - 1)):
            nodes = np.ascontiguousarray(k[i == plane], np.int32)
            areas = np.ascontiguousarray(Ly[j[i == plane]] * Lz[l[i == plane]])
            if not lib.api3_set_con_nodes(cid, len(nodes), iptr(nodes), dptr(areas)):
                raise RuntimeError("api3_set_con_nodes failed")
    npts = int(round(vmax / dv)) + 1
    V = np.round(np.linspace(0.0, vmax, npts), 12)
    return Workload("graph_pn_diode" if graph else "pn_diode", (N, 1, 1) if graph else n,
                    {"anode": ca, "cathode": cc}, [{"fixed": {"cathode": 0.0}, "swept": "anode", "V": V}],
                    {"models": models, "diag": diag, "pos": pos if graph else None})


def floating_base_pnp(lib, n=(24, 5, 4), graph=True, diag=0.0, solver=GUI_SOLVER):
    """A p+ n p+ bar (2 x 0.5 x 0.5 um, p+ 1e18 cm^-3, a 0.4 um n base of 1e17 cm^-3 in the
    middle, tau 1e-7 s) with ohmic contacts on the two p+ ends only: the n base is a
    floating majority block (float_fix).  On a general (graph) mesh built from its tensor
    mesh, or (graph=False) on the tensor mesh itself.  Anode swept 0..1 V."""
    lib.api3_init()
    xs = np.linspace(0, 2e-6, n[0]); ys = np.linspace(0, 0.5e-6, n[1]); zs = np.linspace(0, 0.5e-6, n[2])
    Nx, Ny, Nz = n
    N = Nx * Ny * Nz
    si = lib.api3_add_material(SI, 300.0)
    if graph:
        rp, cj, h, ar, vol, pos = tensor_graph(xs, ys, zs, diag)
        if not lib.api3_set_mesh_graph(N, len(cj), iptr(rp), iptr(cj), dptr(h), dptr(ar), dptr(vol), dptr(pos)):
            raise RuntimeError("api3_set_mesh_graph rejected the graph")
    else:
        _grid(lib, xs, ys, zs)
    lib.api3_set_solver(*solver)
    lib.api3_set_models(7)
    lib.api3_set_mat_tau(si, 1e-7, 1e-7)
    k = np.arange(N)
    i, j, l = k % Nx, (k // Nx) % Ny, k // (Nx * Ny)
    base = (xs[i] >= 0.8e-6) & (xs[i] <= 1.2e-6)
    Nd = np.ascontiguousarray(np.where(base, 1e17, 0.0) * 1e6)
    Na = np.ascontiguousarray(np.where(base, 0.0, 1e18) * 1e6)
    lib.api3_set_node_data(iptr(np.full(N, si, np.int32)), dptr(Nd), dptr(Na), None)
    lib.api3_clear_contacts()
    ca = lib.api3_add_contact_ex(0, 0, Ny - 1, 0, Nz - 1, 0, 0, 0, 0.0, 0.0, 0.0, 0.0)
    cc = lib.api3_add_contact_ex(1, 0, Ny - 1, 0, Nz - 1, 0, 0, 0, 0.0, 0.0, 0.0, 0.0)
    if graph:
        Ly, Lz = fv_len(ys), fv_len(zs)
        for cid, plane in ((ca, 0), (cc, Nx - 1)):
            sel = i == plane
            if not lib.api3_set_con_nodes(cid, int(sel.sum()), iptr(np.ascontiguousarray(k[sel], np.int32)),
                                          dptr(np.ascontiguousarray(Ly[j[sel]] * Lz[l[sel]]))):
                raise RuntimeError("api3_set_con_nodes failed")
    V = np.round(np.linspace(0.0, 1.0, 6), 12)
    return Workload("floating_base_pnp", (N, 1, 1) if graph else n, {"anode": ca, "cathode": cc},
                    [{"fixed": {"cathode": 0.0}, "swept": "anode", "V": V}], {"models": 7, "diag": diag})


def graph_schottky_diode(lib, n=(40, 3, 3), L=1e-6, ND=1e16, phi_m=4.8, models=7 | 64, h0=2e-9,
                         solver=GUI_SOLVER, V=None, diag=0.0):
    """The n-Si Schottky diode of schottky_diode() on a general (graph) mesh built from its
    tensor mesh: the metal face contact (bc 1) and the ohmic cathode as node lists on the
    x = 0 and x = L planes; the metal contact's inward column is walked along the graph."""
    lib.api3_init()
    xs = graded_axis(L, n[0], h0)
    ys = np.linspace(0.0, 0.2e-6, n[1])
    zs = np.linspace(0.0, 0.2e-6, n[2])
    Nx, Ny, Nz = n
    N = Nx * Ny * Nz
    rp, cj, h, ar, vol, pos = tensor_graph(xs, ys, zs, diag)
    si = lib.api3_add_material(SI, 300.0)
    if not lib.api3_set_mesh_graph(N, len(cj), iptr(rp), iptr(cj), dptr(h), dptr(ar), dptr(vol), dptr(pos)):
        raise RuntimeError("api3_set_mesh_graph rejected the graph")
    lib.api3_set_solver(*solver)
    lib.api3_set_models(models)
    mat = np.full(N, si, np.int32)
    lib.api3_set_node_data(iptr(mat), dptr(np.full(N, ND * 1e6)), dptr(np.zeros(N)), None)
    lib.api3_clear_contacts()
    ca = lib.api3_add_contact_ex(0, 0, Ny - 1, 0, Nz - 1, 0, 0, 1, 0.0, phi_m, 0.0, 0.0)
    cc = lib.api3_add_contact_ex(1, 0, Ny - 1, 0, Nz - 1, 0, 0, 0, 0.0, 0.0, 0.0, 0.0)
    k = np.arange(N)
    i, j, l = k % Nx, (k // Nx) % Ny, k // (Nx * Ny)
    Ly, Lz = fv_len(ys), fv_len(zs)
    for cid, plane in ((ca, 0), (cc, Nx - 1)):
        sel = i == plane
        if not lib.api3_set_con_nodes(cid, int(sel.sum()), iptr(np.ascontiguousarray(k[sel], np.int32)),
                                      dptr(np.ascontiguousarray(Ly[j[sel]] * Lz[l[sel]]))):
            raise RuntimeError("api3_set_con_nodes failed")
    if V is None:
        V = np.round(np.linspace(0.0, 0.4, 9), 12)
    return Workload("graph_schottky_diode", (N, 1, 1), {"anode": ca, "cathode": cc},
                    [{"fixed": {"cathode": 0.0}, "swept": "anode", "V": np.asarray(V, float)}],
                    {"ND_cm3": ND, "phi_m_eV": phi_m, "models": models, "diag": diag})


def graph_moscap(lib, models=7 | 32, solver=GUI_SOLVER, diag=0.0):
    """A thin-oxide n-Si MOS capacitor on a general (graph) mesh: n-Si (3e17 cm^-3) 40 nm deep
    under 1.5 nm of SiO2 meshed at 0.5 nm, a metal gate (work function 4.1 eV, a Dirichlet
    gate on the top plane) and an ohmic back contact as node lists; gate swept 0..1.6 V
    (accumulation: direct tunnelling of the accumulated electrons through the oxide nodes)."""
    lib.api3_init()
    ysi = 40e-9 - graded_axis(40e-9, 24, 0.3e-9)[::-1]
    ys = np.concatenate([ysi, 40e-9 + np.array([0.5e-9, 1.0e-9, 1.5e-9])])
    xs = np.linspace(0, 20e-9, 3)
    zs = np.linspace(0, 20e-9, 3)
    Nx, Ny, Nz = len(xs), len(ys), len(zs)
    N = Nx * Ny * Nz
    rp, cj, h, ar, vol, pos = tensor_graph(xs, ys, zs, diag)
    si = lib.api3_add_material(SI, 300.0)
    ox = lib.api3_add_material(SIO2, 300.0)
    if not lib.api3_set_mesh_graph(N, len(cj), iptr(rp), iptr(cj), dptr(h), dptr(ar), dptr(vol), dptr(pos)):
        raise RuntimeError("api3_set_mesh_graph rejected the graph")
    lib.api3_set_solver(*solver)
    lib.api3_set_models(models)
    k = np.arange(N)
    i, j, l = k % Nx, (k // Nx) % Ny, k // (Nx * Ny)
    oxide = j >= Ny - 3
    mat = np.where(oxide, ox, si).astype(np.int32)
    lib.api3_set_node_data(iptr(mat), dptr(np.where(oxide, 0.0, 3e23)), dptr(np.zeros(N)), None)
    lib.api3_clear_contacts()
    cb = lib.api3_add_contact_ex(2, 0, 2, 0, 2, 0, 0, 0, 0.0, 0.0, 0.0, 0.0)
    cg = lib.api3_add_contact_ex(3, 0, 2, 0, 2, 0, 0, 2, 0.0, 4.1, 0.0, 0.0)
    LX, LZ = fv_len(xs), fv_len(zs)
    for cid, sel in ((cb, j == 0), (cg, j == Ny - 1)):
        if not lib.api3_set_con_nodes(cid, int(sel.sum()), iptr(np.ascontiguousarray(k[sel], np.int32)),
                                      dptr(np.ascontiguousarray(LX[i[sel]] * LZ[l[sel]]))):
            raise RuntimeError("api3_set_con_nodes failed")
    V = np.round(np.linspace(0.0, 1.6, 9), 12)
    return Workload("graph_moscap", (N, 1, 1), {"back": cb, "gate": cg},
                    [{"fixed": {"back": 0.0}, "swept": "gate", "V": V}], {"models": models, "diag": diag})


def graph_nmosfet(lib, n=(24, 12, 3), Lx=500e-9, Ly=200e-9, Lz=100e-9, Nbody=1e17, Nsd=1e20, sigma=20e-9,
                  sd_len=100e-9, tox=2e-9, phi_m=4.6, models=4 | 8 | 16, solver=GUI_SOLVER, vd=0.05, vg_max=1.0,
                  dvg=0.25, h0=2e-9, diag=0.0, Nox=0.0, material=None, vds=None):
    """The n-MOSFET of nmosfet() on a general (graph) mesh built from its tensor mesh
    (tensor_graph, optional diagonal edges): contacts as node lists on the y = 0 surface
    (source, drain, the Robin face gate) and the back face (body), and the interface walls
    the host supplies on a graph (api3_set_walls): every semiconductor node under the gate
    has the gate surface as its wall - its distance and its cell's range from it - the
    walls the tensor path's scan finds for a face gate.  One gate sweep per drain bias of
    `vds` (default: the single bias vd)."""
    lib.api3_init()
    xs = np.linspace(0.0, Lx, n[0])
    ys = graded_axis(Ly, n[1], h0)
    zs = np.linspace(0.0, Lz, n[2])
    Nx, Ny, Nz = n
    N = Nx * Ny * Nz
    rp, cj, h, ar, vol, pos = tensor_graph(xs, ys, zs, diag)
    si = lib.api3_add_material(SI if material is None else material, 300.0)
    if not lib.api3_set_mesh_graph(N, len(cj), iptr(rp), iptr(cj), dptr(h), dptr(ar), dptr(vol), dptr(pos)):
        raise RuntimeError("api3_set_mesh_graph rejected the graph")
    lib.api3_set_solver(*solver)
    lib.api3_set_models(models)
    k = np.arange(N)
    i, j, l = k % Nx, (k // Nx) % Ny, k // (Nx * Ny)
    Nd2 = _gauss_sd(xs, ys, 0.0, sd_len, Nsd, sigma) + _gauss_sd(xs, ys, Lx - sd_len, Lx, Nsd, sigma)
    Nd = np.ascontiguousarray(Nd2[j, i] * 1e6)
    Na = np.full(N, Nbody * 1e6)
    mat = np.full(N, si, np.int32)
    lib.api3_set_node_data(iptr(mat), dptr(Nd), dptr(Na), dptr(np.zeros(N)))
    lib.api3_clear_contacts()
    iS1 = int(np.searchsorted(xs, 0.8 * sd_len, side="right")) - 1
    iD0 = int(np.searchsorted(xs, Lx - 0.8 * sd_len, side="left"))
    iG0 = int(np.searchsorted(xs, sd_len - 0.5 * sigma, side="left"))
    iG1 = int(np.searchsorted(xs, Lx - sd_len + 0.5 * sigma, side="right")) - 1
    nz = Nz - 1
    cs = lib.api3_add_contact_ex(2, 0, iS1, 0, nz, 0, 0, 0, 0.0, 0.0, 0.0, 0.0)
    cd = lib.api3_add_contact_ex(2, iD0, Nx - 1, 0, nz, 0, 0, 0, 0.0, 0.0, 0.0, 0.0)
    cg = lib.api3_add_contact_ex(2, iG0, iG1, 0, nz, 0, 0, 2, 0.0, phi_m, tox, Nox)
    cb = lib.api3_add_contact_ex(3, 0, Nx - 1, 0, nz, 0, 0, 0, 0.0, 0.0, 0.0, 0.0)
    LX, LZ = fv_len(xs), fv_len(zs)
    for cid, sel in ((cs, (j == 0) & (i <= iS1)), (cd, (j == 0) & (i >= iD0)),
                     (cg, (j == 0) & (i >= iG0) & (i <= iG1)), (cb, j == Ny - 1)):
        nodes = np.ascontiguousarray(k[sel], np.int32)
        areas = np.ascontiguousarray(LX[i[sel]] * LZ[l[sel]])
        if not lib.api3_set_con_nodes(cid, len(nodes), iptr(nodes), dptr(areas)):
            raise RuntimeError("api3_set_con_nodes failed")
    walls = np.ones((N, 6))
    under = (i >= iG0) & (i <= iG1)
    y = ys[j]
    lo = np.where(j > 0, 0.5 * (ys[np.maximum(j - 1, 0)] + y), y)
    hi = np.where(j < Ny - 1, 0.5 * (y + ys[np.minimum(j + 1, Ny - 1)]), y)
    walls[under, 0] = y[under]
    walls[under, 1] = np.maximum(lo[under], 0.0)
    walls[under, 2] = hi[under]
    lib.api3_set_walls(dptr(np.ascontiguousarray(walls.ravel())))
    npts = int(round(vg_max / dvg)) + 1
    V = np.round(np.linspace(0.0, vg_max, npts), 12)
    return Workload("graph_nmosfet", (N, 1, 1), {"source": cs, "drain": cd, "gate": cg, "body": cb},
                    [{"fixed": {"drain": v, "source": 0.0, "body": 0.0}, "swept": "gate", "V": V}
                     for v in (vds if vds is not None else (vd,))],
                    {"models": models, "diag": diag, "tox_m": tox, "pos": pos})


def graded_axis(L, n, h0):
    """n coordinates on [0, L] whose spacing grows geometrically from h0 at 0."""
    if n < 3:
        return np.linspace(0.0, L, n)
    lo, hi = 1.0, 2.0
    f = lambda g: h0 * (g ** (n - 1) - 1.0) / (g - 1.0) - L
    while f(hi) < 0:
        hi *= 2.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if f(mid) < 0:
            lo = mid
        else:
            hi = mid
    g = 0.5 * (lo + hi)
    h = h0 * g ** np.arange(n - 1)
    x = np.concatenate([[0.0], np.cumsum(h)])
    x *= L / x[-1]
    return x


def _gauss_sd(xs, ys, x0, x1, peak, sigma):
    """n+ implant: peak*exp(-y^2/2s^2) inside [x0, x1], Gaussian lateral falloff outside."""
    X, Y = np.meshgrid(xs, ys, indexing="xy")          # (Ny, Nx)
    d = np.where(X < x0, x0 - X, np.where(X > x1, X - x1, 0.0))
    return peak * np.exp(-0.5 * (Y / sigma) ** 2) * np.exp(-0.5 * (d / sigma) ** 2)


def nmosfet(lib, n=(120, 80, 60), Lx=500e-9, Ly=200e-9, Lz=100e-9, Nbody=1e17,
            Nsd=1e20, sigma=20e-9, sd_len=100e-9, tox=2e-9, phi_m=4.6, models=4,
            solver=GUI_SOLVER, vds=(0.05, 1.0), vg_max=1.2, dvg=0.05, h0=0.5e-9, material=None, Nox=0.0):
    """n-MOSFET: x along the channel, y into the substrate (y = 0 the gate surface),
    z across the width.  Contacts: source / drain ohmic on the surface over the n+
    windows, gate as a Robin face gate (oxide tox, fixed oxide charge Nox per m^2) over the
    channel, body ohmic on the back face.  Silicon unless `material` names another
    reference material id."""
    lib.api3_init()
    xs = np.linspace(0.0, Lx, n[0])
    ys = graded_axis(Ly, n[1], h0)
    zs = np.linspace(0.0, Lz, n[2])
    _grid(lib, xs, ys, zs)
    lib.api3_set_solver(*solver)
    lib.api3_set_models(models)
    si = lib.api3_add_material(SI if material is None else material, 300.0)
    Nd2 = _gauss_sd(xs, ys, 0.0, sd_len, Nsd, sigma) + _gauss_sd(xs, ys, Lx - sd_len, Lx, Nsd, sigma)
    Nd = np.ascontiguousarray(np.broadcast_to(Nd2[None, :, :], (n[2], n[1], n[0])).ravel() * 1e6)
    Na = np.full(Nd.shape, Nbody * 1e6)
    mat = np.full(Nd.shape, si, dtype=np.int32)
    Nf = np.zeros(Nd.shape)
    lib.api3_set_node_data(iptr(mat), dptr(Nd), dptr(Na), dptr(Nf))
    lib.api3_clear_contacts()
    iS1 = int(np.searchsorted(xs, 0.8 * sd_len, side="right")) - 1
    iD0 = int(np.searchsorted(xs, Lx - 0.8 * sd_len, side="left"))
    iG0 = int(np.searchsorted(xs, sd_len - 0.5 * sigma, side="left"))
    iG1 = int(np.searchsorted(xs, Lx - sd_len + 0.5 * sigma, side="right")) - 1
    nz = n[2] - 1
    cs = lib.api3_add_contact_ex(2, 0, iS1, 0, nz, 0, 0, 0, 0.0, 0.0, 0.0, 0.0)
    cd = lib.api3_add_contact_ex(2, iD0, n[0] - 1, 0, nz, 0, 0, 0, 0.0, 0.0, 0.0, 0.0)
    cg = lib.api3_add_contact_ex(2, iG0, iG1, 0, nz, 0, 0, 2, 0.0, phi_m, tox, Nox)
    cb = lib.api3_add_contact_ex(3, 0, n[0] - 1, 0, nz, 0, 0, 0, 0.0, 0.0, 0.0, 0.0)
    npts = int(round(vg_max / dvg)) + 1
    V = np.round(np.linspace(0.0, vg_max, npts), 12)
    sweeps = [{"fixed": {"drain": vd, "source": 0.0, "body": 0.0}, "swept": "gate", "V": V} for vd in vds]
    return Workload("nmosfet", n, {"source": cs, "drain": cd, "gate": cg, "body": cb}, sweeps,
                    {"Lx_m": Lx, "Ly_m": Ly, "Lz_m": Lz, "tox_m": tox, "phi_m_eV": phi_m,
                     "models": models, "Nbody_cm3": Nbody, "Nsd_cm3": Nsd, "sigma_m": sigma})


def finfet(lib, n=(96, 96, 64), Lsd=30e-9, Lg=30e-9, W=10e-9, H=40e-9, tox=1.5e-9, tmet=3e-9, tbox=5e-9,
           Nch=1e17, Nsd=1e20, sigma=3e-9, phi_m=4.6, models=4, solver=GUI_SOLVER,
           vds=(0.05, 0.25, 0.5, 0.75, 1.0), vg_max=1.0, dvg=0.02):
    """Tri-gate FinFET-like device on a tensor mesh: an n-channel Si fin W wide and H tall
    (x along the channel: source extension Lsd, gate Lg, drain extension Lsd) on a buried
    oxide tbox thick, wrapped on both sides and on top by tox of SiO2 and by gate metal tmet
    thick over the gate length (three box gate electrodes - left, right, top - driven
    together); SiO2 spacers fill the rest.  Channel p-type Nch (cm^-3), n+ source / drain
    Nsd with a Gaussian lateral falloff sigma under the gate edges; ohmic source / drain on
    the fin's end faces.  Uniform spacing on each axis; a node takes the region holding its
    position.  Gate swept 0..vg_max in dvg steps at each drain bias of `vds`."""
    lib.api3_init()
    Lx = 2 * Lsd + Lg
    Wt = W + 2 * (tox + tmet)
    Ht = tbox + H + tox + tmet
    xs = np.linspace(0.0, Lx, n[0])
    ys = np.linspace(0.0, Wt, n[1])
    zs = np.linspace(0.0, Ht, n[2])
    _grid(lib, xs, ys, zs)
    lib.api3_set_solver(*solver)
    lib.api3_set_models(models)
    si = lib.api3_add_material(SI, 300.0)
    ox = lib.api3_add_material(SIO2, 300.0)
    eps = 1e-15
    y0, y1 = tmet + tox, tmet + tox + W                 # fin faces across
    z0, z1 = tbox, tbox + H                             # fin bottom / top
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")    # (Nx, Ny, Nz)
    fin = (Y >= y0 - eps) & (Y <= y1 + eps) & (Z >= z0 - eps) & (Z <= z1 + eps)
    d = np.where(X < Lsd, 0.0, np.where(X > Lsd + Lg, 0.0, np.minimum(X - Lsd, Lsd + Lg - X)))
    inside = (X <= Lsd + eps) | (X >= Lsd + Lg - eps)
    dsd = np.where(inside, 0.0, d)
    Nd3 = np.where(fin, Nsd * np.exp(-0.5 * (dsd / sigma) ** 2), 0.0)
    Na3 = np.where(fin, Nch, 0.0)
    mat3 = np.where(fin, si, ox).astype(np.int32)
    tr = lambda a: np.ascontiguousarray(np.transpose(a, (2, 1, 0)).ravel())   # to x-fastest order
    lib.api3_set_node_data(iptr(tr(mat3)), dptr(tr(Nd3) * 1e6), dptr(tr(Na3) * 1e6), None)
    lib.api3_clear_contacts()
    idx = lambda c, lo, hi: (int(np.searchsorted(c, lo - eps, side="left")), int(np.searchsorted(c, hi + eps, side="right")) - 1)
    jf0, jf1 = idx(ys, y0, y1)
    lf0, lf1 = idx(zs, z0, z1)
    iG0, iG1 = idx(xs, Lsd, Lsd + Lg)
    jl1 = int(np.searchsorted(ys, tmet + eps, side="right")) - 1            # left metal: y <= tmet
    jr0 = int(np.searchsorted(ys, Wt - tmet - eps, side="left"))           # right metal: y >= Wt - tmet
    lt0 = int(np.searchsorted(zs, Ht - tmet - eps, side="left"))           # top metal: z >= Ht - tmet
    nx, ny, nz = n[0] - 1, n[1] - 1, n[2] - 1
    cs = lib.api3_add_contact_ex(0, jf0, jf1, lf0, lf1, 0, 0, 0, 0.0, 0.0, 0.0, 0.0)
    cd = lib.api3_add_contact_ex(1, jf0, jf1, lf0, lf1, 0, 0, 0, 0.0, 0.0, 0.0, 0.0)
    gl = lib.api3_add_contact_ex(6, iG0, iG1, 0, jl1, lf0, nz, 2, 0.0, phi_m, 0.0, 0.0)
    gr = lib.api3_add_contact_ex(6, iG0, iG1, jr0, ny, lf0, nz, 2, 0.0, phi_m, 0.0, 0.0)
    gt = lib.api3_add_contact_ex(6, iG0, iG1, 0, ny, lt0, nz, 2, 0.0, phi_m, 0.0, 0.0)
    npts = int(round(vg_max / dvg)) + 1
    V = np.round(np.linspace(0.0, vg_max, npts), 12)
    gates = ("gate_l", "gate_r", "gate_t")
    sweeps = [{"fixed": {"drain": vd, "source": 0.0}, "swept": gates, "V": V} for vd in vds]
    return Workload("finfet", n, {"source": cs, "drain": cd, "gate_l": gl, "gate_r": gr, "gate_t": gt}, sweeps,
                    {"fin_nm": (W * 1e9, H * 1e9), "Lg_m": Lg, "tox_m": tox, "phi_m_eV": phi_m, "models": models,
                     "Nch_cm3": Nch, "Nsd_cm3": Nsd})


def dense_axis(L, n, marks, h_fine, h_coarse, width):
    """n coordinates on [0, L] with a target spacing of h_fine at the planes `marks`,
    growing linearly over `width` to h_coarse away from them (then scaled to fill L)."""
    x = np.linspace(0.0, L, 20001)
    d = np.min(np.abs(x[:, None] - np.asarray(marks, dtype=np.float64)[None, :]), axis=1) if len(marks) else \
        np.full(x.shape, width)
    h = h_fine + (h_coarse - h_fine) * np.minimum(1.0, d / width)
    c = np.concatenate([[0.0], np.cumsum(0.5 * (1.0 / h[1:] + 1.0 / h[:-1]) * np.diff(x))])
    c *= (n - 1) / c[-1]
    out = np.interp(np.arange(n), c, x)
    out[0], out[-1] = 0.0, L
    return out


def power_cell(lib, n=(256, 256, 128), Lx=10e-6, Ly=60e-6, Lz=10e-6, Ndrift=1e15, Nsub=1e19, sub_top=55e-6,
               Nbody=1e17, body_sigma=1.2e-6, body_lat=0.25e-6, jfet_w=3e-6, Nsrc=1e20, src_sigma=0.15e-6,
               src_w=1.5e-6,
               Ntap=1e19, tap_w=1.0e-6, tox=50e-9, phi_m=4.1, gate_over=0.2e-6, models=7,
               solver=GUI_SOLVER, vgs=(10.0,), vd_max=50.0, dvd=1.0):
    """Vertical power-MOSFET cell (the reference's VDMOS template, main.py:984-1058, at the
    size of the large-device configuration): x across the cell, y the depth from the top
    surface, z along the gate fingers (the device is uniform in z).  An n- drift region
    Ndrift (cm^-3) over an n+ substrate Nsub below sub_top; p-body wells Gaussian-diffused
    from the surface (peak Nbody, depth and lateral sigma body_sigma) on both sides of a
    JFET window jfet_w wide in the middle; n+ sources (peak Nsrc, sigma src_sigma) src_w
    wide next to p+ body taps (Ntap) tap_w wide at the cell edges.  Contacts: the two
    sources (tap + source, ohmic, top face), two oxide (Robin) gates tox thick over the
    channels, overlapping the source and the JFET window by gate_over, and the drain
    (ohmic, bottom face).  One drain sweep 0..vd_max in dvd steps per gate bias of `vgs`."""
    lib.api3_init()
    xb = 0.5 * (Lx - jfet_w)                           # body mask edge at the JFET window
    xs_in = tap_w + src_w                              # source edge (channel start)
    xj = xb + body_lat * np.sqrt(2.0 * np.log(Nbody / Ndrift))   # surface junction body / drift
    xs = dense_axis(Lx, n[0], [tap_w, xs_in, xj, Lx - xj, Lx - xs_in, Lx - tap_w], 0.02e-6, 0.2e-6, 1.0e-6)
    ys = dense_axis(Ly, n[1], [0.0, 3 * src_sigma, 2.5 * body_sigma, sub_top], 0.01e-6, 1.0e-6, 4e-6)
    zs = np.linspace(0.0, Lz, n[2])
    _grid(lib, xs, ys, zs)
    lib.api3_set_solver(*solver)
    lib.api3_set_models(models)
    si = lib.api3_add_material(SI, 300.0)
    X, Y = np.meshgrid(xs, ys, indexing="xy")          # (Ny, Nx)

    def lateral(x0, x1, sig):
        d = np.where(X < x0, x0 - X, np.where(X > x1, X - x1, 0.0))
        return np.exp(-0.5 * (d / sig) ** 2)
    gy = lambda sig: np.exp(-0.5 * (Y / sig) ** 2)
    Nd2 = np.where(Y >= sub_top, Nsub, Ndrift) + Nsrc * gy(src_sigma) * (
        lateral(tap_w, xs_in, src_sigma) + lateral(Lx - xs_in, Lx - tap_w, src_sigma))
    Na2 = Nbody * gy(body_sigma) * (lateral(0.0, xb, body_lat) + lateral(Lx - xb, Lx, body_lat)) + \
        Ntap * gy(2 * src_sigma) * (lateral(0.0, tap_w, src_sigma) + lateral(Lx - tap_w, Lx, src_sigma))
    rep = lambda a: np.ascontiguousarray(np.broadcast_to(a[None, :, :], (n[2], n[1], n[0])).ravel())
    Nd, Na = rep(Nd2) * 1e6, rep(Na2) * 1e6
    mat = np.full(Nd.shape, si, dtype=np.int32)
    lib.api3_set_node_data(iptr(mat), dptr(Nd), dptr(Na), dptr(np.zeros(Nd.shape)))
    lib.api3_clear_contacts()
    span = lambda c, lo, hi: (int(np.searchsorted(c, lo - 1e-15, side="left")),
                              int(np.searchsorted(c, hi + 1e-15, side="right")) - 1)
    nz = n[2] - 1
    a0, a1 = span(xs, 0.0, xs_in)
    b0, b1 = span(xs, Lx - xs_in, Lx)
    g0, g1 = span(xs, xs_in - gate_over, xj + gate_over)
    h0, h1 = span(xs, Lx - xj - gate_over, Lx - xs_in + gate_over)
    csl = lib.api3_add_contact_ex(2, a0, a1, 0, nz, 0, 0, 0, 0.0, 0.0, 0.0, 0.0)
    csr = lib.api3_add_contact_ex(2, b0, b1, 0, nz, 0, 0, 0, 0.0, 0.0, 0.0, 0.0)
    cgl = lib.api3_add_contact_ex(2, g0, g1, 0, nz, 0, 0, 2, 0.0, phi_m, tox, 0.0)
    cgr = lib.api3_add_contact_ex(2, h0, h1, 0, nz, 0, 0, 2, 0.0, phi_m, tox, 0.0)
    cd = lib.api3_add_contact_ex(3, 0, n[0] - 1, 0, nz, 0, 0, 0, 0.0, 0.0, 0.0, 0.0)
    npts = int(round(vd_max / dvd)) + 1
    V = np.round(np.linspace(0.0, vd_max, npts), 12)
    sweeps = [{"fixed": {"source_l": 0.0, "source_r": 0.0, "gate_l": vg, "gate_r": vg}, "swept": "drain", "V": V}
              for vg in vgs]
    return Workload("power_cell", n, {"source_l": csl, "source_r": csr, "gate_l": cgl, "gate_r": cgr, "drain": cd},
                    sweeps, {"L_m": (Lx, Ly, Lz), "models": models, "tox_m": tox, "phi_m_eV": phi_m,
                             "Ndrift_cm3": Ndrift, "Nsub_cm3": Nsub, "Nbody_cm3": Nbody})


def diode_variants(count=64, seed=20261203, nmin=32, nmax=72):
    """Parameters of the batched pn-diode family (recorded seed)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        nn = int(rng.integers(nmin ** 3, nmax ** 3 + 1))
        a = int(round(nn ** (1.0 / 3.0)))
        b = int(round((nn / a) ** 0.5))
        c = max(2, int(round(nn / (a * b))))
        NA = 10.0 ** rng.uniform(15.0, 18.0)
        ND = 10.0 ** rng.uniform(15.0, 18.0)
        xj = rng.uniform(0.2e-6, 0.8e-6)
        out.append({"n": (a, b, c), "NA": NA, "ND": ND, "xj": xj})
    return out


def diode_variant(lib, v, vmax=0.7, dv=0.025, solver=GUI_SOLVER):
    """One member of the batched family (constant mobility, tau 1e-7 s, models 0)."""
    w = pn_diode(lib, n=v["n"], NA=v["NA"], ND=v["ND"], xj=v["xj"], solver=solver,
                 vmax=vmax, dv=dv)
    w.name = "diode_variant"
    return w


def bias_vector(w, sweep, Vswept):
    """Contact voltages (by contact id) of one sweep point; `swept` names one contact or a
    tuple of contacts driven together (the three gate electrodes of a tri-gate)."""
    V = {w.contacts[k]: v for k, v in sweep["fixed"].items()}
    sw = sweep["swept"]
    for k in (sw if isinstance(sw, (tuple, list)) else (sw,)):
        V[w.contacts[k]] = float(Vswept)
    return V


def run_sweep(lib, w, sweep, timer=None, on_point=None):
    """Sweep one contact the way main.run_sweep does (main.py:3638-3730): set the
    voltages, api3_resolve per point.  Returns (V, I[npts, ncon], Iflr, conv)."""
    nc = lib.api3_get_ncon()
    V = np.asarray(sweep["V"], dtype=np.float64)
    I = np.zeros((len(V), nc))
    F = np.zeros((len(V), nc))
    conv = np.zeros(len(V), dtype=bool)
    for q, v in enumerate(V):
        for cid, vv in bias_vector(w, sweep, v).items():
            lib.api3_set_contact_V(cid, vv)
        conv[q] = bool(lib.api3_resolve())
        for c in range(nc):
            I[q, c] = lib.api3_get_contact_I(c)
            F[q, c] = lib.api3_get_contact_Ifloor(c)
        if on_point is not None:
            on_point(q, v)
    return V, I, F, conv


def start_sweep(lib, w, sweep):
    """Equilibrium + ramp to the first point of a sweep (api3_solve at that bias)."""
    for cid, vv in bias_vector(w, sweep, sweep["V"][0]).items():
        lib.api3_set_contact_V(cid, vv)
    return bool(lib.api3_solve())


def field(lib, which, shape):
    """api3_bulk_copy of one quantity as an (Nz, Ny, Nx) array."""
    N = int(np.prod(shape))
    buf = np.zeros(N)
    lib.api3_bulk_copy(which, dptr(buf))
    return buf.reshape(shape[2], shape[1], shape[0])
