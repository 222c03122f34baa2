"""Persistent linear solves (one cooperative launch per solve) against the per-pass path.

The persistent kernels run the same passes and the same stop rules as the per-pass
kernels inside device-looped CUDA graphs; only the summation order of the dot products
differs.  Checked here, on the golden devices' own continuity and Poisson systems:

* both paths meet the reference's stop rule (BiCGSTAB: ||b - A x|| <= max(rtol ||r0||,
  atol floor), semiconductor_3d.c:2244-2268; PCG: r.z <= rtol^2 r0.z0, :2207), in FP64 and
  in the refined precision, and take about the same number of iterations;
* their solutions agree to the solve tolerance;
* a whole bias sweep gives the same terminal currents (tight tolerances: 1e-6 relative or
  the reference's round-off floor);
* the persistent path launches far fewer kernels;
* its bounded barrier wait gives up and reports it (a launch whose last block never
  arrives).
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
sys.path.insert(0, HERE)

from oracle import restate as R  # noqa: E402
import semiconductor_devices_simulator_b200 as S  # noqa: E402
from semiconductor_devices_simulator_b200 import devices as D  # noqa: E402
from semiconductor_devices_simulator_b200.abi import dptr, iptr  # noqa: E402
from test_gpu_kernels import setup, load_state, NAMES  # noqa: E402

pytestmark = pytest.mark.gpu
TIGHT = (2000, 1000, 500, 1e-10, 1e-8, 1.0, 1.0)     # validate.py:53


@pytest.fixture(scope="module")
def lib():
    return S.load()


@pytest.fixture(params=[0, 1], ids=["fp64", "refined"])
def precision(lib, request):
    old = lib.api3b_set_precision(request.param)
    yield request.param
    lib.api3b_set_precision(old)


def persist(lib, on):
    return lib.api3b_set_persist(1 if on else 0, -1)


def bicg(lib, g, w, hole, rtol, atol=2e-14):
    N = w.N
    sol = np.zeros(N); rn = np.zeros(1); r0 = np.zeros(1)
    l0 = lib.b200x_launches()
    its = lib.b200x_bicgstab(1000, rtol, atol, -1 if hole else 1, None, dptr(sol), dptr(rn), dptr(r0))
    return its, sol, rn[0], r0[0], lib.b200x_launches() - l0


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("hole", [0, 1])
def test_persistent_bicgstab_matches_per_pass(lib, precision, name, hole):
    g, w = setup(lib, name)
    t = "p" if hole else "n"
    load_state(lib, g, "pert_")
    lib.b200x_cont_assemble(hole, None, None, None, None)
    rtol, atol = 1e-8, 2e-14
    old = persist(lib, True)
    try:
        its_p, x_p, rn_p, r0_p, nl_p = bicg(lib, g, w, hole, rtol, atol)
        persist(lib, False)
        its_g, x_g, rn_g, r0_g, nl_g = bicg(lib, g, w, hole, rtol, atol)
    finally:
        persist(lib, old)
    A, b = g[f"cont{t}_A"], g[f"cont{t}_rhs"]
    dims = tuple(int(v) for v in g["dims"])
    r00 = np.linalg.norm(b - R.matvec(A, dims, np.ones(w.N)))
    tgt = max(rtol * r00, atol * R.bicg_floor(A, dims, b, np.ones(w.N)))
    for x, its in ((x_p, its_p), (x_g, its_g)):
        res = np.linalg.norm(b - R.matvec(A, dims, x))
        assert res <= 1.5 * tgt + 1e-300, (res, tgt, its)
    assert abs(its_p - its_g) <= max(2, its_g // 5), (its_p, its_g)
    assert abs(r0_p - r0_g) <= 1e-9 * r0_g
    # the two solutions differ by at most what the stop rule leaves open
    scale = np.abs(x_g).max()
    assert np.abs(x_p - x_g).max() <= 1e-5 * scale + 1e-300, np.abs(x_p - x_g).max() / scale
    assert nl_p < nl_g, (nl_p, nl_g)


@pytest.mark.parametrize("name", NAMES)
def test_persistent_pcg_matches_per_pass(lib, precision, name):
    g, w = setup(lib, name)
    load_state(lib, g, "pert_")
    F = np.zeros(w.N)
    lib.b200x_poisson(dptr(np.ascontiguousarray(g["pert_phi"])), dptr(F), None, None)
    out = {}
    old = persist(lib, True)
    try:
        for on in (True, False):
            persist(lib, on)
            sol = np.zeros(w.N)
            l0 = lib.b200x_launches()
            its = lib.b200x_pcg(2000, 1e-6, dptr(sol))
            out[on] = (its, sol, lib.b200x_launches() - l0)
    finally:
        persist(lib, old)
    A = g["pois_A"]
    dims = tuple(int(v) for v in g["dims"])
    for on, (its, sol, _) in out.items():
        res = np.linalg.norm(g["pois_F"] - R.matvec(A, dims, sol))
        assert res <= 1e-3 * np.linalg.norm(g["pois_F"]), (on, res, its)
    assert abs(out[True][0] - out[False][0]) <= max(2, out[False][0] // 5)
    scale = np.abs(out[False][1]).max()
    assert np.abs(out[True][1] - out[False][1]).max() <= 1e-3 * scale
    assert out[True][2] < out[False][2]


def test_persistent_sweep_matches_per_pass(lib, precision):
    """A whole Id-Vg sweep of a small MOSFET at tight tolerances, persistent against
    per-pass: every terminal current within 1e-6 relative or its round-off floor."""
    res = {}
    old = persist(lib, True)
    try:
        for on in (True, False):
            persist(lib, on)
            w = D.nmosfet(lib, n=(24, 16, 10), models=4, vds=(1.0,), vg_max=1.2, dvg=0.1, solver=TIGHT)
            s = w.sweeps[0]
            assert D.start_sweep(lib, w, s)
            l0 = lib.b200x_launches()
            V, I, F, conv = D.run_sweep(lib, w, s)
            res[on] = (I, F, conv, lib.b200x_launches() - l0)
    finally:
        persist(lib, old)
    (I1, F1, c1, n1), (I0, F0, c0, n0) = res[True], res[False]
    assert c1.all() and c0.all()
    tol = np.maximum(1e-6 * np.abs(I0), np.maximum(F0, F1))
    assert (np.abs(I1 - I0) <= tol).all(), np.max(np.abs(I1 - I0) / np.maximum(np.abs(I0), 1e-300))
    assert n1 < n0 / 2, (n1, n0)


def test_bounded_barrier_wait_gives_up(lib):
    """A launch whose last block never reaches the barrier: the other blocks stop waiting
    after the limit, set the error word and report it; the context stays usable."""
    w = D.pn_diode(lib, n=(12, 6, 5))
    assert lib.b200x_prepare() == 1
    gave = np.zeros(1, dtype=np.int32)
    err = lib.b200x_persist_probe(4, 0.2, iptr(gave))
    assert err == 1 and gave[0] == 3, (err, gave[0])
    # the device still works: a normal solve afterwards
    s = w.sweeps[0]
    assert D.start_sweep(lib, w, s)


@pytest.mark.parametrize("diag", [0.0, 0.3])
def test_persistent_graph_sweep_matches_per_pass(lib, diag):
    """The general-mesh path (ELL kernels, aggregation multigrid with the multicolour
    smoother): a small graph MOSFET's Id-Vg sweep at tight tolerances, persistent solves
    against the per-launch ones (host-driven Krylov loops) - the same currents within 1e-6
    relative or the floor, far fewer launches.  diag > 0 adds diagonal edges in every x-y
    cell (more colours per level)."""
    res = {}
    old = persist(lib, True)
    try:
        for on in (True, False):
            persist(lib, on)
            w = D.graph_nmosfet(lib, n=(24, 12, 3), models=4, vd=1.0, vg_max=1.0, dvg=0.2, solver=TIGHT, diag=diag)
            s = w.sweeps[0]
            assert D.start_sweep(lib, w, s)
            l0 = lib.b200x_launches()
            V, I, F, conv = D.run_sweep(lib, w, s)
            res[on] = (I, F, conv, lib.b200x_launches() - l0)
    finally:
        persist(lib, old)
    (I1, F1, c1, n1), (I0, F0, c0, n0) = res[True], res[False]
    assert c1.all() and c0.all()
    tol = np.maximum(1e-6 * np.abs(I0), np.maximum(F0, F1))
    assert (np.abs(I1 - I0) <= tol).all(), np.max(np.abs(I1 - I0) / np.maximum(np.abs(I0), 1e-300))
    assert n1 < n0, (n1, n0)
