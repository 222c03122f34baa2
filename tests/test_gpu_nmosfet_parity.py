"""Parity on the benchmark's own workload: the n-MOSFET Id-Vg family (Robin oxide gate,
Gaussian n+ source / drain, velocity-saturated mobility), both drain biases (0.05 V and
1.0 V), all 25 gate points (0..1.2 V in 0.05 V steps) of each sweep.

* 60x40x30 mesh (72,000 nodes), both codes converged tightly (inner solves to round-off,
  validate.py's Gummel tolerances), in FP64 and in the refined precision: every terminal
  current within 1e-4 relative of the reference core's or below its round-off floor Iflr,
  psi within 1e-6 V on every node.
* The full 120x80x60 mesh (576,000 nodes), tight tolerances: the refined path's currents
  within 1e-4 of the FP64 path's (or its floor) at every point of both sweeps, psi within
  1e-6 V.
* The full mesh at the production tolerances (the GUI's solver tuple), both precisions,
  against the reference core run live: every terminal current within 1e-4 relative, the
  floor, or the reference's own convergence error at these tolerances - twice its distance
  to the converged value (the FP64 tight solution, which the 72,000-node case shows equal
  to the reference's tight solution).  The reference converges a carrier's quasi-Fermi
  level only where that carrier carries >= 1e-3 of the local charge
  (semiconductor_3d.c:3136-3144), so its deep-subthreshold currents are converged to
  ~1e-3 only; on-state currents (>= 1 nA) must agree within 1e-4 outright.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
sys.path.insert(0, HERE)

import make_golden as MG  # noqa: E402
import semiconductor_devices_simulator_b200 as S  # noqa: E402
from semiconductor_devices_simulator_b200 import devices as D  # noqa: E402
from test_gpu_sweep import reference_lib, check_currents, PSI_TOL, I_RTOL  # noqa: E402

pytestmark = pytest.mark.gpu
_cache = {}


@pytest.fixture(scope="module")
def lib():
    return S.load()


def sweeps(L, n, tight, prec=None, keep_psi=True):
    """Both Id-Vg sweeps of the MOSFET on mesh n: per sweep (I, Iflr, conv, psi per point)."""
    env = MG.TIGHT_ENV if tight else {}
    old_env = {k: os.environ.get(k) for k in env}
    os.environ.update(env)                       # read by api3_init, as the reference reads them
    old_prec = L.api3b_set_precision(prec) if prec is not None else None
    try:
        w = D.nmosfet(L, n=n, solver=MG.TIGHT_SOLVER if tight else D.GUI_SOLVER)
        out = []
        for s in w.sweeps:
            psi = []
            ok0 = D.start_sweep(L, w, s)
            grab = (lambda q, v: psi.append(D.field(L, 0, w.shape).ravel())) if keep_psi else None
            V, I, F, conv = D.run_sweep(L, w, s, on_point=grab)
            out.append((ok0, I, F, conv, np.array(psi)))
        return out
    finally:
        for k, v in old_env.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
        if prec is not None:
            L.api3b_set_precision(old_prec)


def cached(key, fn):
    if key not in _cache:
        _cache[key] = fn()
    return _cache[key]


@pytest.fixture(params=[0, 1], ids=["fp64", "refined"])
def prec(request):
    return request.param


def test_nmosfet_72k_tight_matches_reference(lib, prec):
    ref = reference_lib()
    ref.api3_set_threads(os.cpu_count() or 1)
    r = cached("ref72t", lambda: sweeps(ref, (60, 40, 30), True))
    g = sweeps(lib, (60, 40, 30), True, prec)
    for (gok, gI, gF, gc, gpsi), (rok, rI, rF, rc, rpsi) in zip(g, r):
        assert gok and rok and gc.all() and rc.all()
        check_currents(gI, rI, rF)
        assert np.abs(gpsi - rpsi).max() <= PSI_TOL


def test_nmosfet_full_size_refined_matches_fp64_tight(lib):
    f64 = cached("gpu576t64", lambda: sweeps(lib, (120, 80, 60), True, 0))
    r32 = sweeps(lib, (120, 80, 60), True, 1)
    for (aok, aI, aF, ac, apsi), (bok, bI, bF, bc, bpsi) in zip(r32, f64):
        assert aok and bok and ac.all() and bc.all()
        check_currents(aI, bI, bF)
        assert np.abs(apsi - bpsi).max() <= PSI_TOL


def test_nmosfet_full_size_default_matches_reference(lib, prec):
    ref = reference_lib()
    ref.api3_set_threads(os.cpu_count() or 1)
    r = cached("ref576", lambda: sweeps(ref, (120, 80, 60), False, keep_psi=False))
    conv = cached("gpu576t64", lambda: sweeps(lib, (120, 80, 60), True, 0))
    g = sweeps(lib, (120, 80, 60), False, prec, keep_psi=False)
    for (gok, gI, gF, gc, _), (rok, rI, rF, rc, _), (_, cI, _, _, _) in zip(g, r, conv):
        assert gok and rok and gc.all() and rc.all()
        own = 2.0 * np.abs(rI - cI)               # the reference's distance to the converged currents
        check_currents(gI, rI, np.maximum(rF, own))
        on = np.abs(rI) >= 1e-9
        assert (np.abs(gI - rI)[on] <= I_RTOL * np.abs(rI)[on]).all()
