"""Per-point outputs of the ABI against the reference core, live: every derived node
quantity of api3_bulk_copy (0..35), the face current densities api3_face_J, api3_get_Emax,
api3_carrier_sums, the quasi-static charge partition (api3_charge_partition,
api3_charge_owner, api3_terminal_charges) and api3_ins_field_max, on the three small
devices solved tightly at one bias by both libraries.

Tolerances: node and face arrays within 1e-5 of the array's largest magnitude, with the
same NaN nodes (current-density components against their vector's largest component, plus
negligible absolute floors for currents and recombination rates, whose round-off on near-
equilibrium devices is pure noise); scalar outputs within 1e-6 relative; charge owners
identical.  The position api3_ins_field_max reports is not compared: these devices are
uniform along an axis, so the maximum is attained on a whole line of nodes and either
code's round-off picks one of them."""
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
from semiconductor_devices_simulator_b200 import abi  # noqa: E402
from semiconductor_devices_simulator_b200.abi import dptr, iptr  # noqa: E402

pytestmark = pytest.mark.gpu
NAMES = ["diode_small", "mos_small", "moscap_small", "sic_small"]


@pytest.fixture(scope="module")
def lib():
    return S.load()


def reference_lib():
    path = os.path.join(ROOT, "oracle", "_ref", "libsemisim_harness.so")
    if not os.path.exists(path):
        pytest.skip("reference core not built (make -C oracle)")
    return abi.bind(ctypes.CDLL(path))


def outputs(L, name):
    w, mat, bias = MG.build(L, name)
    L.api3_set_solver(*MG.TIGHT_SOLVER)
    for cid, v in bias.items():
        L.api3_set_contact_V(cid, v)
    assert L.api3_solve()
    N, nc = w.N, L.api3_get_ncon()
    o = {}
    for q in range(36):
        a = np.zeros(N)
        L.api3_bulk_copy(q, dptr(a))
        o[f"bulk{q}"] = a
    for ax in range(3):
        for car in (0, 1):
            a = np.zeros(N)
            assert L.api3_face_J(ax, car, dptr(a)) == 1
            o[f"J{ax}{car}"] = a
    o["Emax"] = L.api3_get_Emax()
    cs = np.zeros(2)
    L.api3_carrier_sums(dptr(cs))
    o["sums"] = cs
    cterm = np.arange(nc, dtype=np.int32)
    o["meet"] = L.api3_charge_partition(iptr(cterm))
    own = np.zeros(N, np.int32)
    assert L.api3_charge_owner(iptr(own)) == 1
    o["own"] = own
    Qt = np.zeros(nc + 1)
    assert L.api3_terminal_charges(nc, dptr(Qt)) == 1
    o["Qt"] = Qt
    pos = np.zeros(3)
    o["Fins"] = L.api3_ins_field_max(dptr(pos))
    o["Fpos"] = pos
    return o


@pytest.mark.parametrize("name", NAMES)
def test_per_point_outputs_match_reference(lib, name, monkeypatch):
    for k, v in MG.TIGHT_ENV.items():
        monkeypatch.setenv(k, v)
    ref = reference_lib()
    ref.api3_set_threads(os.cpu_count() or 1)
    g, r = outputs(lib, name), outputs(ref, name)
    bad = []
    # a current-density component is measured against the largest component of its vector
    # (a device's currents flow along one axis; the others are round-off), and current
    # densities and recombination rates get an absolute floor far below anything physical
    # (1e-3 A/m^2, 1e12 m^-3 s^-1: devices at or near equilibrium carry pure round-off there)
    groups = {f"bulk{q}": [f"bulk{x}" for x in (7, 8, 9)] for q in (7, 8, 9)}
    groups.update({f"bulk{q}": [f"bulk{x}" for x in (20, 21, 22)] for q in (20, 21, 22)})
    groups.update({f"bulk{q}": [f"bulk{x}" for x in (23, 24, 25)] for q in (23, 24, 25)})
    groups.update({f"J{a}{c}": [f"J{x}{c}" for x in range(3)] for a in range(3) for c in (0, 1)})
    floor = {k: 1e-3 for k in groups}
    floor["bulk12"] = 1e12
    for key in [f"bulk{q}" for q in range(36)] + [f"J{a}{c}" for a in range(3) for c in (0, 1)]:
        a, b = g[key], r[key]
        if not np.array_equal(np.isnan(a), np.isnan(b)):
            bad.append(f"{key}: NaN nodes differ")
            continue
        m = ~np.isnan(b)
        if not m.any():
            continue
        scale = max(np.nanmax(np.abs(r[q])) for q in groups.get(key, [key]))
        err = np.abs(a[m] - b[m]).max()
        if not err <= 1e-5 * scale + floor.get(key, 1e-300):
            bad.append(f"{key}: {err:.3e} of {scale:.3e}")
    for key in ("Emax", "Fins"):
        if not abs(g[key] - r[key]) <= 1e-6 * abs(r[key]) + 1e-300:
            bad.append(f"{key}: {g[key]!r} vs {r[key]!r}")
    if not np.allclose(g["sums"], r["sums"], rtol=1e-6, atol=0):
        bad.append(f"carrier sums {g['sums']} vs {r['sums']}")
    if g["meet"] != r["meet"] or not np.array_equal(g["own"], r["own"]):
        bad.append("charge partition differs")
    qs = np.abs(r["Qt"]).max()
    if not np.abs(g["Qt"] - r["Qt"]).max() <= 1e-6 * qs + 1e-300:
        bad.append(f"terminal charges {g['Qt']} vs {r['Qt']}")
    assert not bad, name + "\n" + "\n".join(bad)


def scalar_outputs(L, N, nc):
    o = {"Emax": L.api3_get_Emax()}
    cs = np.zeros(2)
    L.api3_carrier_sums(dptr(cs))
    o["sums"] = cs
    cterm = np.arange(nc, dtype=np.int32)
    o["meet"] = L.api3_charge_partition(iptr(cterm))
    own = np.zeros(N, np.int32)
    assert L.api3_charge_owner(iptr(own)) == 1
    o["own"] = own
    for nt in (nc, nc + 2, max(nc - 1, 1)):
        Qt = np.zeros(nt + 1)
        assert L.api3_terminal_charges(nt, dptr(Qt)) == 1
        o[f"Qt{nt}"] = Qt
    pos = np.zeros(3)
    o["Fins"] = L.api3_ins_field_max(dptr(pos))
    o["Fpos"] = pos
    return o


@pytest.mark.parametrize("name", NAMES)
def test_output_reductions_on_one_state(lib, name, monkeypatch):
    """The device reductions behind api3_get_Emax, api3_carrier_sums, api3_terminal_charges
    and api3_ins_field_max against the reference core's scans of the same state: this
    library's solution is installed in the reference with api3_set_state, so both evaluate
    identical potentials.  Emax and the insulator field (differences and quotients of the
    same doubles) agree to round-off and the field's position exactly (ties resolve to the
    reference's scan order); the sums differ only by summation order; terminal counts above,
    at and below the number of terminals are covered."""
    for k, v in MG.TIGHT_ENV.items():
        monkeypatch.setenv(k, v)
    ref = reference_lib()
    ref.api3_set_threads(os.cpu_count() or 1)
    states = []
    for L in (lib, ref):
        w, mat, bias = MG.build(L, name)
        L.api3_set_solver(*MG.TIGHT_SOLVER)
        for cid, v in bias.items():
            L.api3_set_contact_V(cid, v)
        assert L.api3_solve()
        states.append(w)
    N, nc = states[0].N, lib.api3_get_ncon()
    phi, phin, phip = np.zeros(N), np.zeros(N), np.zeros(N)
    assert lib.api3_get_state(dptr(phi), dptr(phin), dptr(phip)) == 1
    assert ref.api3_set_state(dptr(phi), dptr(phin), dptr(phip)) == 1
    g, r = scalar_outputs(lib, N, nc), scalar_outputs(ref, N, nc)
    bad = []
    for key, tol in (("Emax", 1e-13), ("Fins", 1e-14)):
        if not abs(g[key] - r[key]) <= tol * abs(r[key]):
            bad.append(f"{key}: {g[key]!r} vs {r[key]!r}")
    if not np.array_equal(g["Fpos"], r["Fpos"], equal_nan=True):
        bad.append(f"field position {g['Fpos']} vs {r['Fpos']}")
    if not np.allclose(g["sums"], r["sums"], rtol=1e-12, atol=0):
        bad.append(f"carrier sums {g['sums']} vs {r['sums']}")
    if g["meet"] != r["meet"] or not np.array_equal(g["own"], r["own"]):
        bad.append("charge partition differs")
    for key in [k for k in r if k.startswith("Qt")]:
        qs = np.abs(r[key]).max()
        if not np.abs(g[key] - r[key]).max() <= 1e-10 * qs:
            bad.append(f"{key}: {g[key]} vs {r[key]}")
    assert not bad, name + "\n" + "\n".join(bad)
