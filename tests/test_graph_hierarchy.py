"""The graph multigrid's hierarchy (pairwise aggregation by coupling strength, contracted
patterns; semiconductor_3d.c:2340-2512) equals the reference's level for level - node
counts, CSR patterns in the same entry order and every node's aggregate, integer for
integer - on graphs from tensor meshes with and without diagonal edges, uniform and graded,
and with the pairing knobs changed.  Host only: no GPU needed."""
import ctypes
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)

import semiconductor_devices_simulator_b200 as S  # noqa: E402
from semiconductor_devices_simulator_b200 import abi, devices as D  # noqa: E402
from semiconductor_devices_simulator_b200.abi import dptr, iptr  # noqa: E402

HX = {"hx_gmg_level": (ctypes.c_int, [ctypes.c_int] + [ctypes.POINTER(ctypes.c_int)] * 5)}


def reference_lib():
    path = os.path.join(ROOT, "oracle", "_ref", "libsemisim_harness.so")
    if not os.path.exists(path):
        pytest.skip("reference core not built (make -C oracle)")
    return abi.bind(ctypes.CDLL(path), HX)


def levels_ref(ref, g):
    rp, cj, h, ar, vol, pos = g
    N = len(vol)
    ref.api3_init()
    ref.api3_add_material(D.SI, 300.0)
    assert ref.api3_set_mesh_graph(N, len(cj), iptr(rp), iptr(cj), dptr(h), dptr(ar), dptr(vol), dptr(pos)) == 1
    return dump(lambda L, *a: ref.hx_gmg_level(L, *a))


def levels_ours(lib, g):
    rp, cj, h, ar, vol, pos = g
    return dump(lambda L, *a: lib.b200x_gmg_plan(len(vol), iptr(rp), iptr(cj), dptr(h), dptr(ar), L, *a))


def dump(fn):
    n, nnz = np.zeros(1, np.int32), np.zeros(1, np.int32)
    nl = fn(0, iptr(n), iptr(nnz), None, None, None)
    out = []
    for L in range(nl):
        fn(L, iptr(n), iptr(nnz), None, None, None)
        rp = np.zeros(n[0] + 1, np.int32)
        cj = np.zeros(max(nnz[0], 1), np.int32)
        agg = np.full(n[0], -7, np.int32)
        fn(L, iptr(n), iptr(nnz), iptr(rp), iptr(cj), iptr(agg))
        out.append((int(n[0]), rp, cj[:nnz[0]], agg))
    return out


GRAPHS = {
    "cube_14": lambda: D.tensor_graph(*(np.linspace(0, 1e-6, 14),) * 3),
    "diag_20x16x6": lambda: D.tensor_graph(np.linspace(0, 1e-6, 20), np.linspace(0, 0.8e-6, 16),
                                           np.linspace(0, 0.3e-6, 6), diag=0.3),
    "graded_24x12x8": lambda: D.tensor_graph(D.graded_axis(1e-6, 24, 2e-9), D.graded_axis(0.2e-6, 12, 1e-9),
                                             np.linspace(0, 0.1e-6, 8), diag=0.2),
}


@pytest.mark.parametrize("knobs", [None, ("2", "0.25")], ids=["default", "passes2_beta0.25"])
@pytest.mark.parametrize("name", sorted(GRAPHS))
def test_hierarchy_equals_reference(name, knobs, monkeypatch):
    if knobs:
        monkeypatch.setenv("SEMISIM_GPASS", knobs[0])
        monkeypatch.setenv("SEMISIM_GBETA", knobs[1])
    else:
        monkeypatch.delenv("SEMISIM_GPASS", raising=False)
        monkeypatch.delenv("SEMISIM_GBETA", raising=False)
    lib = S.load()
    lib.api3_init()                               # reads the pairing knobs
    ref = reference_lib()
    g = GRAPHS[name]()
    a, b = levels_ours(lib, g), levels_ref(ref, g)
    assert len(a) == len(b) and len(a) >= 2
    for L, (x, y) in enumerate(zip(a, b)):
        assert x[0] == y[0], f"level {L} size"
        assert np.array_equal(x[1], y[1]) and np.array_equal(x[2], y[2]), f"level {L} pattern"
        if L < len(a) - 1:
            assert np.array_equal(x[3], y[3]), f"level {L} aggregates"
    assert a[-1][0] <= 160 or a[-1][0] > 0.7 * a[-2][0]
    # the knobs are process state of both libraries (read only when set): back to the
    # defaults, 3 rounds of pairing at beta 0.5
    monkeypatch.setenv("SEMISIM_GPASS", "3")
    monkeypatch.setenv("SEMISIM_GBETA", "0.5")
    lib.api3_init()
    levels_ref(ref, g)
