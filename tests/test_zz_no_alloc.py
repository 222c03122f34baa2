"""The allocation-free residual entry point (api3b_stencil_residual_noalloc).

It serves callers that cannot call cudaMalloc - their device memory belongs to another
allocator, or an allocation on their path is not acceptable - so they pass their own
device buffers and the entry point keeps its reduction scratch in a file-scope device
array.  Checked here against the existing entry point that runs the same computation with
the solver instance's own scratch (b200x_bicgstab: its start kernel computes the initial
residual norm), on two calls in a row, and against the reference's golden vectors.  The
file's name makes pytest collect it last.
"""
import ctypes
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_golden as MG  # noqa: E402
from oracle import restate as R  # noqa: E402
import semiconductor_devices_simulator_b200 as S  # noqa: E402
from semiconductor_devices_simulator_b200.abi import dptr  # noqa: E402

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def _dev(t):
    return ctypes.cast(ctypes.c_void_p(t.data_ptr()), ctypes.POINTER(ctypes.c_double))


def test_noalloc_residual_matches_existing_entry():
    import torch
    lib = S.load()
    g = np.load(os.path.join(HERE, "golden", "diode_small.npz"))
    w, mat, bias = MG.build(lib, "diode_small")
    for cid, v in g["kern_bias"]:
        lib.api3_set_contact_V(int(cid), float(v))
    assert lib.b200x_prepare() == 1
    for which, key in ((0, "pert_phi"), (1, "pert_phin"), (2, "pert_phip"), (3, "pert_n"), (4, "pert_p")):
        assert lib.b200x_set(which, dptr(np.ascontiguousarray(g[key]))) == 1
    for q in range(6):
        assert lib.b200x_set(S.ST_FMU + q, dptr(np.ascontiguousarray(g["pert_fmu"][q]))) == 1
    N = w.N
    Nx, Ny, Nz = w.shape
    A7 = np.zeros(7 * N); rhs = np.zeros(N)
    lib.b200x_cont_assemble(0, dptr(A7), dptr(rhs), None, None)
    x0 = np.ascontiguousarray(g["contn_x"])
    # the existing entry point: BiCGSTAB start (no iterations) reports ||rhs - A x0||
    sol = np.zeros(N); rn = np.zeros(1); r0 = np.zeros(1)
    lib.b200x_bicgstab(0, 1e-4, 2e-14, 1, dptr(x0), dptr(sol), dptr(rn), dptr(r0))
    dA = torch.tensor(A7, dtype=torch.float64, device="cuda")
    dx = torch.tensor(x0, dtype=torch.float64, device="cuda")
    db = torch.tensor(rhs, dtype=torch.float64, device="cuda")
    r_ref = rhs - R.matvec(A7.reshape(7, N), (Nx, Ny, Nz), x0)
    floor_ref = R.bicg_floor(A7.reshape(7, N), (Nx, Ny, Nz), rhs, x0)
    for call in range(2):
        dr = torch.full((N,), float("nan"), dtype=torch.float64, device="cuda")
        norms = np.zeros(2)
        ok = lib.api3b_stencil_residual_noalloc(_dev(dA), _dev(dx), _dev(db), Nx, Ny, Nz, _dev(dr), dptr(norms))
        assert ok == 1, f"call {call}"
        torch.cuda.synchronize()
        assert abs(norms[0] - r0[0]) <= RTOL * r0[0], (call, norms[0], r0[0])
        assert abs(norms[1] - floor_ref) <= RTOL * floor_ref, (call, norms[1], floor_ref)
        r = dr.cpu().numpy()
        assert np.all(np.abs(r - r_ref) <= 1e-12 * np.abs(rhs).max() + RTOL * np.abs(r_ref)), call
    # sizes beyond the maximum are refused before any device access
    big = 1 << 11
    norms = np.zeros(2)
    assert lib.api3b_stencil_residual_noalloc(_dev(dA), _dev(dx), _dev(db), big, big, big, _dev(dr), dptr(norms)) == 0
    # a host output buffer, or an output that aliases an input, is refused before any launch
    host_r = np.zeros(N)
    assert lib.api3b_stencil_residual_noalloc(_dev(dA), _dev(dx), _dev(db), Nx, Ny, Nz, dptr(host_r), dptr(norms)) == 0
    assert lib.api3b_stencil_residual_noalloc(_dev(dA), _dev(dx), _dev(db), Nx, Ny, Nz, _dev(dx), dptr(norms)) == 0
    assert lib.api3b_stencil_residual_noalloc(dptr(A7), _dev(dx), _dev(db), Nx, Ny, Nz, _dev(dr), dptr(norms)) == 0
    # the refusals left the context usable: a valid call still succeeds
    assert lib.api3b_stencil_residual_noalloc(_dev(dA), _dev(dx), _dev(db), Nx, Ny, Nz, _dev(dr), dptr(norms)) == 1
    torch.cuda.synchronize()
    assert abs(norms[0] - r0[0]) <= RTOL * r0[0]
