"""The learned sweep predictor on the GPU, checked against the CPU oracle (oracle/mlp.py):
its feature kernel, the fused seed kernel (features + BF16 MLP + seed write), the
training forward / backward kernels (loss, outputs and gradients), and what the trained
network gains over the linear guess on held-out MOSFET sweeps.

Tolerances: features to one BF16 rounding step; outputs, loss and gradients to 2 %
norm-wise (BF16 operands, FP32 sums on the GPU against FP64 sums in the oracle).
"""
import ctypes
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import semiconductor_devices_simulator_b200 as S  # noqa: E402
from semiconductor_devices_simulator_b200 import devices as D, learned as LR  # noqa: E402
from semiconductor_devices_simulator_b200.abi import dptr, iptr  # noqa: E402
from oracle import mlp as M  # noqa: E402

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def lib():
    return S.load()


def small_mos(lib, n=(24, 16, 12)):
    w = D.nmosfet(lib, n=n, vds=(1.0,))
    assert D.start_sweep(lib, w, w.sweeps[0])
    return w


def device_arrays(lib, w):
    N = w.N
    kind = np.zeros(N, np.int32); con = np.zeros(N, np.int32); gate = np.zeros(N, np.int32)
    assert lib.b200x_masks(iptr(kind), iptr(con), iptr(gate), None) == 1
    net = np.zeros(N)
    lib.api3_bulk_copy(14, dptr(net))
    return kind, con, net


def random_history(w, seed):
    rng = np.random.default_rng(seed)
    N = w.N
    x1 = np.stack([rng.uniform(-0.5, 1.0, N), rng.uniform(-0.2, 0.2, N), rng.uniform(-0.2, 0.2, N)])
    x0 = x1 + rng.normal(0.0, 0.02, (3, N))
    return x1, x0


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


def test_feature_kernel_matches_oracle(lib):
    w = small_mos(lib)
    kind, con, net = device_arrays(lib, w)
    x1, x0 = random_history(w, 1)
    s, dv = 0.8, np.array([0.0, 0.05, 0.0, 0.0])
    d1 = torch.tensor(x1, device="cuda")
    d0 = torch.tensor(x0, device="cuda")
    X = torch.zeros((w.N, M.MI), dtype=torch.bfloat16, device="cuda")
    P = LR._ptr
    assert lib.b200m_seed_features(P(d1[0]), P(d1[1]), P(d1[2]), P(d0[0]), P(d0[1]), P(d0[2]), s,
                                   dv.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), P(X), None)
    torch.cuda.synchronize()
    got = X.float().cpu().numpy()
    ref = M.bf16(M.features(w.shape, x1, x0, s, dv, lib.b200x_vtref(), net, 0.0, kind, con))
    err = np.abs(got - ref)
    assert (err <= 2.0 ** -7 * np.abs(ref) + 1e-6).all(), err.max()


def test_forward_backward_match_oracle(lib):
    small_mos(lib)                                  # a current instance (the kernels need none)
    B = 200                                         # ragged: not a multiple of the 64-row tile
    rng = np.random.default_rng(2)
    Xh = M.bf16(rng.normal(0.0, 1.0, (B, M.MI)))
    Th = rng.normal(0.0, 0.5, (B, 3)).astype(np.float32)
    P0 = LR.init_params(M.NPARAM, seed=3, out_scale=1.0)
    tr = LR.Trainer(lib, torch, batch=B, params=P0)
    Xd = torch.tensor(Xh, dtype=torch.bfloat16, device="cuda")
    Td = torch.tensor(Th, device="cuda")
    tr.grad(Xd, Td)
    torch.cuda.synchronize()
    loss, G, Y = M.loss_and_grad(Xh, Th, P0)
    assert rel(tr.Y[:, :3].cpu().numpy(), Y[:, :3]) < 2e-2
    assert abs(tr.loss.item() - loss) <= 2e-2 * loss
    Gg = tr.G.cpu().numpy()
    for a, b, name in ((M.OW1, M.OB1, "W1"), (M.OB1, M.OW2, "b1"), (M.OW2, M.OB2, "W2"), (M.OB2, M.OW3, "b2"),
                       (M.OW3, M.OB3, "W3"), (M.OB3, M.OW4, "b3"), (M.OW4, M.OB4, "W4"), (M.OB4, M.NPARAM, "b4")):
        assert rel(Gg[a:b], G[a:b]) < 2e-2, name


def test_seed_kernel_matches_oracle(lib):
    w = small_mos(lib)
    kind, con, net = device_arrays(lib, w)
    x1, x0 = random_history(w, 4)
    for c in range(3):
        assert lib.b200x_set(S.ST_H1 + c, dptr(np.ascontiguousarray(x1[c]))) == 1
        assert lib.b200x_set(S.ST_E2 + c, dptr(np.ascontiguousarray(x0[c]))) == 1
    P0 = LR.init_params(M.NPARAM, seed=5, out_scale=1.0)
    LR.load(lib, P0)
    lib.api3b_seed_enable(0)                        # the hook runs the kernel itself
    s, dv = 1.0, np.array([0.0, 0.0, 0.05, 0.0])
    assert lib.b200x_seed_run(s, dv.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) == 1
    got = np.stack([np.zeros(w.N) for _ in range(3)])
    for c in range(3):
        assert lib.b200x_get(c, dptr(got[c])) == 1
    VT = lib.b200x_vtref()
    F = M.bf16(M.features(w.shape, x1, x0, s, dv, VT, net, 0.0, kind, con))
    Y, _, _ = M.forward(F, P0)
    lin = x1 + s * (x1 - x0)
    assert rel((got - lin) / VT, Y[:, :3].T) < 2e-2


def test_training_reduces_loss(lib):
    small_mos(lib)
    B, n = 4096, 65536
    g = torch.Generator(device="cuda").manual_seed(6)
    X = torch.randn((n, M.MI), generator=g, device="cuda").to(torch.bfloat16)
    A = torch.randn((M.MI, 3), generator=g, device="cuda") / 8.0
    T = torch.tanh(X.float() @ A).contiguous()
    tr = LR.Trainer(lib, torch, batch=B, seed=7)
    hist = tr.fit(X, T, steps=300, lr=2e-3, lr_end=2e-4, log_every=50)
    assert hist[-1][1] < 0.2 * hist[0][1], hist


def sweep(lib, w, s, seeded, params=None):
    """One Id-Vg sweep; returns currents, Gummel iterations, converged flags."""
    assert D.start_sweep(lib, w, s)
    if params is not None:
        LR.load(lib, params)
    lib.api3b_seed_enable(1 if seeded else 0)
    g0 = lib.api3_get_stat(3)
    V, I, F, conv = D.run_sweep(lib, w, s)
    return I, F, lib.api3_get_stat(3) - g0, conv


def test_trained_seed_gains_over_linear_guess(lib):
    """Trained on the solver's own solutions at gate voltages half a step off the test
    sweeps' (Vd = 0.05 and 1 V, 60x40x30 n-MOSFET), the network's guess of the next bias
    point is at least twice as close to the converged solution as the linear guess on the
    held-out sweeps (RMS over nodes, points and the three fields; each of psi, phi_n and
    phi_p at least 30 % closer).  Seeding
    the Vd = 1 V sweep with it, every point converges and the on-state drain current is the
    same to 1e-4; the Gummel iterations of both runs are printed.  The same points started
    each from its own converged solution take fewer iterations than either guess: the room a
    better seed would have."""
    w = D.nmosfet(lib, n=(60, 40, 30), vds=(0.05, 1.0))
    lib.api3b_seed_enable(0)

    def data(shift):
        F, T = [], []
        for s in w.sweeps:
            s2 = dict(s)
            s2["V"] = np.round(s["V"] + shift, 12)
            Vs, Xs, ok = LR.collect(lib, w, s2)
            assert ok
            f, t = LR.pair_data(lib, torch, Vs, Xs)
            F.append(f)
            T.append(t)
        return torch.cat(F), torch.cat(T)
    Ftr, Ttr = data(0.025)
    Fte, Tte = data(0.0)
    tr = LR.Trainer(lib, torch, batch=16384, seed=0)
    tr.fit(Ftr, Ttr, steps=6000, lr=1e-3, lr_end=1e-4)
    lin, mlp = tr.evaluate(Fte, Tte)
    print(f"held-out RMS error / VT (psi, phi_n, phi_p): linear {lin}, learned {mlp}")
    assert np.linalg.norm(mlp) < 0.5 * np.linalg.norm(lin), (lin, mlp)
    assert (mlp < 0.7 * lin).all(), (lin, mlp)
    params = tr.params()
    test = w.sweeps[1]
    I0, F0, its0, c0 = sweep(lib, w, test, False)
    u0, f0 = LR.stats(lib)
    try:
        I1, F1, its1, c1 = sweep(lib, w, test, True, params)
    finally:
        lib.api3b_seed_enable(0)
    used, fb = LR.stats(lib)
    print(f"Gummel iterations: linear guess {its0}, learned guess {its1} "
          f"(seeded steps {used - u0}, redone from the linear guess {fb - f0})")
    assert c0.all() and c1.all()
    assert used - u0 > 0
    on = np.abs(I0[:, 1]) > 1e-9
    assert on.any()
    d = np.abs(I1[on, 1] - I0[on, 1]) / np.abs(I0[on, 1])
    assert d.max() <= 1e-4, d.max()
    # what any seed could save: each point re-solved from its own converged solution
    floor = converged_start_floor(lib, w, test)
    print(f"Gummel iterations from converged starts: {floor}")
    assert floor < its0 and floor < its1, (floor, its0, its1)


def converged_start_floor(lib, w, s):
    """Gummel iterations of the sweep's points (after its first) when each starts from its
    own converged solution: api3_set_state at the point's bias, then api3_resolve, whose
    Gummel loop runs until the acceptance test passes.  No starting guess can do better."""
    assert D.start_sweep(lib, w, s)
    states = []
    for v in s["V"][1:]:
        for cid, vv in D.bias_vector(w, s, v).items():
            lib.api3_set_contact_V(cid, vv)
        assert lib.api3_resolve() == 1
        st = [np.empty(w.N) for _ in range(3)]
        lib.api3_get_state(*(dptr(x) for x in st))
        states.append(st)
    tot = 0
    for v, st in zip(s["V"][1:], states):
        for cid, vv in D.bias_vector(w, s, v).items():
            lib.api3_set_contact_V(cid, vv)
        lib.api3_set_state(*(dptr(x) for x in st))
        g0 = lib.api3_get_stat(3)
        assert lib.api3_resolve() == 1
        tot += lib.api3_get_stat(3) - g0
    return tot
