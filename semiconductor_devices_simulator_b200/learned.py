"""Learned sweep predictor: training data from the solver's own sweeps, training on the
GPU with the library's kernels, and the model files.

The network (48 node features -> 3 x 128 SiLU -> 3, BF16 weights, FP32 accumulation)
corrects the sweep predictor's linear guess x1 + s (x1 - x0) of (psi, phi_n, phi_p) at
the first continuation step of each new bias point; the Gummel loop then converges to
its usual tolerance (api3b_seed_* in include/semisim_b200.h).

Training data: consecutive converged bias points (x0, x1, x2) of sweeps the solver
itself runs; the features of (x0, x1) come from the library's feature kernel
(b200m_seed_features), the target is (x2 - x1 - s (x1 - x0)) / VT.  Training: the
library's forward / backward / Adam kernels (b200m_mlp_*) on device buffers.  PyTorch
only provides the device memory, the stream and the random batch indices.
"""
import ctypes
import math
import time

import numpy as np

from . import devices as D

MI, MH, MO, MOUT = 48, 128, 8, 3


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream(torch):
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def init_params(nparam, seed=0, out_scale=0.1):
    """PyTorch-style uniform initialisation (output rows 3-7 zero, output layer scaled so
    the untrained correction starts near zero)."""
    rng = np.random.default_rng(seed)
    P = np.zeros(nparam, dtype=np.float32)
    off = 0

    def lin(nout, nin, rows_used=None, scale=1.0):
        nonlocal off
        b = 1.0 / math.sqrt(nin)
        W = np.zeros((nout, nin), dtype=np.float32)
        ru = nout if rows_used is None else rows_used
        W[:ru] = scale * rng.uniform(-b, b, (ru, nin))
        P[off:off + nout * nin] = W.ravel()
        off += nout * nin
        bb = np.zeros(nout, dtype=np.float32)
        bb[:ru] = scale * rng.uniform(-b, b, ru)
        P[off:off + nout] = bb
        off += nout
    lin(MH, MI)
    lin(MH, MH)
    lin(MH, MH)
    lin(MO, MH, rows_used=MOUT, scale=out_scale)
    assert off == nparam
    return P


def collect(lib, w, sweep):
    """Run one sweep (api3_solve at the first point, api3_resolve after) and return the
    contact voltages (npts, ncon) and converged (psi, phi_n, phi_p) of every point,
    (npts, 3, N) float64."""
    nc = lib.api3_get_ncon()
    Vs, X = [], []
    ok = D.start_sweep(lib, w, sweep)

    def grab(q, v):
        Vs.append([lib.api3_get_contact_Vsolved(c) for c in range(nc)])
        X.append(np.stack([D.field(lib, k, w.shape).ravel() for k in (0, 15, 16)]))
    V, I, F, conv = D.run_sweep(lib, w, sweep, on_point=grab)
    return np.array(Vs), np.array(X), bool(ok and conv.all())


def step_ratio(V0, V1, V2):
    """Extrapolation ratio of the sweep predictor for the step V1 -> V2 after V0 -> V1
    (the least-squares ratio of the voltage steps, as the solver computes it)."""
    b = V1 - V0
    a = V2 - V1
    den = float(b @ b)
    return float(a @ b) / den if den > 0 else 0.0


def pair_data(lib, torch, Vs, X, per_pair=None, seed=0):
    """Features (BF16 [M][48]) and targets (FP32 [M][3]) of every consecutive triple of
    points; per_pair nodes sampled at random per triple (all when None)."""
    dev = torch.device("cuda")
    VT = lib.b200x_vtref()
    g = torch.Generator(device="cpu").manual_seed(seed)
    N = X.shape[2]
    feats, targs = [], []
    Xf = torch.empty((N, MI), dtype=torch.bfloat16, device=dev)
    for k in range(1, X.shape[0] - 1):
        s = step_ratio(Vs[k - 1], Vs[k], Vs[k + 1])
        dv = np.zeros(4)
        d = Vs[k + 1] - Vs[k]
        dv[:min(4, len(d))] = d[:4]
        x0 = torch.tensor(X[k - 1], device=dev)
        x1 = torch.tensor(X[k], device=dev)
        x2 = torch.tensor(X[k + 1], device=dev)
        ok = lib.b200m_seed_features(_ptr(x1[0]), _ptr(x1[1]), _ptr(x1[2]), _ptr(x0[0]), _ptr(x0[1]), _ptr(x0[2]),
                                     s, dv.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), _ptr(Xf), _stream(torch))
        if not ok:
            raise RuntimeError("b200m_seed_features failed")
        tgt = ((x2 - x1 - s * (x1 - x0)) / VT).T.float()
        if per_pair is not None and per_pair < N:
            idx = torch.randperm(N, generator=g)[:per_pair].to(dev)
            feats.append(Xf.index_select(0, idx))
            targs.append(tgt.index_select(0, idx).contiguous())
        else:
            feats.append(Xf.clone())
            targs.append(tgt.contiguous())
    return torch.cat(feats), torch.cat(targs)


class Trainer:
    """Adam training of the predictor with the library's kernels."""

    def __init__(self, lib, torch, batch=16384, seed=0, params=None):
        self.lib, self.torch, self.B = lib, torch, batch
        n, nw, nb = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        lib.b200m_mlp_sizes(ctypes.byref(n), ctypes.byref(nw), ctypes.byref(nb))
        self.nparam = n.value
        dev = torch.device("cuda")
        P0 = init_params(self.nparam, seed) if params is None else np.asarray(params, np.float32)
        f32 = dict(dtype=torch.float32, device=dev)
        self.P = torch.tensor(P0, **f32)
        self.M = torch.zeros(self.nparam, **f32)
        self.V = torch.zeros(self.nparam, **f32)
        self.G = torch.zeros(self.nparam, **f32)
        self.Wb = torch.zeros(nw.value, dtype=torch.bfloat16, device=dev)
        self.bias = torch.zeros(nb.value, **f32)
        B = batch
        self.Y = torch.zeros((B, MO), **f32)
        self.Z = torch.zeros((3, B, MH), **f32)
        self.H = torch.zeros((3, B, MH), dtype=torch.bfloat16, device=dev)
        self.dZ = torch.zeros((3, B, MH), dtype=torch.bfloat16, device=dev)
        self.dY = torch.zeros((B, MO), dtype=torch.bfloat16, device=dev)
        self.loss = torch.zeros(1, **f32)
        self.t = 0
        self._check(lib.b200m_mlp_pack(_ptr(self.P), _ptr(self.Wb), _ptr(self.bias), _stream(torch)))

    @staticmethod
    def _check(ok):
        if not ok:
            raise RuntimeError("learned-predictor kernel launch failed")

    def grad(self, X, T):
        """Loss and gradient (in self.G) of a batch of exactly `batch` rows."""
        lib, torch = self.lib, self.torch
        st = _stream(torch)
        self.G.zero_()
        self.loss.zero_()
        B = X.shape[0]
        self._check(lib.b200m_mlp_forward(_ptr(X), B, _ptr(self.Wb), _ptr(self.bias), _ptr(self.Y), _ptr(self.Z),
                                          _ptr(self.H), st))
        self._check(lib.b200m_mlp_backward(_ptr(X), B, _ptr(self.Wb), _ptr(self.Y), _ptr(T), _ptr(self.Z),
                                           _ptr(self.H), _ptr(self.dZ), _ptr(self.dY), _ptr(self.G),
                                           _ptr(self.loss), st))

    def step(self, X, T, lr):
        self.grad(X, T)
        self.t += 1
        self._check(self.lib.b200m_mlp_adam(_ptr(self.P), _ptr(self.G), _ptr(self.M), _ptr(self.V), lr, self.t,
                                            _ptr(self.Wb), _ptr(self.bias), _stream(self.torch)))

    def fit(self, Xall, Tall, steps=2000, lr=1e-3, lr_end=1e-4, seed=0, log_every=0):
        torch = self.torch
        g = torch.Generator(device="cuda").manual_seed(seed)
        n = Xall.shape[0]
        hist = []
        t0 = time.time()
        for i in range(steps):
            idx = torch.randint(0, n, (self.B,), device="cuda", generator=g)
            Xb = Xall.index_select(0, idx)
            Tb = Tall.index_select(0, idx)
            lr_i = lr_end + 0.5 * (lr - lr_end) * (1.0 + math.cos(math.pi * i / max(steps - 1, 1)))
            self.step(Xb, Tb, lr_i)
            if log_every and (i % log_every == 0 or i == steps - 1):
                hist.append((i, float(self.loss.item())))
        torch.cuda.synchronize()
        self.seconds = time.time() - t0
        return hist

    def params(self):
        return self.P.detach().cpu().numpy().copy()

    def evaluate(self, Xall, Tall):
        """Per-channel RMS of the linear guess's error (the targets) and of the learned
        guess's error (targets - outputs) over a data set, in units of VT."""
        torch = self.torch
        n = Xall.shape[0]
        s_lin = torch.zeros(3, dtype=torch.float64, device="cuda")
        s_mlp = torch.zeros(3, dtype=torch.float64, device="cuda")
        for a in range(0, n, self.B):
            b = min(n, a + self.B)
            X, T = Xall[a:b].contiguous(), Tall[a:b].contiguous()
            self.grad(X, T)
            Y = self.Y[:b - a, :3]
            s_lin += (T.double() ** 2).sum(0)
            s_mlp += ((T - Y).double() ** 2).sum(0)
        return (s_lin / n).sqrt().cpu().numpy(), (s_mlp / n).sqrt().cpu().numpy()


def load(lib, params):
    """Load a model into the calling thread's current instance (after its first solve)."""
    P = np.ascontiguousarray(params, dtype=np.float32)
    ok = lib.api3b_seed_set_model(P.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), P.size)
    if not ok:
        raise RuntimeError("api3b_seed_set_model failed (wrong size, or the instance has not solved yet)")


def stats(lib):
    a, b = ctypes.c_longlong(0), ctypes.c_longlong(0)
    lib.api3b_seed_stats(ctypes.byref(a), ctypes.byref(b))
    return a.value, b.value
