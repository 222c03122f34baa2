"""CPU oracle of the learned sweep predictor (test infrastructure only).

numpy restatement of what the library's learned-predictor kernels compute, used by the
tests to check the GPU kernels: the 48 node features, the forward pass and the gradient
of the mean squared error.  The reference has no learned component, so this follows the
library's own definition (its header include/semisim_b200_learned.h and the kernel file's
comment), with the same BF16 rounding points: features, weights, hidden activations,
dY and dZ are rounded to BF16; products are summed here in FP64 (the kernels sum in
FP32, so results agree to FP32 summation-order differences plus the odd BF16 rounding
that lands on the other side of a tie).
"""
import numpy as np

MI, MH, MO, MOUT = 48, 128, 8, 3
OW1 = 0
OB1 = OW1 + MH * MI
OW2 = OB1 + MH
OB2 = OW2 + MH * MH
OW3 = OB2 + MH
OB3 = OW3 + MH * MH
OW4 = OB3 + MH
OB4 = OW4 + MO * MH
NPARAM = OB4 + MO


def bf16(a):
    """Round to the nearest BF16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(a.shape)


def unpack(P):
    P = np.asarray(P, dtype=np.float64 if np.asarray(P).dtype == np.float64 else np.float32)
    return (P[OW1:OB1].reshape(MH, MI), P[OB1:OW2], P[OW2:OB2].reshape(MH, MH), P[OB2:OW3],
            P[OW3:OB3].reshape(MH, MH), P[OB3:OW4], P[OW4:OB4].reshape(MO, MH), P[OB4:NPARAM])


def init_params(seed=0, out_scale=0.1):
    """PyTorch-style uniform initialisation; output rows 3-7 zero, output layer scaled."""
    rng = np.random.default_rng(seed)
    P = np.zeros(NPARAM, dtype=np.float32)

    def lin(ow, ob, nout, nin, scale=1.0):
        b = 1.0 / np.sqrt(nin)
        P[ow:ow + nout * nin] = scale * rng.uniform(-b, b, nout * nin)
        P[ob:ob + nout] = scale * rng.uniform(-b, b, nout)
    lin(OW1, OB1, MH, MI)
    lin(OW2, OB2, MH, MH)
    lin(OW3, OB3, MH, MH)
    lin(OW4, OB4, MOUT, MH, out_scale)
    return P


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def _id(a):
    return np.asarray(a, dtype=np.float64)


def forward(X, P, exact=False):
    """X [B][48] (BF16 values) -> Y [B][8], with (Z, H) of the hidden layers.  exact:
    no BF16 rounding anywhere (FP64 throughout), for finite-difference checks."""
    bf16 = _id if exact else globals()["bf16"]
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(P)
    Ws = [bf16(W1), bf16(W2), bf16(W3)]
    bs = [b1, b2, b3]
    A = np.asarray(X, dtype=np.float64)
    Zs, Hs = [], []
    for W, b in zip(Ws, bs):
        Z = A @ W.astype(np.float64).T + b
        H = bf16(silu(Z))
        Zs.append(Z)
        Hs.append(H)
        A = H.astype(np.float64)
    Y = A @ bf16(W4).astype(np.float64).T + b4
    return Y, Zs, Hs


def loss_and_grad(X, T, P, exact=False):
    """Mean squared error over B x 3 and its gradient (NPARAM), the kernels' way."""
    bf16 = _id if exact else globals()["bf16"]
    B = X.shape[0]
    if exact:
        P = np.asarray(P, dtype=np.float64)
        W1, b1, W2, b2, W3, b3, W4, b4 = (P[OW1:OB1].reshape(MH, MI), P[OB1:OW2], P[OW2:OB2].reshape(MH, MH),
                                          P[OB2:OW3], P[OW3:OB3].reshape(MH, MH), P[OB3:OW4],
                                          P[OW4:OB4].reshape(MO, MH), P[OB4:NPARAM])
    else:
        W1, b1, W2, b2, W3, b3, W4, b4 = unpack(P)
    Y, Zs, Hs = forward(X, P, exact)
    d = Y[:, :MOUT] - T
    loss = float((d ** 2).sum() / (3.0 * B))
    dY = np.zeros((B, MO))
    dY[:, :MOUT] = bf16(2.0 * d / (3.0 * B))
    G = np.zeros(NPARAM)
    dH = dY @ bf16(W4).astype(np.float64)
    Wb = [bf16(W1), bf16(W2), bf16(W3)]
    dZs = [None] * 3
    for L in (2, 1, 0):
        dZ = bf16(dH * dsilu(Zs[L])).astype(np.float64)
        dZs[L] = dZ
        if L > 0:
            dH = dZ @ Wb[L].astype(np.float64)
    Ain = [np.asarray(X, np.float64), Hs[0].astype(np.float64), Hs[1].astype(np.float64)]
    for L, (ow, ob) in enumerate(((OW1, OB1), (OW2, OB2), (OW3, OB3))):
        G[ow:ob] = (dZs[L].T @ Ain[L]).ravel()
        G[ob:ob + MH] = dZs[L].sum(0)
    G[OW4:OB4] = (dY.T @ Hs[2].astype(np.float64)).ravel()
    G[OB4:NPARAM] = dY.sum(0)
    return loss, G, Y


def features(shape, x1, x0, s, dv, VT, Nd, Na, kind, con):
    """The 48 features of every node (float64, before BF16 rounding).  x1, x0: (3, N)
    psi, phi_n, phi_p; shape (Nx, Ny, Nz); nodes x fastest."""
    Nx, Ny, Nz = shape
    N = Nx * Ny * Nz

    def nbrs(a):
        a = a.reshape(Nz, Ny, Nx)
        out = [a]
        for ax in (2, 1, 0):                      # x, y, z
            for sgn in (-1, +1):                  # minus neighbour, then plus
                b = np.roll(a, -sgn, axis=ax)     # b[i] = a[i + sgn]
                idx = [slice(None)] * 3
                idx[ax] = 0 if sgn < 0 else -1
                b[tuple(idx)] = a[tuple(idx)]
                out.append(b)
        return [o.ravel() for o in out]
    f = np.zeros((N, MI))
    d = (x1 - x0) / VT
    u1 = (x1[0] - x1[1]) / (40.0 * VT)
    u2 = (x1[2] - x1[0]) / (40.0 * VT)
    for c in range(3):
        for q, v in enumerate(nbrs(d[c])):
            f[:, 7 * c + q] = v
    for q, v in enumerate(nbrs(u1)):
        f[:, 21 + q] = v
    for q, v in enumerate(nbrs(u2)):
        f[:, 28 + q] = v
    f[:, 35] = np.float32(s)
    for q in range(4):
        f[:, 36 + q] = np.float32(dv[q]) / VT * 0.1
    f[:, 40] = np.arcsinh((Nd - Na) * 1e-22) * 0.1
    f[:, 41] = (kind == 0)
    f[:, 42] = (con > 0)
    f[:, 43] = 1.0
    return f
