"""FP64 numpy restatement of the learned stencil smoother (test infrastructure).

The learned smoother has no counterpart in the reference, so this file is
pinned by finite differences (tests/test_learned_oracle.py) and serves as the
checker of the device kernels in parmoon_b200/csrc/learned.cu:

  features  F[k][L] = a(i, nb_k(i)) / a(i, i) for active rows i at node L
  network   three 3x3x3 convolutions with zero padding, 27 -> 32 (ReLU) -> 32
            (ReLU) -> 27; parameters flat [W1 b1 W2 b2 W3 b3], W[c_out][c_in][27];
            the device rounds weights and every layer's input to BF16
  stencil   W_k(L) = out3[k][L] / a(i, i)  (0 on Dirichlet nodes)
  loss      |A (e - S r)|^2 / |r|^2 for one pair (e, r = A e), S r = sum_k W_k r(nb_k)
"""
import numpy as np

C0, C1, C2, C3 = 27, 32, 32, 27
SIZES = [C1 * C0 * 27, C1, C2 * C1 * 27, C2, C3 * C2 * 27, C3]


def n_params():
    return sum(SIZES)


def unpack(theta):
    out, o = [], 0
    for s in SIZES:
        out.append(theta[o:o + s])
        o += s
    W1, b1, W2, b2, W3, b3 = out
    return (W1.reshape(C1, C0, 27), b1, W2.reshape(C2, C1, 27), b2, W3.reshape(C3, C2, 27), b3)


def offsets():
    return [((k % 3) - 1, (k // 3) % 3 - 1, k // 9 - 1) for k in range(27)]


def shift(x, o):
    """y[.., i, j, k] = x[.., i+o0, j+o1, k+o2] with zero padding; arrays indexed [c, k, j, i]."""
    di, dj, dk = o
    y = np.zeros_like(x)
    n = x.shape[-1]
    src = lambda d: slice(max(d, 0), n + min(d, 0))
    dst = lambda d: slice(max(-d, 0), n - max(d, 0))
    y[..., dst(dk), dst(dj), dst(di)] = x[..., src(dk), src(dj), src(di)]
    return y


def conv(x, W, b):
    """x [cin, n, n, n] -> [cout, n, n, n]; W [cout, cin, 27]."""
    out = np.broadcast_to(b[:, None, None, None], (W.shape[0],) + x.shape[1:]).copy()
    for k, o in enumerate(offsets()):
        xs = shift(x, o)
        out += np.tensordot(W[:, :, k], xs, axes=([1], [0]))
    return out


def conv_bwd(dz, x, W):
    """Gradients of conv w.r.t. x, W, b given dL/dout = dz."""
    dx = np.zeros_like(x)
    dW = np.zeros_like(W)
    for k, o in enumerate(offsets()):
        xs = shift(x, o)
        dW[:, :, k] = np.tensordot(dz, xs, axes=([1, 2, 3], [1, 2, 3]))
        # out(L) += W x(L + o) -> x(L) receives dz(L - o)
        dx += np.tensordot(W[:, :, k].T, shift(dz, tuple(-v for v in o)), axes=([1], [0]))
    db = dz.sum(axis=(1, 2, 3))
    return dx, dW, db


def features(n1, rowptr, kcol, A, Na, dof_lat):
    N = rowptr.size - 1
    F = np.zeros((27, n1, n1, n1))
    dscale = np.zeros((n1, n1, n1))
    ijk = np.stack([dof_lat % n1, (dof_lat // n1) % n1, dof_lat // (n1 * n1)], axis=1)
    for r in range(Na):
        cols = kcol[rowptr[r]:rowptr[r + 1]]
        vals = A[rowptr[r]:rowptr[r + 1]]
        diag = vals[cols == r][0]
        i, j, k = ijk[r]
        for c, v in zip(cols, vals):
            d = ijk[c] - ijk[r]
            if np.all(np.abs(d) <= 1):
                kk = (d[0] + 1) + 3 * (d[1] + 1) + 9 * (d[2] + 1)
                F[kk, k, j, i] = v / diag
        dscale[k, j, i] = 1.0 / diag
    return F, dscale


def forward(theta, F, dscale, act_bf16=True):
    """The network on the feature lattice.  act_bf16: every layer's input is
    rounded to BF16 as the device stores it (the features, and the ReLU
    outputs of the hidden layers); False gives the unrounded function whose
    gradient the finite-difference test pins."""
    rnd = bf16_round if act_bf16 else (lambda x: x)
    W1, b1, W2, b2, W3, b3 = unpack(theta)
    F = rnd(F)
    z1 = conv(F, W1, b1)
    a1 = rnd(np.maximum(z1, 0))
    z2 = conv(a1, W2, b2)
    a2 = rnd(np.maximum(z2, 0))
    out3 = conv(a2, W3, b3)
    Wst = out3 * dscale[None]
    return Wst, (F, z1, a1, z2, a2, out3)


def to_lattice(v, dof_lat, n1):
    x = np.zeros(n1 ** 3)
    x[dof_lat] = v
    return x.reshape(n1, n1, n1)  # [k, j, i]


def apply_stencil(Wst, rl):
    c = np.zeros_like(rl)
    for k, o in enumerate(offsets()):
        c += Wst[k] * shift(rl, o)
    return c


def loss_and_grad(theta, n1, rowptr, kcol, A, Na, dof_lat, e, r, act_bf16=True):
    """Returns (loss, dloss/dtheta) for one pair (e, r).  With act_bf16 the
    forward rounds the layer inputs to BF16 and the gradient passes the
    rounding as the identity (the weight gradients use the rounded inputs),
    as the device's backward does."""
    N = rowptr.size - 1
    F, dscale = features(n1, rowptr, kcol, A, Na, dof_lat)
    Wst, (F, z1, a1, z2, a2, out3) = forward(theta, F, dscale, act_bf16)
    rl = to_lattice(r, dof_lat, n1)
    cl = apply_stencil(Wst, rl).reshape(-1)
    c = cl[dof_lat]
    c[Na:] = 0.0
    u = e - c
    rows = np.repeat(np.arange(N), np.diff(rowptr))
    Ad = np.zeros((N, N))
    Ad[rows, kcol] = A
    v = Ad @ u
    rr = float(r @ r)
    loss = float(v @ v) / rr
    dv = 2 * v / rr
    du = Ad.T @ dv
    dc = -du
    dc[Na:] = 0.0
    dcl = to_lattice(dc, dof_lat, n1)
    dout3 = np.zeros_like(out3)
    for k, o in enumerate(offsets()):
        dout3[k] = dcl * shift(rl, o) * dscale
    W1, b1, W2, b2, W3, b3 = unpack(theta)
    da2, dW3, db3 = conv_bwd(dout3, a2, W3)
    dz2 = da2 * (z2 > 0)
    da1, dW2, db2 = conv_bwd(dz2, a1, W2)
    dz1 = da1 * (z1 > 0)
    _, dW1, db1 = conv_bwd(dz1, F, W1)
    g = np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dW3.ravel(), db3])
    return loss, g


def stencil(theta, n1, rowptr, kcol, A, Na, dof_lat, act_bf16=True):
    F, dscale = features(n1, rowptr, kcol, A, Na, dof_lat)
    Wst, _ = forward(theta, F, dscale, act_bf16)
    return Wst  # [27, k, j, i] == channel-major lattice order


def bf16_round(x):
    """Round FP32 values to BF16 (round to nearest even) and back, as the device stores weights."""
    x = np.asarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16 << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)
