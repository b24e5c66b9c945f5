"""Learned preconditioner and Teter-Payne-Allan preconditioner (oracle; test infrastructure only).

The reference has no learned preconditioner: its correction step is r_i / (|k+G_i|^2 - lambda)
(src/features/linalg/lobpcg/common.zig:214-226).  This module restates, in float64 numpy, the
arithmetic of the library's alternative preconditioners so the CUDA forward and backward kernels
can be checked against it (and it against finite differences):

  TPA   q_i = K(x_i) r_i,  x_i = |k+G_i|^2 / E_kin,b,
        K(x) = (27 + 18x + 12x^2 + 8x^3) / (27 + 18x + 12x^2 + 8x^3 + 16x^4)
        (Teter, Payne, Allan, Phys. Rev. B 40, 12255 (1989))
  MLP   q_i = m(u_i) r_i,  u = (log(x + 0.05), log(|r_i| / rms(r) + 1e-6), min(t / 20, 2)),
        h1 = tanh(W1 u + b1), h2 = tanh(W2 h1 + b2), z = w3 . h2 + b3   (3 -> 64 -> 64 -> 1),
        m = K(x) exp(clamp(z, -8, 8)) with x = exp(u0) - 0.05 (a refinement of TPA)
  loss  L = mean_b [1 - |A_b|^2 / (Q_b D_b)],  A_b = sum_i m_i c_i,  Q_b = sum_i m_i^2 w_i,
        c_i = conj(r_i) delta_i, w_i = |r_i|^2, D_b = ||delta_b||^2.

Parameter vector layout (4481 floats): W1[64][3], b1[64], W2[64][64] (row = output), b2[64], w3[64], b3.
"""
from __future__ import annotations

import numpy as np

H = 64
NPARAM = H * 3 + H + H * H + H + H + 1


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    W1 = p[o:o + H * 3].reshape(H, 3); o += H * 3
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    w3 = p[o:o + H]; o += H
    b3 = p[o]
    return W1, b1, W2, b2, w3, b3


def pack(W1, b1, W2, b2, w3, b3):
    return np.concatenate([W1.ravel(), b1, W2.ravel(), b2, w3, [b3]])


def features(kin, ekin, rabs, rms, t):
    x = kin / max(ekin, 1e-6)
    return np.stack([np.log(x + 0.05), np.log(rabs / max(rms, 1e-300) + 1e-6), np.full_like(x, min(t / 20.0, 2.0))], axis=1)


def tpa(x):
    num = 27.0 + x * (18.0 + x * (12.0 + 8.0 * x))
    return num / (num + 16.0 * x ** 4)


def softplus(z):
    return np.where(z > 20.0, z, np.log1p(np.exp(np.minimum(z, 20.0))))


def forward(p, u):
    W1, b1, W2, b2, w3, b3 = unpack(p)
    h1 = np.tanh(u @ W1.T + b1)
    h2 = np.tanh(h1 @ W2.T + b2)
    z = h2 @ w3 + b3
    return z, h1, h2


def _mult(u0, z):
    x = np.maximum(np.exp(u0) - 0.05, 0.0)
    return tpa(x) * np.exp(np.clip(z, -8.0, 8.0))


def multiplier(p, u):
    return _mult(u[:, 0], forward(p, u)[0])


def loss_grad(p, off, feat, cc, w, dnorm):
    """Loss and gradient over the bands [off[b], off[b+1]) of the sample arrays."""
    off = np.asarray(off)
    nb = len(off) - 1
    z, h1, h2 = forward(p, feat)
    m = _mult(feat[:, 0], z)
    sig = np.where((z > -8.0) & (z < 8.0), m, 0.0)  # dm/dz
    W1, b1, W2, b2, w3, b3 = unpack(p)
    band = np.repeat(np.arange(nb), np.diff(off))
    A = np.bincount(band, weights=m * cc.real, minlength=nb) + 1j * np.bincount(band, weights=m * cc.imag, minlength=nb)
    Q = np.maximum(np.bincount(band, weights=m * m * w, minlength=nb), 1e-300)
    D = np.maximum(dnorm, 1e-300)
    L = float(np.mean(1.0 - np.abs(A) ** 2 / (Q * D)))
    Ab, Qb, Db = A[band], Q[band], D[band]
    re = (np.conj(Ab) * cc).real
    dm = -2.0 / (Db * Qb) * (re - np.abs(Ab) ** 2 / Qb * m * w) / nb
    dz = dm * sig
    gw3 = dz @ h2
    gb3 = dz.sum()
    da2 = dz[:, None] * w3[None, :] * (1.0 - h2 ** 2)
    gW2 = da2.T @ h1
    gb2 = da2.sum(axis=0)
    da1 = (da2 @ W2) * (1.0 - h1 ** 2)
    gW1 = da1.T @ feat
    gb1 = da1.sum(axis=0)
    return L, pack(gW1, gb1, gW2, gb2, gw3, gb3)


def random_problem(nbands=6, per_band=(40, 90), seed=0):
    """A small random sample set (for gradient checks)."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(per_band[0], per_band[1], size=nbands)
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)
    n = int(off[-1])
    kin = rng.uniform(0.0, 20.0, n)
    feat = np.stack([np.log(kin / 3.0 + 0.05), rng.normal(-1.0, 1.0, n), np.full(n, 0.25)], axis=1)
    r = rng.normal(size=n) + 1j * rng.normal(size=n)
    delta = r * (1.0 / (1.0 + kin)) + 0.1 * (rng.normal(size=n) + 1j * rng.normal(size=n))
    cc = np.conj(r) * delta
    w = np.abs(r) ** 2
    dnorm = np.bincount(np.repeat(np.arange(nbands), sizes), weights=np.abs(delta) ** 2)
    return off, feat, cc, w, dnorm


def init_params(seed=0, scale=0.3):
    rng = np.random.default_rng(seed)
    W1 = rng.normal(0.0, scale, (H, 3))
    b1 = rng.normal(0.0, scale, H)
    W2 = rng.normal(0.0, scale / np.sqrt(H), (H, H))
    b2 = rng.normal(0.0, scale, H)
    w3 = rng.normal(0.0, scale / np.sqrt(H), H)
    return pack(W1, b1, W2, b2, w3, 0.5)


# ---- Fourier neural operator for the first SCF density -------------------------------------------
# The same network as the library's (4 Fourier layers, 16 modes per axis f = -8..7, 8 channels,
# GELU in tanh form after layers 0-2, partial DFTs over the kept modes, real part of the inverse),
# written with torch float64 on the CPU so its gradient comes from autograd: an independent check of
# the hand-written backward kernels.

FNO_W, FNO_M, FNO_L, FNO_IN = 8, 16, 4, 2
FNO_K = FNO_M ** 3
FNO_LAYER = 2 * FNO_K * FNO_W * FNO_W + FNO_W * FNO_W + FNO_W
FNO_NPARAM = FNO_W * FNO_IN + FNO_W + FNO_L * FNO_LAYER + FNO_W + 1


def _fno_twiddle(n, torch):
    f = np.arange(FNO_M) - FNO_M // 2
    x = np.arange(n)
    r = np.mod(np.outer(f, x), n)
    return torch.tensor(np.exp(-2j * np.pi * r / n))  # [16][n]


def fno_forward_torch(params, u, dims):
    """params: torch float64 vector (may require grad); u: [2][nx ny nz] -> [nx ny nz]."""
    import torch

    nx, ny, nz = dims
    P = params
    o = 0
    Pw = P[o:o + FNO_W * FNO_IN].reshape(FNO_W, FNO_IN); o += FNO_W * FNO_IN
    Pb = P[o:o + FNO_W]; o += FNO_W
    tx, ty, tz = _fno_twiddle(nx, torch), _fno_twiddle(ny, torch), _fno_twiddle(nz, torch)
    uu = torch.as_tensor(u, dtype=torch.float64).reshape(FNO_IN, nz, ny, nx)
    v = torch.einsum("oi,izyx->ozyx", Pw, uu) + Pb[:, None, None, None]
    for l in range(FNO_L):
        R = P[o:o + 2 * FNO_K * FNO_W * FNO_W].reshape(FNO_K, FNO_W, FNO_W, 2); o += 2 * FNO_K * FNO_W * FNO_W
        Wl = P[o:o + FNO_W * FNO_W].reshape(FNO_W, FNO_W); o += FNO_W * FNO_W
        bl = P[o:o + FNO_W]; o += FNO_W
        Rc = torch.complex(R[..., 0], R[..., 1]).reshape(FNO_M, FNO_M, FNO_M, FNO_W, FNO_W)  # [jz][jy][jx][o][i]
        vc = v.to(torch.complex128)
        vh = torch.einsum("czyx,ax,by,dz->cdba", vc, tx, ty, tz) / (nx * ny * nz)  # [c][jz][jy][jx], normalised
        wh = torch.einsum("dbaoi,idba->odba", Rc, vh)
        spec = torch.einsum("odba,ax,by,dz->ozyx", wh, tx.conj(), ty.conj(), tz.conj()).real
        pre = torch.einsum("oi,izyx->ozyx", Wl, v) + bl[:, None, None, None] + spec
        if l < FNO_L - 1:
            s = 0.7978845608028654
            v = 0.5 * pre * (1.0 + torch.tanh(s * (pre + 0.044715 * pre ** 3)))
        else:
            v = pre
    q = P[o:o + FNO_W]; o += FNO_W
    q0 = P[o]
    return (torch.einsum("c,czyx->zyx", q, v) + q0).reshape(-1)


def fno_loss_grad(params, samples):
    """samples: list of (dims, u [2][N], target [N]).  Mean over samples of the MSE; gradient by autograd."""
    import torch

    p = torch.tensor(np.asarray(params, dtype=np.float64), requires_grad=True)
    loss = 0.0
    for dims, u, t in samples:
        d = fno_forward_torch(p, u, dims)
        loss = loss + torch.mean((d - torch.as_tensor(t, dtype=torch.float64)) ** 2)
    loss = loss / len(samples)
    loss.backward()
    return float(loss.detach()), p.grad.numpy().copy()


def fno_init_params(seed=0, spec_scale=0.5, scale=0.3):
    rng = np.random.default_rng(seed)
    parts = [rng.normal(0.0, scale, FNO_W * FNO_IN), np.zeros(FNO_W)]
    for _ in range(FNO_L):
        parts.append(rng.normal(0.0, spec_scale / FNO_W, 2 * FNO_K * FNO_W * FNO_W))
        parts.append(rng.normal(0.0, scale / np.sqrt(FNO_W), FNO_W * FNO_W))
        parts.append(np.zeros(FNO_W))
    parts.append(rng.normal(0.0, scale / np.sqrt(FNO_W), FNO_W))
    parts.append([0.0])
    return np.concatenate(parts)
