"""Test infrastructure: the CPU restatement of the SCF potential build and Pulay mixing that the
device module (dft-zig_b200/csrc/potential.cu) is checked against.  Only tests, the smoke check and
the benchmark's CPU-baseline leg use it.

Fields live on the FFT box with x fastest; G-space fields are f(G) = (1/N) sum_r f(r) e^{-iGr}
(numpy fftn of the (z, y, x) array divided by N)."""
from __future__ import annotations

import math

import numpy as np


def lda_pz(n):
    """xc/xc.zig:195-211 (lda_pz), 344-384 (PZ correlation energy and potential): f per volume and
    v = df/dn in Ry; both zero for n <= 1e-12."""
    n = np.asarray(n, dtype=np.float64)
    f = np.zeros_like(n)
    v = np.zeros_like(n)
    m = n > 1e-12
    nn = n[m]
    n13 = np.power(nn, 1.0 / 3.0)
    c_x = -0.75 * math.pow(3.0 / math.pi, 1.0 / 3.0)
    rs = np.power(3.0 / (4.0 * math.pi * nn), 1.0 / 3.0)
    eps_c = np.empty_like(nn)
    v_c = np.empty_like(nn)
    lo = rs < 1.0
    a, b, c, d = 0.0311, -0.048, 0.0020, -0.0116
    r = rs[lo]
    lr = np.log(r)
    e = a * lr + b + c * r * lr + d * r
    eps_c[lo] = e
    v_c[lo] = e - (r / 3.0) * (a / r + c * lr + c + d)
    g, b1, b2 = -0.1423, 1.0529, 0.3334
    r = rs[~lo]
    sr = np.sqrt(r)
    den = 1.0 + b1 * sr + b2 * r
    e = g / den
    eps_c[~lo] = e
    v_c[~lo] = e - (r / 3.0) * (-g * (0.5 * b1 / sr + b2) / (den * den))
    f[m] = 2.0 * (nn * c_x * n13 + nn * eps_c)
    v[m] = 2.0 * (4.0 / 3.0 * c_x * n13 + v_c)
    return f, v


def pw92_correlation(rs):
    """xc/xc.zig:320-342: Perdew-Wang 92 unpolarised correlation (Hartree): eps, d eps / d rs and
    v_c = eps - rs/3 d eps / d rs."""
    rs = np.asarray(rs, dtype=np.float64)
    a, a1, b1, b2, b3, b4 = 0.031091, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294
    sq = np.sqrt(rs)
    f = b1 * sq + b2 * rs + b3 * rs * sq + b4 * rs * rs
    g = 1.0 + 1.0 / (2.0 * a * f)
    lg = np.log(g)
    eps = -2.0 * a * (1.0 + a1 * rs) * lg
    dfr = 0.5 * b1 / sq + b2 + 1.5 * b3 * sq + 2.0 * b4 * rs
    dlg = -(1.0 / (2.0 * a * f * f * g)) * dfr
    deps = -2.0 * a * (a1 * lg + (1.0 + a1 * rs) * dlg)
    return eps, deps, eps - (rs / 3.0) * deps


def pbe(n, g2):
    """xc/xc.zig:213-318 (pbe, pbe_exchange, pbe_correlation): f per volume, df/dn and df/d|grad n|^2,
    in Ry; all zero for n <= 1e-12."""
    n = np.asarray(n, dtype=np.float64)
    g2 = np.asarray(g2, dtype=np.float64)
    f = np.zeros_like(n)
    vn = np.zeros_like(n)
    vg = np.zeros_like(n)
    m = n > 1e-12
    nn, gg = n[m], g2[m]
    pi = math.pi
    # exchange
    mu, kappa = 0.2195149727645171, 0.804
    c_x = -0.75 * math.pow(3.0 / pi, 1.0 / 3.0)
    n13 = np.power(nn, 1.0 / 3.0)
    ex0 = nn * c_x * n13
    kf = np.power(3.0 * pi * pi * nn, 1.0 / 3.0)
    den_x = 4.0 * kf * kf * nn * nn
    s2 = np.where((gg > 0.0) & (den_x > 0.0), gg / np.where(den_x > 0.0, den_x, 1.0), 0.0)
    t = 1.0 + mu * s2 / kappa
    fx = 1.0 + kappa - kappa / t
    dfs = mu / (t * t)
    ex_dn = 4.0 / 3.0 * c_x * n13 * fx + ex0 * dfs * (-8.0 / 3.0 * s2 / nn)
    ex_dg = ex0 * dfs * np.where(den_x > 0.0, 1.0 / np.where(den_x > 0.0, den_x, 1.0), 0.0)
    # correlation
    beta, gamma = 0.06672455060314922, 0.031090690869654895
    rs = np.power(3.0 / (4.0 * pi * nn), 1.0 / 3.0)
    eps_c, deps_drs, v_c = pw92_correlation(rs)
    deps_dn = deps_drs * (-rs / (3.0 * nn))
    ks2 = 4.0 * kf / pi
    den_c = 4.0 * ks2 * nn * nn
    t2 = np.where((gg > 0.0) & (den_c > 0.0), gg / np.where(den_c > 0.0, den_c, 1.0), 0.0)
    bg = beta / gamma
    x = bg * t2
    u = np.exp(-eps_c / gamma)
    um = u - 1.0
    big = np.abs(um) > 1e-12
    A = np.where(big, bg / np.where(big, um, 1.0), 0.0)
    y = A * t2
    d2 = 1.0 + y + y * y
    q = (1.0 + y) / d2
    arg = 1.0 + x * q
    pos = arg > 0.0
    H = gamma * np.where(pos, np.log(np.where(pos, arg, 1.0)), 0.0)
    d2s = d2 * d2
    dq_dt2 = -A * y * (2.0 + y) / d2s
    darg = bg * q + x * dq_dt2
    safe_arg = np.where(pos, arg, 1.0)
    dH_dt2 = np.where(pos, gamma * darg / safe_arg, 0.0)
    dH_dA = np.where(pos, -gamma * x * t2 * y * (2.0 + y) / (safe_arg * d2s), 0.0)
    dA_dn = np.where(big, bg * u / (gamma * np.where(big, um, 1.0) ** 2) * deps_dn, 0.0)
    dH_dn = dH_dt2 * (-7.0 / 3.0 * t2 / nn) + dH_dA * dA_dn
    dH_dg = dH_dt2 * np.where(den_c > 0.0, 1.0 / np.where(den_c > 0.0, den_c, 1.0), 0.0)
    f[m] = 2.0 * (ex0 * fx + nn * (eps_c + H))
    vn[m] = 2.0 * (ex_dn + v_c + H + nn * dH_dn)
    vg[m] = 2.0 * (ex_dg + nn * dH_dg)
    return f, vn, vg


def g_vectors_cart(dims, recip):
    """Cartesian G of every box point in FFT order (N x 3)."""
    f = [np.fft.fftfreq(n, 1.0 / n) for n in dims]
    hz, hy, hx = np.meshgrid(f[2], f[1], f[0], indexing="ij")
    return np.stack([hx.ravel(), hy.ravel(), hz.ravel()], axis=1) @ np.asarray(recip, dtype=np.float64)


def gga_xc_fields(rho, dims, recip, xc=pbe):
    """compute_gga_xc_fields (scf/xc_fields.zig:108-142): grad n by FFT (gradient_from_real,
    xc_fields.zig:306-339), the point functional, V_xc = df/dn - 2 div(df/dg2 grad n) with the
    divergence by FFT (divergence_from_real, xc_fields.zig:341-375).  Returns (f, V_xc) on the grid."""
    rho = np.asarray(rho, dtype=np.float64)
    G = g_vectors_cart(dims, recip)
    rg = to_g(rho, dims)
    grad = [np.fft.ifftn((1j * G[:, d] * rg).reshape(dims[2], dims[1], dims[0])).ravel().real * rho.size for d in range(3)]
    g2 = grad[0] ** 2 + grad[1] ** 2 + grad[2] ** 2
    f, vn, vg = xc(rho, g2)
    div_g = sum(1j * G[:, d] * to_g(vg * grad[d], dims) for d in range(3))
    div = to_r(div_g, dims)
    return f, vn - 2.0 * div


def g2_table(dims, recip):
    """|G|^2 of every box point, G = h b1 + k b2 + l b3 with h, k, l in FFT order (gvec_iter)."""
    f = [np.fft.fftfreq(n, 1.0 / n) for n in dims]
    hz, hy, hx = np.meshgrid(f[2], f[1], f[0], indexing="ij")
    G = np.stack([hx.ravel(), hy.ravel(), hz.ravel()], axis=1) @ np.asarray(recip, dtype=np.float64)
    return (G * G).sum(axis=1)


def to_g(fr, dims):
    n = dims[0] * dims[1] * dims[2]
    return np.fft.fftn(np.asarray(fr).reshape(dims[2], dims[1], dims[0])).ravel() / n


def to_r(fg, dims):
    n = dims[0] * dims[1] * dims[2]
    return np.fft.ifftn(np.asarray(fg).reshape(dims[2], dims[1], dims[0])).ravel().real * n


def hxc_potential(rho, dims, recip, volume, v_in_g=None, functional="lda"):
    """build_potential_grid (scf/potential.zig:144-203) without core charge, cutoff Coulomb or an
    ecutrho filter: V(G) = 8 pi rho(G)/G^2 [G^2 > 1e-12] + V_xc(G) (hartree_potential_at_g,
    potential.zig:34-44), V_xc of LDA-PZ or PBE (compute_xc_fields, xc_fields.zig:377-389).  Energy terms as scf/energy.zig:372-396: E_H = (vol/2) sum 8 pi |rho(G)|^2/G^2,
    E_xc = (vol/N) sum f_xc, and int v_in rho = (vol/N) sum_r v_in(r) rho(r).
    Returns (v_out_g, e_hartree, e_xc, int_vin_rho)."""
    rho = np.asarray(rho, dtype=np.float64)
    n = rho.size
    g2 = g2_table(dims, recip)
    rg = to_g(rho, dims)
    f, vxc = lda_pz(rho) if functional == "lda" else gga_xc_fields(rho, dims, recip)
    m = g2 > 1e-12
    vh = np.zeros_like(rg)
    vh[m] = 8.0 * math.pi * rg[m] / g2[m]
    v_out = vh + to_g(vxc, dims)
    e_h = 0.5 * volume * float(np.sum(8.0 * math.pi * np.abs(rg[m]) ** 2 / g2[m]))
    e_xc = float(f.sum()) * volume / n
    ivr = 0.0
    if v_in_g is not None:
        ivr = float(np.dot(to_r(v_in_g, dims), rho)) * volume / n
    return v_out, e_h, e_xc, ivr


def potential_real(v_g, vloc_r, dims):
    """build_local_potential_real (scf/potential.zig:320-334): V(r) = V_loc(r) + FFT^-1 V(G)."""
    out = to_r(v_g, dims)
    return out if vloc_r is None else out + np.asarray(vloc_r, dtype=np.float64)


def solve_pulay_system(B, rhs, scaled: bool = False, singular=None):
    """scf/mixing.zig:341-405: Gaussian elimination with partial pivoting; a pivot below 1e-12
    returns equal weights (and 0 for the multiplier).  scaled: the overlap block is first divided by
    its largest diagonal entry (the device module's form), which leaves the weights unchanged and
    makes the pivot test relative to the residual size."""
    A = np.array(B, dtype=np.float64)
    if scaled:
        m = A.shape[0] - 1
        d = float(np.max(np.diag(A)[:m]))
        if d > 0.0:
            A[:m, :m] /= d
    b = np.array(rhs, dtype=np.float64)
    size = b.size
    for col in range(size):
        max_row = col + int(np.argmax(np.abs(A[col:, col])))
        if np.abs(A[max_row, col]) <= np.abs(A[col, col]):
            max_row = col
        if max_row != col:
            A[[col, max_row]] = A[[max_row, col]]
            b[[col, max_row]] = b[[max_row, col]]
        pivot = A[col, col]
        if abs(pivot) < 1e-12:
            if singular is not None:
                return singular
            r = np.full(size, 1.0 / (size - 1))
            r[-1] = 0.0
            return r
        for row in range(col + 1, size):
            factor = A[row, col] / pivot
            A[row, col:] -= factor * A[col, col:]
            b[row] -= factor * b[col]
    r = np.zeros(size)
    for i in range(size - 1, -1, -1):
        r[i] = (b[i] - np.dot(A[i, i + 1:], r[i + 1:])) / A[i, i]
    return r


class Pulay:
    """PulayMixer.mix_with_residual (scf/mixing.zig:182-248): append (x, r), drop the oldest beyond
    `history`; fewer than two pairs -> x + beta r; else sum c_i (x_i + beta r_i) with the bordered
    system B_ij = <r_i|r_j>, sum c_i = 1.

    device_form: the library's variant -- the overlap block scaled by its largest diagonal entry
    and, where the reference would average the history on a pivot below 1e-12, the oldest pair
    dropped and the system solved again (down to plain linear mixing)."""

    def __init__(self, history: int, scaled: bool = False, device_form: bool = False):
        self.history = history
        self.scaled = scaled or device_form
        self.device_form = device_form
        self.xs, self.rs = [], []

    def mix(self, x, r, beta):
        self.xs.append(np.array(x, dtype=np.float64))
        self.rs.append(np.array(r, dtype=np.float64))
        while len(self.xs) > self.history:
            self.xs.pop(0)
            self.rs.pop(0)
        m = len(self.xs)
        first = 0
        c = None
        while m - first >= 2:
            k = m - first
            B = np.zeros((k + 1, k + 1))
            for i in range(k):
                for j in range(k):
                    B[i, j] = float(np.dot(self.rs[first + i], self.rs[first + j]))
                B[i, k] = B[k, i] = -1.0
            rhs = np.zeros(k + 1)
            rhs[k] = -1.0
            c = solve_pulay_system(B, rhs, self.scaled, singular=False if self.device_form else None)
            if c is not False:
                break
            c = None
            first += 1
        if c is None:
            return self.xs[-1] + beta * self.rs[-1]
        out = np.zeros_like(self.xs[0])
        for i in range(m - first):
            out += c[i] * (self.xs[first + i] + beta * self.rs[first + i])
        return out


def ionic_potential(gth, atom_species, positions, dims, recip, volume, g2max=0.0):
    """build_ionic_potential_grid (scf/potential.zig:279-318) with the analytic Goedecker-Teter-Hutter
    local form factor (Hartree, x2 for Ry): V(G) = (2/vol) sum_a ff_s(|G|) e^{-iG.tau_a} for
    1e-12 < G^2 <= g2max (no cut for g2max <= 0).  gth[s] = (Z, r_loc, C1, C2, C3, C4).
    Returns (V(G), V_loc(r))."""
    gth = np.asarray(gth, dtype=np.float64).reshape(-1, 6)
    f = [np.fft.fftfreq(n, 1.0 / n) for n in dims]
    hz, hy, hx = np.meshgrid(f[2], f[1], f[0], indexing="ij")
    gv = np.stack([hx.ravel(), hy.ravel(), hz.ravel()], axis=1) @ np.asarray(recip, dtype=np.float64)
    g2 = (gv * gv).sum(axis=1)
    keep = g2 > 1e-12
    if g2max > 0.0:
        keep &= g2 <= g2max
    safe = np.where(keep, g2, 1.0)
    vg = np.zeros(g2.size, complex)
    pos = np.asarray(positions, dtype=np.float64).reshape(-1, 3)
    for s, (Z, r, c1, c2, c3, c4) in enumerate(gth):
        y = safe * r * r
        e = np.exp(-0.5 * y)
        poly = c1 + c2 * (3 - y) + c3 * (15 - 10 * y + y * y) + c4 * (105 - 105 * y + 21 * y * y - y ** 3)
        ff = -4 * math.pi * Z / safe * e + math.sqrt(8 * math.pi ** 3) * r ** 3 * e * poly
        sf = np.zeros(g2.size, complex)
        for a in np.where(np.asarray(atom_species) == s)[0]:
            sf += np.exp(-1j * (gv @ pos[a]))
        vg += np.where(keep, sf * 2.0 * ff / volume, 0.0)
    return vg, to_r(vg, dims)
