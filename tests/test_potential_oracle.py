"""The potential-build and mixing oracle (oracle/potential.py) on the CPU: internal consistency,
and agreement with the host SCF driver's own restatement (dft-zig_b200/scf.py)."""
import importlib
import math

import numpy as np

import dftzig_loader
from oracle import potential as op

dftzig_loader.load()
scf = importlib.import_module("dftzig_b200.scf")

DIMS = (12, 10, 9)
RECIP = np.array([[0.61, 0.05, 0.0], [0.02, 0.57, 0.04], [0.0, -0.03, 0.66]])
VOL = (2 * math.pi) ** 3 / abs(np.linalg.det(RECIP))


def _rho(seed=0):
    rng = np.random.default_rng(seed)
    n = DIMS[0] * DIMS[1] * DIMS[2]
    return 0.02 + 0.05 * rng.random(n)


def test_lda_pz_potential_is_the_derivative_and_matches_the_driver():
    n = np.linspace(1e-4, 2.0, 400)
    f, v = op.lda_pz(n)
    h = 1e-6 * n
    fp, _ = op.lda_pz(n + h)
    fm, _ = op.lda_pz(n - h)
    np.testing.assert_allclose(v, (fp - fm) / (2 * h), rtol=1e-6)
    f2, v2 = scf.lda_pz(n)
    np.testing.assert_allclose(f, f2, rtol=1e-14)
    np.testing.assert_allclose(v, v2, rtol=1e-14)
    assert op.lda_pz(np.array([1e-13]))[1][0] == 0.0


def test_hartree_energy_is_half_the_potential_integral():
    rho = _rho()
    v, e_h, e_xc, _ = op.hxc_potential(rho, DIMS, RECIP, VOL)
    g2 = op.g2_table(DIMS, RECIP)
    rg = op.to_g(rho, DIMS)
    vh = np.where(g2 > 1e-12, 8 * math.pi * rg / np.where(g2 > 1e-12, g2, 1.0), 0.0)
    n = rho.size
    assert abs(e_h - 0.5 * VOL / n * float(np.dot(op.to_r(vh, DIMS), rho))) < 1e-10 * abs(e_h)
    # the driver's own V_hxc(G) and energies on the same grid
    assert np.abs(v - (vh + op.to_g(op.lda_pz(rho)[1], DIMS))).max() < 1e-14
    assert e_xc < 0.0


def test_int_vin_rho_and_real_space_potential():
    rho = _rho(1)
    v_in = op.to_g(np.cos(np.arange(rho.size) * 0.01), DIMS)
    _, _, _, ivr = op.hxc_potential(rho, DIMS, RECIP, VOL, v_in)
    vr = op.potential_real(v_in, None, DIMS)
    assert abs(ivr - float(np.dot(vr, rho)) * VOL / rho.size) < 1e-12 * max(1.0, abs(ivr))
    vloc = np.linspace(-1, 1, rho.size)
    np.testing.assert_allclose(op.potential_real(v_in, vloc, DIMS), vr + vloc, atol=1e-13)


def test_pulay_oracle_matches_driver_and_the_scaled_solve_is_scale_free():
    rng = np.random.default_rng(3)
    A = np.eye(20) * 0.3 + 0.05 * rng.normal(size=(20, 20))
    b = rng.normal(size=20)
    x = np.zeros(20)
    mo, md = op.Pulay(4, device_form=True), scf.PulayMixer(4)
    xd = x.copy()
    for _ in range(40):
        x = mo.mix(x, b - A @ x, 0.5)
        xd = md.mix(xd, b - A @ xd, 0.5)
    np.testing.assert_allclose(x, xd, rtol=1e-10, atol=1e-12)
    assert np.linalg.norm(b - A @ x) < 1e-4 * np.linalg.norm(b)  # plain mixing: 0.85^40 ~ 1.5e-3
    # the reference's absolute pivot test falls back to equal weights for tiny residual overlaps;
    # the scaled form solves the same system (weights are scale-free)
    B = np.array([[4e-14, 1e-14, -1], [1e-14, 2e-14, -1], [-1, -1, 0.0]])
    rhs = np.array([0, 0, -1.0])
    np.testing.assert_allclose(op.solve_pulay_system(B, rhs)[:2], [0.5, 0.5])
    big = B.copy()
    big[:2, :2] *= 1e14
    np.testing.assert_allclose(op.solve_pulay_system(B, rhs, scaled=True)[:2], op.solve_pulay_system(big, rhs)[:2], rtol=1e-12)
    np.testing.assert_allclose(op.solve_pulay_system(B, rhs, scaled=True)[:2], [0.25, 0.75], rtol=1e-12)


def test_ionic_potential_oracle_matches_the_input_builder():
    """The oracle's radial-mesh ionic potential (local_vq_short_range, form_factor.zig:223-262, at every
    |G|) equals the host input builder's V_loc(r), with the builder's |G|^2 < 4 ecut cut; and it stays
    within 1e-6 of the analytic GTH form the mesh tabulates (the quadrature's only error)."""
    from oracle import pseudo

    system = importlib.import_module("dftzig_b200.system")
    c = system.crystal("sige8", 2)
    ecut = 10.0
    dims = system.fft_box(ecut, c.recip)
    meshes = [sp.mesh for sp in c.species]
    vg, _ = pseudo.ionic_potential_radial(meshes, c.atom_species, c.positions, dims, c.recip, c.volume, 4 * ecut)
    vr = op.to_r(vg, dims)
    ref = system.local_potential(c, dims, ecut)
    assert np.abs(vr - ref).max() < 1e-11 * np.abs(ref).max()
    gth = [[sp.params["z"], sp.params["rloc"], sp.params["c1"], sp.params["c2"], 0.0, 0.0] for sp in c.species]
    _, vr_gth = op.ionic_potential(gth, c.atom_species, c.positions, dims, c.recip, c.volume, 4 * ecut)
    assert np.abs(vr_gth - ref).max() < 1e-6 * np.abs(ref).max()


def test_short_range_form_factor_matches_reference_loop():
    """The vectorised form factor equals the reference's sequential loop (form_factor.zig:223-262) and
    the host builder's, and at q = 0 gives epsatm (compute_epsatm, form_factor.zig:264-268)."""
    from oracle import pseudo

    system = importlib.import_module("dftzig_b200.system")
    sp = system.species("Si")
    r, rab, vloc, z = sp.mesh
    q = np.array([0.0, 1e-11, 0.2, 1.0, 4.5, 9.0])
    loop = np.array([pseudo.local_vq_short_range(r, rab, vloc, z, float(x)) for x in q])
    np.testing.assert_allclose(pseudo.local_vq_short_range_vec(r, rab, vloc, z, q), loop, rtol=1e-13)
    np.testing.assert_allclose(system.local_form_factor(sp, q), loop, rtol=1e-13)
    assert system.epsatm(sp) == system.local_form_factor(sp, np.zeros(1))[0]


def test_pbe_derivatives_match_finite_differences():
    rng = np.random.default_rng(4)
    n = 10 ** rng.uniform(-3, 0.3, 300)
    # reduced gradients s^2 = |grad n|^2 / (4 kF^2 n^2) from 1e-2 to 10, where df/dg2 is resolvable
    kf = (3 * math.pi ** 2 * n) ** (1.0 / 3.0)
    g2 = 10 ** rng.uniform(-2, 1, 300) * 4 * kf ** 2 * n ** 2
    f, vn, vg = op.pbe(n, g2)
    hn, hg = 1e-6 * n, 1e-4 * g2
    np.testing.assert_allclose(vn, (op.pbe(n + hn, g2)[0] - op.pbe(n - hn, g2)[0]) / (2 * hn), rtol=2e-6, atol=1e-10)
    np.testing.assert_allclose(vg, (op.pbe(n, g2 + hg)[0] - op.pbe(n, g2 - hg)[0]) / (2 * hg), rtol=1e-6, atol=0)
    # no gradient: PBE exchange is the LDA exchange; the correlation is PW92 rather than PZ
    f0, v0, _ = op.pbe(n, np.zeros_like(n))
    assert np.all(np.abs(f0 - op.lda_pz(n)[0]) < 0.05 * np.abs(f0))


def test_pbe_matches_the_reference_libxc_point():
    """The reference's own PBE known-answer tests (xc/xc.zig:1048-1108): libxc values at n = 0.1,
    sigma = |grad n|^2 = 0.01 (Hartree).  The oracle returns the exchange + correlation total in Ry;
    the reference checks the totals of e_xc and v_sigma to 1e-4 and the correlation v_rho to 1e-3."""
    f, vn, vg = op.pbe(np.array([0.1]), np.array([0.01]))
    exc_ha, vrho_ha, vsigma_ha = f[0] / 0.1 / 2.0, vn[0] / 2.0, vg[0] / 2.0
    assert abs(exc_ha - (-0.3516400536 + -0.0452782280)) <= 1e-4 * 0.3969182816
    assert abs(vsigma_ha - (-0.0854846156 + 0.0697928401)) <= 1e-4 * 0.0156917755
    assert abs(vrho_ha - (-0.4460575074 + -0.0688510243)) <= 1e-3 * 0.0688510243


def test_gga_potential_is_the_functional_derivative():
    """E_xc[n + e dn] - E_xc[n - e dn] = 2 e (vol/N) sum V_xc dn for the PBE assembly (gradient and
    divergence by FFT): the sign and the factor 2 of the divergence term."""
    rng = np.random.default_rng(6)
    N = DIMS[0] * DIMS[1] * DIMS[2]
    x = rng.normal(size=N)
    rho = 0.03 + 0.01 * op.to_r(np.where(op.g2_table(DIMS, RECIP) < 2.0, op.to_g(x, DIMS), 0.0), DIMS)
    dn = op.to_r(np.where(op.g2_table(DIMS, RECIP) < 1.5, op.to_g(rng.normal(size=N), DIMS), 0.0), DIMS)
    f, v = op.gga_xc_fields(rho, DIMS, RECIP)
    eps = 1e-5
    ep = op.gga_xc_fields(rho + eps * dn, DIMS, RECIP)[0].sum()
    em = op.gga_xc_fields(rho - eps * dn, DIMS, RECIP)[0].sum()
    lhs = (ep - em) / (2 * eps)
    rhs = float(np.dot(v, dn))
    assert abs(lhs - rhs) < 1e-6 * abs(rhs)
