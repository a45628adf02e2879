"""Pin the CPU oracle (sdft_oracle.c) to the reference's own C code.

oracle/_ref/libpinyref.so is built by oracle/build_ref.sh from the
reference sources (filter.c, normh.c, energy-wrapper-scf.c,
cp-energy-eext-stodft.c, cp-energy-ee-rho-stodft.c, cp_energy_eext_nonloc.c,
fft_package.c, coeff.c, calc-chempot-chebyshev.c, mathlib.c, set_cp_ewald.c,
...) and driven through PINY's own data structures by oracle/ref_harness.c.
The committed golden fixtures (tests/golden/) carry the same pins where the
reference tree is absent."""
import numpy as np
import pytest

from conftest import rel_l2
from oracle import oracle as O
from oracle import ref as R

pytestmark = pytest.mark.skipif(not R.available(), reason="reference-compiled oracle (oracle/_ref) not built")


@pytest.fixture(scope="module")
def both(sys1):
    return R.RefSys(sys1, 8), O.OracleSys(sys1)


def _rand(nc, ns, seed):
    rng = np.random.default_rng(seed)
    cr = rng.standard_normal(ns * nc)
    ci = rng.standard_normal(ns * nc)
    ci.reshape(ns, nc)[:, -1] = 0.0
    return cr, ci


def test_gvec_pinned(wl, sys1, sys2):
    for s in (sys1, sys2):
        ka, kb, kc, b1, b2 = R.gvec(s["hmat"], wl.ECUT_HA, [20, 20, 20], s["ncoef"])
        for x, y in ((ka, s["ka"]), (kb, s["kb"]), (kc, s["kc"]), (b1, s["ib1"]), (b2, s["ib2"])):
            assert np.array_equal(x, y)


@pytest.mark.parametrize("ns", [1, 4, 5])
def test_hpsi_pinned(both, sys1, ns):
    r, o = both
    cr, ci = _rand(sys1["ncoef"], ns, ns)
    fr, fi, e = r.hpsi(cr, ci)
    gr, gi, ge = o.hpsi(cr, ci, want_enl=True)
    assert rel_l2(np.concatenate([gr, gi]), np.concatenate([fr, fi])) < 1e-14
    assert abs(ge - e) < 1e-13 * abs(e)


@pytest.mark.parametrize("ns", [1, 5])
def test_nl_force_pinned(both, sys1, ns):
    """KB atomic forces: calcNlPseudoPostScf (control_ewd_non_loc / get_nlmat,
    getnl_pot_pv_fatm) against the oracle's restatement."""
    r, o = both
    cr, ci = _rand(sys1["ncoef"], ns, 40 + ns)
    fr, er = r.nl_force(cr, ci)
    fo, eo = o.nl_force(cr, ci)
    assert np.abs(fo - fr).max() < 1e-13 * np.abs(fr).max()
    assert abs(eo - er) < 1e-13 * abs(er)


def test_filter_cheby_pinned(pkg, both, sys1):
    r, o = both
    cr, ci = _rand(sys1["ncoef"], 5, 3)
    emin, emax = -1.0, 45.0
    scale, em = 2.0 / (emax - emin), 0.5 * (emin + emax)
    ec = np.stack([pkg.calcChebyCoeff(20, emax - emin, em, 1000.0, mu) for mu in (0.2, 0.35)], axis=1).ravel()
    a = r.filter(True, cr, ci, ec, 2, scale, em, moments=True)
    b = o.filter_cheby(cr, ci, ec, 2, scale, em, store_moments=True)
    for k in range(2):
        assert rel_l2(np.concatenate([b[0][k], b[1][k]]), np.concatenate([a[0][k], a[1][k]])) < 1e-13
    assert rel_l2(b[2][:20], a[2][:20]) < 1e-13


def test_filter_newton_pinned(pkg, both, sys1):
    r, o = both
    cr, ci = _rand(sys1["ncoef"], 4, 5)
    emin, emax = -1.0, 45.0
    scale = 4.0 / (emax - emin)
    samp, unsc = pkg.genSampNewtonHermit(24, -2.0, 2.0, scale, emin)
    ec = pkg.genCoeffNewtonHermit(24, 0.2, 1000.0, samp, unsc)
    a = r.filter(False, cr, ci, ec, 1, scale, 0.5 * (emin + emax), samp=samp)
    b = o.filter_newton(cr, ci, ec, samp, 1, scale, 0.5 * (emin + emax))
    assert rel_l2(np.concatenate([b[0][0], b[1][0]]), np.concatenate([a[0][0], a[1][0]])) < 1e-13


@pytest.mark.parametrize("L", [12, 17])
def test_moments_pinned(both, sys1, L):
    r, o = both
    cr, ci = _rand(sys1["ncoef"], 3, 9)
    emin, emax = -1.0, 45.0
    scale, em = 2.0 / (emax - emin), 0.5 * (emin + emax)
    a = r.moments(cr, ci, L, scale, em)
    b = o.moments(cr, ci, L, scale, em)
    M = L // 2 + 1 if L % 2 == 0 else (L + 1) // 2
    n = 2 * M - 1  # entries written by calcChebyMoments
    assert rel_l2(b[:n], a[:n]) < 1e-13


def test_coefficients_pinned(pkg):
    for n in (64 * 32, 256 * 32, 512 * 32, 1000):
        assert R.round_fft(n) == O.round_fft(n) == pkg.roundFFT(n)
    for L, fun in ((64, 1), (128, 2)):
        a = R.cheby_coeff(L, 40.0, 19.0, 1000.0, 0.2, fun)
        assert np.allclose(O.cheby_coeff(L, 40.0, 19.0, 1000.0, 0.2, fun), a, rtol=0, atol=1e-14)
        assert np.allclose(pkg.calcChebyCoeff(L, 40.0, 19.0, 1000.0, 0.2, fun_flag=fun), a, rtol=0, atol=1e-13)
    for L in (16, 64):
        s, u, e = R.newton(L, 4.0 / 40.0, -0.5, 1000.0, 0.2)
        s2, u2 = O.newton_samp(L, -2.0, 2.0, 4.0 / 40.0, -0.5)
        assert np.array_equal(s, s2) and np.array_equal(u, u2)
        assert np.array_equal(e, O.newton_coeff(L, 0.2, 1000.0, s2, u2))


def test_gaussran2_pinned(pkg):
    for seed in (10.0, 3.7e10, 123456.75):
        a, qa = R.gaussran2(2001, seed)
        b, qb = O.gaussran2(2001, seed)
        c, qc = pkg.gaussran2(2001, seed)
        assert np.array_equal(a, b) and np.array_equal(a, c) and qa == qb == qc


@pytest.mark.parametrize("grid,strain", [((24, 24, 24), (0.0, 0.0, 0.0)), ((24, 48, 24), (0.0, 0.0, 0.0)),
                                         ((36, 24, 48), (0.01, -0.02, 0.015))])
def test_noise_and_density_pinned(wl, grid, strain):
    """genNoiseOrbitalReal (gen-noise.c) and rhoCalcRealStoHybrid
    (density.c) of the reference against the oracle, cubic and non-cubic."""
    s = wl.make_system(1, grid, strain=strain)
    r, o = R.RefSys(s, 6), O.OracleSys(s)
    a = r.noise(5, 10.0)
    b = o.noise(5, 10.0)
    assert rel_l2(np.concatenate(b), np.concatenate(a)) < 1e-14
    rho_r = r.density(*b)
    rho_o = o.density(*b)
    assert rel_l2(rho_o, rho_r) < 1e-14


@pytest.mark.parametrize("init,gap", [(0.2, 0.05), (1.5, 0.1), (-0.8, 0.1), (0.25, 0.4)])
def test_chempot_pinned(pkg, wl, sys1, init, gap):
    """mu by the reference's own calcChemPotCheby (calc-chempot-chebyshev.c:30-314:
    its own moments of the noise, the bracket widened down from 0.2 and 1.5
    and up from -0.8, one secant step, bisection to 1e-11 Ne) against
    sdft_chempot_cheby on the same normalised moments; calcNumElecCheby
    (:918-971) against sdft_num_elec_cheby at mu and two other points."""
    r = R.RefSys(sys1, 8)
    cr, ci = r.noise(8, 10.0)
    emin, emax, L = -1.2, 42.0, 64
    ediff, em = emax - emin, 0.5 * (emin + emax)
    mu_r, ne_r = r.chem_pot(cr, ci, L, emin, emax, wl.BETA, wl.OCC, sys1["num_elec"], init, gap)
    m = r.moments(cr, ci, L, 2.0 / ediff, em) / 8
    mu, ne = pkg.calcChemPotCheby(L, ediff, em, wl.BETA, wl.OCC, m, sys1["num_elec"], init, gap)
    assert abs(mu - mu_r) <= 1e-14 * abs(mu_r)
    assert abs(ne - ne_r) <= 1e-13 * ne_r
    for x in (mu_r, 0.1, 0.3):
        a = R.num_elec(L, emin, emax, wl.BETA, wl.OCC, m, x)
        b = pkg.calcNumElecCheby(L, ediff, em, wl.BETA, x, wl.OCC, m)
        assert abs(a - b) <= 1e-13 * abs(a)


@pytest.fixture(scope="module")
def dens_sys(wl):
    """The 8-atom cell on the grid that holds its density sphere (32^3)."""
    return wl.make_system(1, wl.density_grid(wl.make_system(1, (24, 24, 24))["L"]))


def test_vks_pinned(pkg, wl, dens_sys):
    """The density side of the SCF step: the reference's controlEwdLocPreScf,
    calcRhoStoRecipFullg and cpGetVksStodft (run by oracle/_ref on its own
    density sphere from setkvec3d) against the numpy restatement
    (oracle/vks.py), and the sphere against the library's setkvec3d_sm at
    4 Ecut."""
    from oracle import vks as V
    s = dens_sys
    r = R.RefSys(s, 4)
    o = O.OracleSys(s)
    cr, ci = o.noise(4, 10.0)
    rho = o.density(cr, ci)
    rho_in = rho * (s["num_elec"] / rho.mean())
    vtab, gmin, dg, gz = wl.local_table()
    ref = r.vks(wl.ECUT_HA, vtab, gmin, dg, gz, 1, rho_in)
    ka, kb, kc = ref["ka"], ref["kb"], ref["kc"]
    lk = pkg.setkvec3d_sm(s["hmat"], 4 * wl.ECUT_HA, list(s["grid"]))
    for x, y in zip(lk[:3], (ka, kb, kc)):
        assert np.array_equal(x, y)
    vre, vim = V.vext(s["hmat"], ka, kb, kc, s["pos"], vtab, vtab.shape[1], gmin, dg, gz)
    assert rel_l2(vre, ref["vext_re"]) < 1e-13 and rel_l2(vim, ref["vext_im"]) < 1e-13
    vf, rre, rim, e = V.vks_from_rho(s["grid"], s["hmat"], ka, kb, kc, ref["vext_re"], ref["vext_im"], rho_in)
    assert rel_l2(rre, ref["rhog_re"]) < 1e-13 and rel_l2(rim, ref["rhog_im"]) < 1e-13
    assert rel_l2(vf, ref["vks"]) < 1e-13
    assert np.all(np.abs(e - ref["energies"]) <= 1e-13 * np.abs(ref["energies"]))
    # the local pseudopotential alone, back in real space, is the Gaussian potential of the workload
    v0, _, _, _ = V.vks_from_rho(s["grid"], s["hmat"], ka, kb, kc, vre, vim, np.zeros_like(rho_in), xc=False)
    assert rel_l2(v0, s["vks"]) < 1e-10


@pytest.mark.parametrize("q_pseud", [4.0, 3.5])
def test_local_forces_pinned(wl, q_pseud):
    """The local-pseudopotential + Ewald reciprocal forces of calcLocExtPostScf
    (control_ewd_loc) and the Ewald self / background energies
    (ewald3d_selfbgr_cp) of the reference against the numpy restatement, with
    the charge correction on (q_pseud 3.5) and off; and the restatement's
    force is -dE/dR of E_loc + vrecip at fixed rho(G) (central differences)."""
    from oracle import vks as V
    s = wl.make_system(1, (32, 32, 32), disp_sigma=0.05, seed=2)
    r = R.RefSys(s, 4)
    o = O.OracleSys(s)
    cr, ci = o.noise(4, 10.0)
    rho = o.density(cr, ci)
    rho_in = rho * (s["num_elec"] / rho.mean())
    vtab, gmin, dg, gz = wl.local_table()
    q = np.full(s["natm"], 4.0)
    ref = r.vks(wl.ECUT_HA, vtab, gmin, dg, gz, 1, rho_in, q=q, q_pseud=q_pseud, alp_ewd=1.2)
    ka, kb, kc = ref["ka"], ref["kb"], ref["kc"]
    args = (s["hmat"], ka, kb, kc)
    F, e = V.local_forces(*args, s["pos"], q, q_pseud, vtab, vtab.shape[1], gmin, dg, ref["rhog_re"],
                          ref["rhog_im"], 1.2)
    assert np.abs(F - ref["force"]).max() < 1e-12 * np.abs(ref["force"]).max()
    assert np.all(np.abs(e - ref["ewald"]) <= 1e-13 * np.abs(ref["ewald"]))
    # E(R) = 2 sum_G Re(vt-weighted vext . rho) + vrecip, rho(G) fixed
    import math
    h = np.asarray(s["hmat"], float)
    vol = abs(np.linalg.det(h))
    G = V.gvec_cart(s["hmat"], ka[:-1], kb[:-1], kc[:-1])
    g2 = (G ** 2).sum(axis=1)
    v = V.spline(vtab, vtab.shape[1], gmin, dg, np.sqrt(g2))
    kk = np.stack([ka[:-1], kb[:-1], kc[:-1]], axis=1).astype(float)
    rr, ri = ref["rhog_re"][:-1], ref["rhog_im"][:-1]

    def energy(pos):
        sfr = pos @ np.linalg.inv(h).T
        arg = 2.0 * math.pi * (kk @ sfr.T)
        vt = v[:, None] - 4.0 * math.pi * (q[None, :] - q_pseud) / g2[:, None]
        ve_r = (np.cos(arg) * vt).sum(axis=1) / vol
        ve_i = -(np.sin(arg) * vt).sum(axis=1) / vol
        sr_, si_ = np.cos(arg) @ q, np.sin(arg) @ q
        preg = np.exp(-g2 / (4.0 * 1.2 ** 2)) * 4.0 * math.pi / (g2 * vol)
        return 2.0 * np.sum(ve_r * rr + ve_i * ri) + np.sum(preg * (sr_ ** 2 + si_ ** 2))
    d = 1e-5
    for a, c in ((0, 0), (3, 1), (5, 2)):
        p1, p2 = s["pos"].copy(), s["pos"].copy()
        p1[a, c] += d
        p2[a, c] -= d
        num = -(energy(p1) - energy(p2)) / (2 * d)
        assert abs(num - F[a, c]) < 1e-6 * np.abs(F).max()


@pytest.mark.parametrize("alp,ishift", [(0.3, 0), (0.9, 0), (0.3, 1), (0.3, 2), (1.2, 2)])
def test_coul_pair_pinned(alp, ishift):
    """The real-space Ewald pair term of the restatement (vcoul_bin's fitted
    erfc with spline_vdv's shift or switch) against the reference's own
    table on its own r grid."""
    from oracle import vks as V
    r, v, dv = R.coul_table(3000, 0.5, 9.0, alp, 3.7, ishift, 1.5)
    ov, odv = V.coul_pair(r, 3.7, alp, 9.0, ishift, 1.5)
    assert np.abs(ov - v).max() <= 1e-14 * np.abs(v).max()
    assert np.abs(odv - dv).max() <= 1e-14 * np.abs(dv).max()


def test_ewald_real_forces_and_alpha(wl):
    """The restated real-space ion-ion Ewald sum: its force is -dE/dR (central
    differences), and the full Ewald energy -- this sum plus the reference's
    own reciprocal, self and background terms -- does not depend on the
    splitting parameter, to the accuracy of the erfc fit (2.3e-9)."""
    from oracle import vks as V
    s = wl.make_system(1, (32, 32, 32), disp_sigma=0.05, seed=2)
    q = np.full(s["natm"], 4.0)
    F, E = V.ewald_real(s["hmat"], s["pos"], q, 1.0, 9.0)
    d = 1e-5
    for a, c in ((0, 0), (3, 1), (5, 2)):
        p1, p2 = s["pos"].copy(), s["pos"].copy()
        p1[a, c] += d
        p2[a, c] -= d
        num = -(V.ewald_real(s["hmat"], p1, q, 1.0, 9.0)[1] - V.ewald_real(s["hmat"], p2, q, 1.0, 9.0)[1]) / (2 * d)
        assert abs(num - F[a, c]) < 1e-7 * np.abs(F).max()
    r = R.RefSys(s, 4)
    vtab, gmin, dg, gz = wl.local_table()
    rho_in = np.full(int(np.prod(s["grid"])), s["num_elec"] / np.prod(s["grid"]))
    # alp 0.4 and 0.5 with a 20 bohr cutoff: the real-space part moves from
    # 0.70 to 0.10 hartree of a -33.6 total, the reciprocal part from 3.9 to 8.4
    tot, real = [], []
    for alp in (0.4, 0.5):
        ref = r.vks(wl.ECUT_HA, vtab, gmin, dg, gz, 1, rho_in, q=q, q_pseud=4.0, alp_ewd=alp)
        real.append(V.ewald_real(s["hmat"], s["pos"], q, alp, 20.0)[1])
        tot.append(real[-1] + ref["ewald"].sum())
    assert real[0] - real[1] > 0.5
    assert abs(tot[0] - tot[1]) < 1e-9 * abs(tot[1])
