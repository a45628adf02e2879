"""CPU tests: oracle physics, host FP64 pieces of the product vs the oracle."""
import numpy as np
import pytest

from conftest import rel_l2
from oracle import oracle as O


@pytest.fixture(scope="module")
def ora1(sys1):
    return O.OracleSys(sys1)


def _hc(fr, fi):
    hr, hi = -0.25 * fr, -0.25 * fi
    hr[..., -1] = -0.5 * fr[..., -1]
    hi[..., -1] = 0.0
    return hr, hi


def test_gvec_matches_oracle(wl, sys1, sys2):
    for s in (sys1, sys2):
        ka, kb, kc, b1, b2 = O.gvec(s["hmat"], wl.ECUT_HA, [20, 20, 20])
        for x, y in ((ka, s["ka"]), (kb, s["kb"]), (kc, s["kc"]), (b1, s["ib1"]), (b2, s["ib2"])):
            assert np.array_equal(x, y)
    assert sys1["ncoef"] == 824 and sys2["ncoef"] == 6567


def test_fft_maps_match_setfft_indx(pkg, sys1):
    m, mc = pkg.fft_maps(24, 24, 24, sys1["ka"], sys1["kb"], sys1["kc"])
    n = 24
    w = lambda k: k % n
    exp = (w(sys1["ka"][:-1]) * n + w(sys1["kb"][:-1])) * n + w(sys1["kc"][:-1])
    expc = (w(-sys1["ka"][:-1]) * n + w(-sys1["kb"][:-1])) * n + w(-sys1["kc"][:-1])
    assert np.array_equal(m[:-1], exp) and np.array_equal(mc[:-1], expc)
    assert m[-1] == 0 and mc[-1] == 0


def test_oracle_hamiltonian_hermitian(wl, sys1, ora1):
    nc = sys1["ncoef"]
    rng = np.random.default_rng(1)
    a, b = rng.standard_normal((2, nc)), rng.standard_normal((2, nc))
    a[1, -1] = b[1, -1] = 0
    fr, fi = ora1.hpsi(np.concatenate([a[0], b[0]]), np.concatenate([a[1], b[1]]))
    hr, hi = _hc(fr.reshape(2, nc), fi.reshape(2, nc))
    d1 = wl.half_dot(nc, a[0], a[1], hr[1], hi[1])
    d2 = wl.half_dot(nc, hr[0], hi[0], b[0], b[1])
    assert abs(d1 - d2) < 1e-12 * abs(d1)


def test_oracle_plane_wave_and_constant_shift(wl, sys1):
    s = dict(sys1)
    s["kb_desc"] = None
    s["vks"] = np.full_like(sys1["vks"], 0.7)
    o = O.OracleSys(s)
    nc = s["ncoef"]
    c = np.zeros(nc)
    c[5] = 1.0
    fr, fi = o.hpsi(c, np.zeros(nc))
    hr, _ = _hc(fr, fi)
    G = 2 * np.pi * np.array([s["ka"][5], s["kb"][5], s["kc"][5]]) / np.diag(s["hmat"])
    assert abs(hr[5] - (0.5 * G @ G + 0.7)) < 1e-12


def test_round_fft_and_cheby_coeff(pkg):
    for n in (64 * 32, 256 * 32, 512 * 32, 1000, 777):
        assert pkg.roundFFT(n) == O.round_fft(n)
    for L, fun in ((64, 1), (256, 2), (512, 2)):
        a = pkg.calcChebyCoeff(L, 40.0, 19.0, 1000.0, 0.2, fun_flag=fun)
        b = O.cheby_coeff(L, 40.0, 19.0, 1000.0, 0.2, fun)
        assert np.allclose(a, b, rtol=0, atol=1e-13)


def test_cheby_coeff_reproduces_function(pkg):
    # sum_k c_k T_k(x) ~ F at a point inside the band
    L, ed, em, beta, mu = 512, 4.0, 1.0, 20.0, 1.2
    c = pkg.calcChebyCoeff(L, ed, em, beta, mu, fun_flag=1)
    for x in (0.1, 1.0, 2.5):
        t = np.clip((x - em) / (ed / 2), -1, 1)
        val = np.polynomial.chebyshev.chebval(t, c)
        assert abs(val - 1 / (1 + np.exp(beta * (x - mu)))) < 1e-10


def test_newton_points_and_coeff(pkg):
    for L in (16, 64):
        s1, u1 = pkg.genSampNewtonHermit(L, -2.0, 2.0, 4.0 / 40.0, -0.5)
        s2, u2 = O.newton_samp(L, -2.0, 2.0, 4.0 / 40.0, -0.5)
        assert np.array_equal(s1, s2) and np.array_equal(u1, u2)
        e1 = pkg.genCoeffNewtonHermit(L, 0.2, 1000.0, s1, u1)
        e2 = O.newton_coeff(L, 0.2, 1000.0, s2, u2)
        assert np.array_equal(e1, e2)


def test_gaussran2_matches_oracle(pkg):
    for seed in (10.0, 3.7e10, 123456.75):
        a, qa = pkg.gaussran2(1001, seed)
        b, qb = O.gaussran2(1001, seed)
        assert np.array_equal(a, b) and qa == qb


def test_chempot_bisection_monotone(pkg):
    # moments of a diagonal model spectrum: m_k = sum_i T_k(x_i)
    ev = np.linspace(-0.9, 0.9, 41)
    L = 128
    k = np.arange(L + 1)
    m = np.cos(np.outer(k, np.arccos(ev))).sum(axis=1) / 1.0
    ed, em = 2.0, 0.0
    mu, ne = pkg.calcChemPotCheby(L, ed, em, 50.0, 2.0, m, 40.0, 0.0, 0.2)
    assert abs(ne - 40.0) <= 1e-11 * 40
    n_lo = pkg.calcNumElecCheby(L, ed, em, 50.0, mu - 0.05, 2.0, m)
    n_hi = pkg.calcNumElecCheby(L, ed, em, 50.0, mu + 0.05, 2.0, m)
    assert n_lo < 40.0 < n_hi


def test_oracle_nl_force_is_minus_energy_gradient(sys1):
    """F_a = -dE_NL/dR_a by central differences (h = 1e-5 bohr) on a few
    coordinates: the force sums are the derivative of the energy sums."""
    ns, nc = 3, sys1["ncoef"]
    rng = np.random.default_rng(5)
    cr, ci = rng.standard_normal(ns * nc), rng.standard_normal(ns * nc)
    ci.reshape(ns, nc)[:, -1] = 0.0
    f, _ = O.OracleSys(sys1).nl_force(cr, ci)
    p0 = np.asarray(sys1["kb_desc"]["pos"], float).reshape(-1)

    def energy(pos):
        s2 = dict(sys1)
        s2["kb_desc"] = dict(sys1["kb_desc"], pos=pos)
        return O.OracleSys(s2).nl_force(cr, ci)[1]

    h = 1e-5
    for a, d in ((0, 1), (3, 0), (5, 2)):
        pp, pm = p0.copy(), p0.copy()
        pp[3 * a + d] += h
        pm[3 * a + d] -= h
        fd = -(energy(pp) - energy(pm)) / (2 * h)
        assert abs(fd - f[a, d]) < 1e-6 * np.abs(f).max()
