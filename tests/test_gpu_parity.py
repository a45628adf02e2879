"""GPU parity of the CUDA path (through the C ABI) against the CPU oracle.

Tolerances: FP64 plain form rel-L2 <= 1e-10 (filtered orbitals, density);
single H applications <= 1e-12.  Mixed precision: density rel-L2 vs the
FP64 result <= 1e-5 on these short filters."""
import numpy as np
import pytest

from conftest import rel_l2
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL_H = 1e-12
TOL = 1e-10


def _ctx(pkg, s, nmax, prec=0, kb=True):
    c = pkg.Context(*s["grid"], s["ka"], s["kb"], s["kc"], s["hmat"], precision=prec, max_states=nmax)
    c.set_vks(s["vks"])
    if kb:
        c.set_kb(s["kb_desc"])
    return c


@pytest.fixture(scope="module")
def o1(sys1):
    return O.OracleSys(sys1)


@pytest.fixture(scope="module")
def c1(pkg, sys1):
    c = _ctx(pkg, sys1, 16)
    yield c
    c.close()


def _rand(nc, ns, seed):
    rng = np.random.default_rng(seed)
    cr = rng.standard_normal(ns * nc)
    ci = rng.standard_normal(ns * nc)
    ci.reshape(ns, nc)[:, -1] = 0.0
    return cr, ci


@pytest.mark.parametrize("ns", [1, 2, 5, 16])
def test_hpsi_cfg1(c1, o1, sys1, ns):
    cr, ci = _rand(sys1["ncoef"], ns, ns)
    fr, fi, e = c1.calc_coef_force(cr, ci, want_enl=True)
    orr, oi, oe = o1.hpsi(cr, ci, want_enl=True)
    assert rel_l2(np.concatenate([fr, fi]), np.concatenate([orr, oi])) < TOL_H
    assert abs(e - oe) < 1e-12 * abs(oe)


def test_hpsi_local_only_and_kinetic_cap(pkg, sys1):
    s = dict(sys1)
    c = _ctx(pkg, s, 4, kb=False)
    s0 = dict(s)
    s0["kb_desc"] = None
    o = O.OracleSys(s0)
    cr, ci = _rand(s["ncoef"], 3, 7)
    a = c.calc_coef_force(cr, ci)
    b = o.hpsi(cr, ci)
    assert rel_l2(np.concatenate(a), np.concatenate(b)) < TOL_H
    c.close()


def test_hpsi_cfg2(pkg, sys2):
    c = _ctx(pkg, sys2, 3)
    o = O.OracleSys(sys2)
    cr, ci = _rand(sys2["ncoef"], 3, 3)
    a = c.calc_coef_force(cr, ci)
    b = o.hpsi(cr, ci)
    assert rel_l2(np.concatenate(a), np.concatenate(b)) < TOL_H
    c.close()


def test_noise_matches_oracle(c1, o1, sys1):
    for ns, myid, np_ in ((16, 0, 1), (5, 2, 4)):
        a = c1.genNoiseOrbitalReal(ns, seed=10.0, np_states=np_, myid=myid)
        b = o1.noise(ns, seed=10.0, np_states=np_, myid=myid)
        assert rel_l2(np.concatenate(a), np.concatenate(b)) < 1e-13


def _bounds(c, s):
    import __graft_entry__ as g
    wl = g.load_workload()
    return wl.lanczos_bounds(lambda r, i: c.calc_coef_force(r, i), s["ncoef"])


def test_filter_newton_config1_full(pkg, wl, c1, o1, sys1):
    """Config 1 as specified: 16 orbitals, Newton L=64, mu = 0.2 Ha, beta 1000."""
    emin, emax = _bounds(c1, sys1)
    ediff = emax - emin
    scale = 4.0 / ediff
    samp, unsc = pkg.genSampNewtonHermit(64, -2.0, 2.0, scale, emin)
    ec = pkg.genCoeffNewtonHermit(64, 0.2, wl.BETA, samp, unsc)
    cr, ci = c1.genNoiseOrbitalReal(16, seed=10.0)
    (sr,), (si,) = c1.filterNewtonPolyHerm(cr, ci, ec, samp, 1, scale, 0.5 * (emin + emax))
    osr, osi = o1.filter_newton(cr, ci, ec, samp, 1, scale, 0.5 * (emin + emax))
    assert rel_l2(np.concatenate([sr, si]), np.concatenate([osr[0], osi[0]])) < TOL
    rho = c1.rhoCalcRealStoHybrid(sr, si)
    orho = o1.density(osr[0], osi[0])
    assert rel_l2(rho, orho) < TOL


@pytest.mark.parametrize("ns,L,nmu", [(6, 32, 1), (5, 17, 2)])
def test_filter_cheby_with_moments(pkg, c1, o1, sys1, ns, L, nmu):
    emin, emax = -1.0, 45.0
    scale, em = 2.0 / (emax - emin), 0.5 * (emin + emax)
    ec = np.stack([pkg.calcChebyCoeff(L, emax - emin, em, 1000.0, mu) for mu in (0.2, 0.3)[:nmu]], axis=1).ravel()
    cr, ci = c1.genNoiseOrbitalReal(ns, seed=3.0)
    sre, sim, m = c1.filterChebyPolyHerm(cr, ci, ec, nmu, scale, em, store_moments=True)
    osr, osi, om = o1.filter_cheby(cr, ci, ec, nmu, scale, em, store_moments=True)
    for k in range(nmu):
        assert rel_l2(np.concatenate([sre[k], sim[k]]), np.concatenate([osr[k], osi[k]])) < TOL
    assert rel_l2(m[:L], om[:L]) < TOL


@pytest.mark.parametrize("L", [16, 33])
def test_cheby_moments(c1, o1, sys1, L):
    emin, emax = -1.0, 45.0
    scale, em = 2.0 / (emax - emin), 0.5 * (emin + emax)
    cr, ci = c1.genNoiseOrbitalReal(7, seed=10.0)
    m = c1.calcChebyMoments(cr, ci, L, scale, em)
    om = o1.moments(cr, ci, L, scale, em)
    assert rel_l2(m, om) < TOL


def test_normh_steps(c1, o1, sys1):
    nc = sys1["ncoef"]
    cr, ci = _rand(nc, 3, 11)
    wr, wi = _rand(nc, 3, 12)
    scale, em = 0.05, 20.0
    a = [x.copy() for x in (cr, ci, wr, wi)]
    fr, fi = c1.normHCheby(a[0], a[1], a[2], a[3], 3, scale, em)
    b = [x.copy() for x in (cr, ci, wr, wi)]
    ofr, ofi = np.zeros_like(cr), np.zeros_like(ci)
    O.lib().oracle_normh_cheby(o1._p, 3, 3, 1, scale, em, O._d(b[0]), O._d(b[1]), O._d(b[2]), O._d(b[3]),
                               O._d(ofr), O._d(ofi))
    assert rel_l2(np.concatenate([fr, fi]), np.concatenate([ofr, ofi])) < TOL_H
    for x, y in zip(a, b):
        assert rel_l2(x, y) < TOL_H
    c = [cr.copy(), ci.copy()]
    fr, fi = c1.normHNewtonHerm(c[0], c[1], scale, em, 0.3)
    d = [cr.copy(), ci.copy()]
    O.lib().oracle_normh_newton(o1._p, 3, scale, em, 0.3, O._d(d[0]), O._d(d[1]), O._d(ofr), O._d(ofi))
    assert rel_l2(np.concatenate(c), np.concatenate(d)) < TOL_H


def test_density_odd(c1, o1, sys1):
    cr, ci = c1.genNoiseOrbitalReal(5, seed=2.0)
    rho = c1.rhoCalcRealStoHybrid(cr, ci)
    assert rel_l2(rho, o1.density(cr, ci)) < 1e-12
    # electron-count identity: sum(rho)/N = sum_s <c_s|c_s> (Parseval over the half sphere)
    nc = sys1["ncoef"]
    tot = sum(2 * np.dot(cr[i * nc:(i + 1) * nc], cr[i * nc:(i + 1) * nc]) +
              2 * np.dot(ci[i * nc:(i + 1) * nc], ci[i * nc:(i + 1) * nc]) - cr[i * nc + nc - 1] ** 2
              for i in range(5))
    assert abs(rho.sum() / rho.size - tot) < 1e-10 * tot


def test_cfg2_filter_short(pkg, sys2):
    c = _ctx(pkg, sys2, 4)
    o = O.OracleSys(sys2)
    emin, emax = -1.0, 45.0
    scale, em = 2.0 / (emax - emin), 0.5 * (emin + emax)
    ec = pkg.calcChebyCoeff(12, emax - emin, em, 1000.0, 0.2)
    cr, ci = c.genNoiseOrbitalReal(4, seed=10.0)
    (sr,), (si,) = c.filterChebyPolyHerm(cr, ci, ec, 1, scale, em)
    osr, osi = o.filter_cheby(cr, ci, ec, 1, scale, em)
    assert rel_l2(np.concatenate([sr, si]), np.concatenate([osr[0], osi[0]])) < TOL
    c.close()


def test_mixed_precision_close_to_fp64(pkg, sys1):
    cd = _ctx(pkg, sys1, 8, prec=0)
    cm = _ctx(pkg, sys1, 8, prec=1)
    emin, emax = -1.0, 45.0
    scale, em = 2.0 / (emax - emin), 0.5 * (emin + emax)
    ec = pkg.calcChebyCoeff(64, emax - emin, em, 1000.0, 0.2)
    cr, ci = cd.genNoiseOrbitalReal(8, seed=10.0)
    (a,), (b,) = cd.filterChebyPolyHerm(cr, ci, ec, 1, scale, em)
    (x,), (y,) = cm.filterChebyPolyHerm(cr, ci, ec, 1, scale, em)
    assert rel_l2(np.concatenate([x, y]), np.concatenate([a, b])) < 1e-5
    ra = cd.rhoCalcRealStoHybrid(a, b)
    rx = cm.rhoCalcRealStoHybrid(x, y)
    assert rel_l2(rx, ra) < 1e-5
    cd.close()
    cm.close()


@pytest.mark.parametrize("generic", [False, True])
def test_fast_and_generic_fft_paths(pkg, sys1, o1, generic, monkeypatch):
    if generic:
        monkeypatch.setenv("SDFT_GENERIC_FFT", "1")
    c = _ctx(pkg, sys1, 6)
    cr, ci = _rand(sys1["ncoef"], 6, 21)
    a = c.calc_coef_force(cr, ci)
    b = o1.hpsi(cr, ci)
    assert rel_l2(np.concatenate(a), np.concatenate(b)) < TOL_H
    nc = c.genNoiseOrbitalReal(3, seed=4.0)
    assert rel_l2(np.concatenate(nc), np.concatenate(o1.noise(3, seed=4.0))) < 1e-13
    rho = c.rhoCalcRealStoHybrid(cr, ci)
    assert rel_l2(rho, o1.density(cr, ci)) < 1e-12
    c.close()


@pytest.mark.parametrize("grid,strain", [((24, 48, 24), (0.0, 0.0, 0.0)), ((48, 24, 72), (0.01, -0.02, 0.015)),
                                         ((36, 36, 36), (0.0, 0.0, 0.0))])
def test_noncubic_and_generic_grids(pkg, wl, grid, strain):
    s = wl.make_system(1, grid, strain=strain, disp_sigma=0.05, seed=3)
    c = _ctx(pkg, s, 5)
    o = O.OracleSys(s)
    cr, ci = _rand(s["ncoef"], 5, 5)
    a = c.calc_coef_force(cr, ci)
    b = o.hpsi(cr, ci)
    assert rel_l2(np.concatenate(a), np.concatenate(b)) < TOL_H
    rho = c.rhoCalcRealStoHybrid(cr, ci)
    assert rel_l2(rho, o.density(cr, ci)) < 1e-12
    nz = c.genNoiseOrbitalReal(3, seed=9.0)
    assert rel_l2(np.concatenate(nz), np.concatenate(o.noise(3, seed=9.0))) < 1e-13
    c.close()


@pytest.mark.parametrize("which,ns", [("sys1", 5), ("sys2", 130)])
def test_mixed_hpsi_tensor_core(pkg, which, ns, request):
    """Mixed context: FP32 FFT + INT8 Ozaki tcgen05 KB GEMMs vs the FP64 oracle."""
    s = request.getfixturevalue(which)
    c = _ctx(pkg, s, ns, prec=1)
    o = O.OracleSys(s)
    cr, ci = _rand(s["ncoef"], ns, 17)
    fr, fi, e = c.calc_coef_force(cr, ci, want_enl=True)
    orr, oi, oe = o.hpsi(cr, ci, want_enl=True)
    # FP32 FFTs bound the force error (~2e-8 measured); the digit GEMMs keep
    # the nonlocal energy within ~1e-8 (E_NL partly cancels between the
    # +0.5 s and -0.5 p channels)
    assert rel_l2(np.concatenate([fr, fi]), np.concatenate([orr, oi])) < 2e-7
    assert abs(e - oe) < 1e-6 * abs(oe)
    c.sync()
    c.close()


@pytest.mark.parametrize("which,ns", [("sys1", 5), ("sys2", 130)])
def test_mixed_fast_hpsi(pkg, which, ns, request):
    """SDFT_PREC_MIXED_FAST: the back projection on 24-bit digits (3 x 8 bits,
    6 products) -- the force error grows to a few 1e-7, the nonlocal energy
    (from the 28-bit projection) is unchanged."""
    s = request.getfixturevalue(which)
    c = _ctx(pkg, s, ns, prec=pkg.SDFT_PREC_MIXED_FAST)
    o = O.OracleSys(s)
    cr, ci = _rand(s["ncoef"], ns, 17)
    fr, fi, e = c.calc_coef_force(cr, ci, want_enl=True)
    orr, oi, oe = o.hpsi(cr, ci, want_enl=True)
    assert rel_l2(np.concatenate([fr, fi]), np.concatenate([orr, oi])) < 6e-7
    assert abs(e - oe) < 1e-6 * abs(oe)
    c.sync()
    c.close()


def test_mixed_newton_and_moments_close_to_fp64(pkg, sys1):
    """Mixed-precision Newton filter (in-place recurrence, paired accumulation,
    fused packing of the next step) and Chebyshev moments against FP64."""
    cd = _ctx(pkg, sys1, 6, prec=0)
    cm = _ctx(pkg, sys1, 6, prec=1)
    emin, emax = -1.0, 45.0
    scale = 4.0 / (emax - emin)
    samp, unsc = pkg.genSampNewtonHermit(48, -2.0, 2.0, scale, emin)
    ec = pkg.genCoeffNewtonHermit(48, 0.2, 1000.0, samp, unsc)
    cr, ci = cd.genNoiseOrbitalReal(6, seed=12.0)
    (a,), (b,) = cd.filterNewtonPolyHerm(cr, ci, ec, samp, 1, scale, 0.5 * (emin + emax))
    (x,), (y,) = cm.filterNewtonPolyHerm(cr, ci, ec, samp, 1, scale, 0.5 * (emin + emax))
    assert rel_l2(np.concatenate([x, y]), np.concatenate([a, b])) < 1e-5
    s2, em = 2.0 / (emax - emin), 0.5 * (emin + emax)
    md = cd.calcChebyMoments(cr, ci, 33, s2, em)
    mm = cm.calcChebyMoments(cr, ci, 33, s2, em)
    assert np.max(np.abs(mm - md)) < 1e-6 * np.max(np.abs(md))
    cd.close()
    cm.close()


def test_call_order_and_sizes_checked(pkg, sys1):
    """Host-side refusals on a live context: no potential yet, nstate outside
    1..max_states, a filter of fewer than two terms; the context stays usable."""
    c = pkg.Context(*sys1["grid"], sys1["ka"], sys1["kb"], sys1["kc"], sys1["hmat"], max_states=2)
    try:
        nc = sys1["ncoef"]
        z = np.zeros(nc)
        with pytest.raises(pkg.SdftError) as e:
            c.calc_coef_force(z, z)
        assert e.value.code == 4  # SDFT_ERR_STATE: V_KS not set
        c.set_vks(sys1["vks"])
        c.set_kb(sys1["kb_desc"])
        with pytest.raises(pkg.SdftError) as e:
            c.calc_coef_force(np.zeros(3 * nc), np.zeros(3 * nc))
        assert e.value.code == 1  # 3 orbitals > max_states 2
        with pytest.raises(pkg.SdftError) as e:
            c.upload(z, z)
            c.filter_cheby_dev(1, np.zeros(0), 1, 0.1, 0.0)
        assert e.value.code == 1
        rng = np.random.default_rng(1)
        cr, ci = rng.standard_normal(nc), rng.standard_normal(nc)
        ci[-1] = 0.0
        fr, fi = c.calc_coef_force(cr, ci)
        gr, gi = O.OracleSys(sys1).hpsi(cr, ci)
        assert rel_l2(np.concatenate([fr, fi]), np.concatenate([gr, gi])) < 1e-12
    finally:
        c.close()


@pytest.mark.parametrize("grid", [(24, 24, 24), (48, 48, 48), (96, 96, 96)])
def test_plane_threads_same_result(pkg, wl, grid):
    """The 128-thread plane-stage instance (the default for 48 x 48 to 72 x 72 planes,
    an autotuner choice) computes the same units as the 256-thread one:
    bitwise equal H.psi for 256, 128 and the default, and the knob is refused
    where it does not exist (FP64)."""
    nrep = grid[0] // 24
    s = wl.make_system(nrep, grid)
    c = _ctx(pkg, s, 6, prec=1)
    try:
        cr, ci = _rand(s["ncoef"], 6, 8)
        out = []
        for nt in (256, 128, 0):
            c.set_plane_threads(nt)
            out.append(np.concatenate(c.calc_coef_force(cr, ci)))
        assert np.array_equal(out[0], out[1]) and np.array_equal(out[0], out[2])
    finally:
        c.close()
    d = _ctx(pkg, s, 2, prec=0)
    try:
        with pytest.raises(pkg.SdftError) as e:
            d.set_plane_threads(128)
        assert e.value.code == 5
    finally:
        d.close()


@pytest.mark.parametrize("prec_name", ["SDFT_PREC_MIXED", "SDFT_PREC_MIXED_FAST"])
def test_gemm_tile_width_bitwise(pkg, sys2, prec_name):
    """The 64- and 128-column tiles of the KB GEMMs give bitwise-equal H.psi
    and E_NL: each output is the same exact integer sum per K range.  The
    orbital counts leave a 64-wide tile partly empty, fill it exactly, and
    cross 128 (where the per-call choice takes 64 for 130 and 128 for 200)."""
    prec = getattr(pkg, prec_name)
    c = _ctx(pkg, sys2, 200, prec=prec)
    try:
        for ns in (5, 64, 130, 200):
            cr, ci = _rand(sys2["ncoef"], ns, 31 + ns)
            out = {}
            for bn in (128, 64, 0):
                c.set_gemm_bn(bn)
                fr, fi, e = c.calc_coef_force(cr, ci, want_enl=True)
                out[bn] = (np.concatenate([fr, fi]), e)
            assert np.array_equal(out[64][0], out[128][0]), ns
            assert out[64][1] == out[128][1], ns
            assert np.array_equal(out[0][0], out[128][0]), ns
        with pytest.raises(pkg.SdftError) as e:
            c.set_gemm_bn(32)
        assert e.value.code == 1
    finally:
        c.close()


def test_tuner_sets_shapes(pkg, wl, sys2):
    """The autotuner times the GEMM tile width, the split-K and the plane CTA
    size on the context's own orbitals, sets them, caches the entry, and the
    tuned context filters the same orbitals as an untuned one (to the mixed
    filter's rounding)."""
    tuner_mod = __import__(pkg.__name__ + ".tuner", fromlist=["Tuner"])
    ns = 40
    cr, ci = _rand(sys2["ncoef"], ns, 5)
    res = []
    for tuned in (False, True):
        c = _ctx(pkg, sys2, ns, prec=1)
        try:
            emin, emax = c.lanczos_bounds(12, seed=15, margin=0.1)[:2]
            scale, em = 2.0 / (emax - emin), 0.5 * (emin + emax)
            if tuned:
                t = tuner_mod.Tuner(pkg, steps=2)
                c.upload(cr, ci)
                t.tune(c, ns, 4 * sys2["natm"], scale, em)
                entry = t.cache[t.key(c, ns, 4 * sys2["natm"])]
                assert entry["gemm_bn"] in (0, 64, 128) and set(entry["gemm_bn_ms"]) == {"0", "64", "128"}
                assert entry["plane_threads"] in (0, 128, 256) and set(entry["plane_ms"]) == {"0", "128", "256"}
                assert entry["split"] in (0, 1, 2, 4, 8, 16, 32)
            coef = pkg.calcChebyCoeff(16, emax - emin, em, 10.0, em, fun_flag=2)
            (sr,), (si,) = c.filterChebyPolyHerm(cr, ci, coef, 1, scale, em)
            res.append(np.concatenate([sr, si]))
        finally:
            c.close()
    assert rel_l2(res[1], res[0]) < 1e-6


def test_forced_split_sums_written_partials(pkg, sys2):
    """A forced split-K that does not divide the K tiles evenly (32 asked for
    206 K tiles: 7 each, 30 partials written) reduces only the partials the
    launch wrote.  The 128-wide tile at that split runs first and leaves its
    partials in the buffer at another stride; the 64-wide tile's filter must
    still equal the cost model's."""
    ns = 40
    cr, ci = _rand(sys2["ncoef"], ns, 5)
    c = _ctx(pkg, sys2, ns, prec=1)
    try:
        emin, emax = c.lanczos_bounds(12, seed=15, margin=0.1)[:2]
        scale, em = 2.0 / (emax - emin), 0.5 * (emin + emax)
        coef = pkg.calcChebyCoeff(16, emax - emin, em, 10.0, em, fun_flag=2)
        (r0,), (i0,) = c.filterChebyPolyHerm(cr, ci, coef, 1, scale, em)
        ref = np.concatenate([r0, i0])
        for bn in (128, 64):
            c.set_gemm_bn(bn)
            c.set_gemm_split(32)
            (r,), (i,) = c.filterChebyPolyHerm(cr, ci, coef, 1, scale, em)
            assert rel_l2(np.concatenate([r, i]), ref) < 1e-12, bn
    finally:
        c.close()
