"""Device Lanczos bounds (the role of genEnergyMax/genEnergyMin,
stodft/calc-spectral-range.c:33,339, run as 20 Lanczos steps) and the
energies of the filtered orbitals (calcEnergyChemPot, stodft/calc-energy.c:
32-207) against the host Lanczos of the same H and against the oracle."""
import math

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _ctx(pkg, s, prec, n):
    c = pkg.Context(*s["grid"], s["ka"], s["kb"], s["kc"], s["hmat"], precision=prec, max_states=n)
    c.set_vks(s["vks"])
    c.set_kb(s["kb_desc"])
    return c


@pytest.mark.parametrize("which,prec,tol", [("sys1", "fp64", 1e-9), ("sys2", "fp64", 1e-9), ("sys2", "mixed", 1e-6)])
def test_lanczos_bounds_match_host_lanczos(pkg, wl, sys1, sys2, which, prec, tol):
    s = sys1 if which == "sys1" else sys2
    p = pkg.SDFT_PREC_FP64 if prec == "fp64" else pkg.SDFT_PREC_MIXED
    host = _ctx(pkg, s, p, 1)
    dev = _ctx(pkg, s, p, 1)
    try:
        lo_h, hi_h = wl.lanczos_bounds(lambda r, i: host.calc_coef_force(r, i), s["ncoef"])
        lo_d, hi_d, al, be = dev.lanczos_bounds(20, seed=15, margin=0.1)
    finally:
        host.close()
        dev.close()
    assert len(al) == 20 and np.all(be > 0)
    assert abs(lo_d - lo_h) <= tol and abs(hi_d - hi_h) <= tol
    # the tridiagonal extremes by Sturm bisection agree with a dense solver
    T = np.diag(al) + np.diag(be[:-1], 1) + np.diag(be[:-1], -1)
    ev = np.linalg.eigvalsh(T)
    assert abs(ev[0] - 0.1 - lo_d) < 1e-10 and abs(ev[-1] + 0.1 - hi_d) < 1e-10


def _ak2(s):
    L = np.diag(np.asarray(s["hmat"], float))
    g = [2.0 * math.pi * np.asarray(s[k], float) / L[i] for i, k in enumerate(("ka", "kb", "kc"))]
    return g[0] ** 2 + g[1] ** 2 + g[2] ** 2


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("mixed", 2e-7)])
def test_energy_chempot_matches_oracle(pkg, wl, sys1, prec, tol):
    s = sys1
    ns, L = 6, 32
    rng = np.random.default_rng(21)
    cr = rng.standard_normal(ns * s["ncoef"])
    ci = rng.standard_normal(ns * s["ncoef"])
    ci.reshape(ns, -1)[:, -1] = 0.0
    o = O.OracleSys(s)
    lo, hi = wl.lanczos_bounds(lambda r, i: o.hpsi(r, i), s["ncoef"])
    ediff, emean = hi - lo, 0.5 * (hi + lo)
    ec = pkg.calcChebyCoeff(L, ediff, emean, wl.BETA, 0.1, fun_flag=2)
    p = pkg.SDFT_PREC_FP64 if prec == "fp64" else pkg.SDFT_PREC_MIXED
    ctx = _ctx(pkg, s, p, ns)
    try:
        ctx.upload(cr, ci)
        ctx.filter_cheby_dev(ns, ec, 1, 2.0 / ediff, emean)
        ek, ep = ctx.energy_chempot_dev(ns, 0, occ=2.0, nsto_total=ns)
        fr, fi = ctx.download_filtered(ns)
    finally:
        ctx.close()
    # expectation from the FP64 oracle filter of the same orbitals
    orr, oii = (a[0] for a in o.filter_cheby(cr, ci, ec, 1, 2.0 / ediff, emean))
    ak2 = _ak2(s)[:-1]
    R, I = orr.reshape(ns, -1)[:, :-1], oii.reshape(ns, -1)[:, :-1]
    ek_ref = 2.0 * 0.5 * float(np.sum(2.0 * ak2 * (R * R + I * I))) / ns
    ep_ref = 2.0 * o.hpsi(orr, oii, want_enl=True)[2] / ns
    assert abs(ek - ek_ref) <= tol * abs(ek_ref)
    assert abs(ep - ep_ref) <= tol * abs(ep_ref)


def _filtered_ctx(pkg, wl, s, p, ns, seed, L=32):
    """Context holding ns Chebyshev-filtered random orbitals; returns it with
    the orbitals and the filter parameters."""
    rng = np.random.default_rng(seed)
    cr = rng.standard_normal(ns * s["ncoef"])
    ci = rng.standard_normal(ns * s["ncoef"])
    ci.reshape(ns, -1)[:, -1] = 0.0
    o = O.OracleSys(s)
    lo, hi = wl.lanczos_bounds(lambda r, i: o.hpsi(r, i), s["ncoef"])
    ediff, emean = hi - lo, 0.5 * (hi + lo)
    ec = pkg.calcChebyCoeff(L, ediff, emean, wl.BETA, 0.1, fun_flag=2)
    ctx = _ctx(pkg, s, p, ns)
    ctx.upload(cr, ci)
    ctx.filter_cheby_dev(ns, ec, 1, 2.0 / ediff, emean)
    return ctx, o, cr, ci, ec, ediff, emean


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-11), ("mixed", 1e-6)])
def test_nl_force_matches_oracle(pkg, wl, sys1, prec, tol):
    """calcEnergyForce's nonlocal forces of filtered orbitals: device against
    the oracle (pinned to calcNlPseudoPostScf) on the oracle's own filter."""
    s, ns = sys1, 6
    p = pkg.SDFT_PREC_FP64 if prec == "fp64" else pkg.SDFT_PREC_MIXED
    ctx, o, cr, ci, ec, ediff, emean = _filtered_ctx(pkg, wl, s, p, ns, 33)
    try:
        f, ep = ctx.nl_force_dev(ns, 0, occ=2.0, nsto_total=ns)
        ek, ep2 = ctx.energy_chempot_dev(ns, 0, occ=2.0, nsto_total=ns)
    finally:
        ctx.close()
    orr, oii = (a[0] for a in o.filter_cheby(cr, ci, ec, 1, 2.0 / ediff, emean))
    fo, eo = o.nl_force(orr, oii)
    fo, eo = fo * 2.0 / ns, eo * 2.0 / ns
    assert f.shape == fo.shape
    assert np.abs(f - fo).max() <= tol * np.abs(fo).max()
    assert abs(ep - eo) <= tol * abs(eo) and abs(ep - ep2) <= 1e-12 * abs(ep2)


def test_nl_force_is_energy_gradient_64_atoms(pkg, wl, sys2):
    """Size-independent property at the 64-atom cell (FP64): the device force
    equals minus the central difference of the device E_NL
    (energy_chempot_dev) with one atom moved by +-h, on the same resident
    filtered orbitals."""
    s, ns = sys2, 8
    ctx, *_ = _filtered_ctx(pkg, wl, s, pkg.SDFT_PREC_FP64, ns, 7, L=16)
    try:
        ctx.energy_chempot_dev(ns, 0, occ=2.0, nsto_total=ns)  # allocates its reduction scratch
        b0 = ctx.device_bytes
        f, _ = ctx.nl_force_dev(ns, 0, occ=2.0, nsto_total=ns)
        p0 = np.asarray(s["kb_desc"]["pos"], float).reshape(-1)
        h = 1e-4
        for a, d in ((0, 0), (17, 1), (63, 2)):
            e = []
            for sg in (1, -1):
                pos = p0.copy()
                pos[3 * a + d] += sg * h
                ctx.set_kb(dict(s["kb_desc"], pos=pos))
                e.append(ctx.energy_chempot_dev(ns, 0, occ=2.0, nsto_total=ns)[1])
            fd = -(e[0] - e[1]) / (2 * h)
            assert abs(fd - f[a, d]) <= 1e-6 * np.abs(f).max(), (a, d, fd, f[a, d])
        # rebuilding the projectors releases the old set (and the force's Z copy)
        assert ctx.device_bytes == b0
    finally:
        ctx.close()


def test_nl_force_mixed_matches_fp64_64_atoms(pkg, sys2):
    """64 atoms, 40 orbitals: the INT8 tensor-core projections give the FP64
    forces to 1e-6 of the largest component (orbitals taken as filtered
    unchanged, T_0 only, so both modes hold identical inputs)."""
    s, ns = sys2, 40
    rng = np.random.default_rng(11)
    cr = rng.standard_normal(ns * s["ncoef"])
    ci = rng.standard_normal(ns * s["ncoef"])
    ci.reshape(ns, -1)[:, -1] = 0.0
    out = []
    for p in (pkg.SDFT_PREC_FP64, pkg.SDFT_PREC_MIXED):
        ctx = _ctx(pkg, s, p, ns)
        try:
            ctx.upload(cr, ci)
            ctx.filter_cheby_dev(ns, np.array([1.0, 0.0]), 1, 0.1, 0.0)
            out.append(ctx.nl_force_dev(ns, 0, occ=2.0, nsto_total=ns))
        finally:
            ctx.close()
    (f64_, e64), (fmx, emx) = out
    assert np.abs(fmx - f64_).max() <= 1e-6 * np.abs(f64_).max()
    assert abs(emx - e64) <= 1e-7 * abs(e64)


def test_nl_force_edges(pkg, wl, sys1):
    """One orbital; no projectors (empty force, zero energy); no filtered
    orbitals yet (an error, as energy_chempot_dev reports it)."""
    s = sys1
    ctx = _ctx(pkg, s, pkg.SDFT_PREC_FP64, 2)
    try:
        with pytest.raises(pkg.SdftError):
            ctx.nl_force_dev(1, 0)
        rng = np.random.default_rng(3)
        cr, ci = rng.standard_normal(s["ncoef"]), rng.standard_normal(s["ncoef"])
        ci[-1] = 0.0
        ctx.upload(cr, ci)
        ctx.filter_cheby_dev(1, np.array([1.0, 0.0]), 1, 0.1, 0.0)
        f, e = ctx.nl_force_dev(1, 0, occ=2.0, nsto_total=1)
        fo, eo = O.OracleSys(s).nl_force(cr, ci)
        assert np.abs(f - 2.0 * fo).max() <= 1e-11 * np.abs(fo).max() and abs(e - 2.0 * eo) <= 1e-11 * abs(eo)
        ctx.set_kb(None)
        f0, e0 = ctx.nl_force_dev(1, 0)
        assert f0.shape == (0, 3) and e0 == 0.0
    finally:
        ctx.close()
