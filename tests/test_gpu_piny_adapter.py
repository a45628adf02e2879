"""The PINY adapter (stochastic-density-functional-theory-piny_b200/csrc/piny/
sdft_piny_adapter.c) as a drop-in: oracle/build_ref.sh links it into the
reference's own objects in place of the routines it replaces
(filterChebyPolyHerm, filterNewtonPolyHerm, normHCheby, normHNewtonHerm,
calcChebyMoments, calcCoefForceWrapSCF, rhoCalcRealStoHybrid) and the same
harness drives the reference's structures and callers.  The harness keeps its
own genNoiseOrbitalReal there (it injects the orbitals of calcChebyMoments), so
the adapter's noise is checked through its body, sdft_piny_noise.  Results are checked
against the golden fixture, which the reference alone produced, in both
precisions (the adapter reads SDFT_PINY_PRECISION when it creates a
system's context)."""
import os

import numpy as np
import pytest

from conftest import rel_l2
from oracle import ref as R

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cfg1_reference.npz")
EMIN, EMAX = -1.0, 45.0
SCALE, EMEAN = 2.0 / (EMAX - EMIN), 0.5 * (EMAX + EMIN)

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not R.available(adapter=True), reason="oracle/_ref/libpinyref_adapter.so not built")]

# relative tolerances: FP64 as the GPU parity tests; mixed as the mixed-precision
# ones (h: H c, e: its KB energy, f: filters and moments, d: density, whose
# transforms are FP64 in both modes)
TOL = {"fp64": dict(h=1e-12, e=1e-12, f=1e-10, d=1e-12), "mixed": dict(h=2e-7, e=1e-6, f=1e-6, d=1e-10)}


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(GOLD))


def _cat(a, b):
    return np.concatenate([np.ravel(a), np.ravel(b)])


@pytest.fixture(scope="module", params=["fp64", "mixed"])
def adsys(request, sys1, gold):
    old = os.environ.get("SDFT_PINY_PRECISION")
    os.environ["SDFT_PINY_PRECISION"] = request.param
    try:
        r = R.RefSys(sys1, 8, adapter=True)
        # calcCoefForceWrapSCF: the first call creates the system's context
        fr, fi, e = r.hpsi(gold["in_re"], gold["in_im"])
    finally:
        if old is None:
            os.environ.pop("SDFT_PINY_PRECISION", None)
        else:
            os.environ["SDFT_PINY_PRECISION"] = old
    return request.param, r, (fr, fi, e)


def test_adapter_hpsi(adsys, gold):
    prec, _, (fr, fi, e) = adsys
    assert rel_l2(_cat(fr, fi), _cat(gold["hpsi_re"], gold["hpsi_im"])) < TOL[prec]["h"]
    assert abs(e - gold["hpsi_enl"]) < TOL[prec]["e"] * abs(gold["hpsi_enl"])


def test_adapter_filters_and_moments(adsys, gold):
    prec, r, _ = adsys
    t = TOL[prec]["f"]
    cr, ci = gold["in_re"], gold["in_im"]
    sr, si, mom = r.filter(True, cr, ci, gold["cheby_ec"], 2, SCALE, EMEAN, moments=True)
    for k in range(2):
        assert rel_l2(_cat(sr[k], si[k]), _cat(gold["cheby_re"][k], gold["cheby_im"][k])) < t
    assert rel_l2(mom[:20], gold["cheby_mom"][:20]) < t
    nr, ni = r.filter(False, cr, ci, gold["newton_ec"], 1, 4.0 / (EMAX - EMIN), EMEAN, samp=gold["newton_samp"])
    assert rel_l2(_cat(nr[0], ni[0]), _cat(gold["newton_re"], gold["newton_im"])) < t
    m = r.moments(cr, ci, 16, SCALE, EMEAN)
    assert rel_l2(m[:17], gold["moments_L16"][:17]) < t


def test_adapter_noise(adsys, gold):
    """genNoiseOrbitalReal through the adapter: the reference's noise orbitals
    from randSeed 10 (FP64 transforms in both precisions)."""
    _, r, _ = adsys
    nr, ni = r.noise_adapter(4, 10.0)
    assert rel_l2(_cat(nr, ni), _cat(gold["noise_re"], gold["noise_im"])) < 1e-13


def test_adapter_density(adsys, gold):
    prec, r, _ = adsys
    rho = r.density(gold["noise_re"], gold["noise_im"])
    assert rel_l2(rho, gold["density"]) < TOL[prec]["d"]

