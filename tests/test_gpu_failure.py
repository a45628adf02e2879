"""Failure paths on the device, in forms that fault and hang nothing.

* A bounded device wait that runs out: the self-test kernel waits on an
  mbarrier that nothing arrives at, through the tensor-core GEMMs' own
  bounded-wait helper capped at a few hundred polls.  The host must read
  SDFT_ERR_TIMEOUT at the next sync, once, and the context must then compute
  correct results again (FP64 and the mixed form whose GEMMs share the
  error word).
* An allocation refused on the host: a cap on the library's device memory
  just above what it holds makes the next large allocation fail with
  SDFT_ERR_NOMEM.  The cap holds, a refused call leaks nothing, the failed
  call leaves its context usable, a context that cannot be created frees
  what it took, and lifting the cap restores normal service.
"""
import numpy as np
import pytest

from conftest import rel_l2
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _ctx(pkg, s, nmax, prec=0):
    c = pkg.Context(*s["grid"], s["ka"], s["kb"], s["kc"], s["hmat"], precision=prec, max_states=nmax)
    c.set_vks(s["vks"])
    c.set_kb(s["kb_desc"])
    return c


def _rand(nc, ns, seed):
    rng = np.random.default_rng(seed)
    cr = rng.standard_normal(ns * nc)
    ci = rng.standard_normal(ns * nc)
    ci.reshape(ns, nc)[:, -1] = 0.0
    return cr, ci


@pytest.mark.parametrize("prec,tol", [(0, 1e-12), (1, 2e-7)])
def test_wait_that_runs_out_reports_timeout_once(pkg, sys1, prec, tol):
    c = _ctx(pkg, sys1, 4, prec)
    try:
        c.selftest_wait(500)
        with pytest.raises(pkg.SdftError) as e:
            c.sync()
        assert e.value.code == pkg.SDFT_ERR_TIMEOUT
        c.sync()  # reported once, then cleared
        cr, ci = _rand(sys1["ncoef"], 3, 31)
        fr, fi = c.calc_coef_force(cr, ci)
        c.sync()
        orr, oi = O.OracleSys(sys1).hpsi(cr, ci)
        assert rel_l2(np.concatenate([fr, fi]), np.concatenate([orr, oi])) < tol
        with pytest.raises(pkg.SdftError) as e:
            c.selftest_wait(0)  # outside 1..2^22: refused before any launch
        assert e.value.code == pkg.SDFT_ERR_ARG
    finally:
        c.close()


def test_allocation_cap_reports_nomem_and_context_stays_usable(pkg, sys1):
    dev = 0
    base = pkg.device_memory_in_use(dev)
    c = _ctx(pkg, sys1, 6)
    try:
        assert pkg.device_memory_in_use(dev) - base >= c.device_bytes > 0
        emin, emax = -1.0, 45.0
        scale, em = 2.0 / (emax - emin), 0.5 * (emin + emax)
        ec2 = np.stack([pkg.calcChebyCoeff(12, emax - emin, em, 1000.0, mu) for mu in (0.2, 0.3)], axis=1).ravel()
        cr, ci = c.genNoiseOrbitalReal(6, seed=5.0)
        o = O.OracleSys(sys1)
        oa, ob = o.filter_cheby(cr, ci, ec2[0::2], 1, scale, em)
        (a,), (b,) = c.filterChebyPolyHerm(cr, ci, ec2[0::2], 1, scale, em)  # its buffers now exist
        # the two-potential filter needs a second accumulator block: refused under the cap
        held = pkg.device_memory_in_use(dev)
        pkg.set_device_memory_limit(dev, held + 1024)
        with pytest.raises(pkg.SdftError) as e:
            c.filterChebyPolyHerm(cr, ci, ec2, 2, scale, em)
        assert e.value.code == pkg.SDFT_ERR_NOMEM
        after = pkg.device_memory_in_use(dev)
        assert after <= held + 1024  # the cap held; smaller scratch may have grown first
        with pytest.raises(pkg.SdftError) as e:  # refused again, and nothing leaks
            c.filterChebyPolyHerm(cr, ci, ec2, 2, scale, em)
        assert e.value.code == pkg.SDFT_ERR_NOMEM
        assert pkg.device_memory_in_use(dev) == after
        # a new context does not fit either: it frees what it took
        with pytest.raises(pkg.SdftError) as e:
            _ctx(pkg, sys1, 6)
        assert e.value.code == pkg.SDFT_ERR_NOMEM
        assert pkg.device_memory_in_use(dev) == after
        # the context still computes what fits (one potential, no new allocation)
        (a,), (b,) = c.filterChebyPolyHerm(cr, ci, ec2[0::2], 1, scale, em)
        assert rel_l2(np.concatenate([a, b]), np.concatenate([oa[0], ob[0]])) < 1e-10
        assert pkg.device_memory_in_use(dev) == after
        # cap lifted: the refused call now runs and is correct
        pkg.set_device_memory_limit(dev, 0)
        sr, si = c.filterChebyPolyHerm(cr, ci, ec2, 2, scale, em)
        osr, osi = o.filter_cheby(cr, ci, ec2, 2, scale, em)
        for k in range(2):
            assert rel_l2(np.concatenate([sr[k], si[k]]), np.concatenate([osr[k], osi[k]])) < 1e-10
    finally:
        pkg.set_device_memory_limit(dev, 0)
        c.close()
    c2 = _ctx(pkg, sys1, 2)
    c2.close()
