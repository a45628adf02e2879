"""sdft_half_dots_noalloc (allocation-free, static device scratch) against
the moments entry point sdft_cheby_moments: per orbital, <chi|chi> is
moment 0 and <chi|T_1 chi> = <chi|normH chi> is moment 1.  Two calls in a
row must both match (the scratch carries nothing from one call to the
next).  Collected last on purpose: it must also pass after every other GPU
test has run in the same process."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative to <chi|chi>; both sides sum the same products in different orders


def test_half_dots_noalloc_matches_moments(pkg, sys1):
    import torch

    s, ns = sys1, 5
    nc = s["ncoef"]
    c = pkg.Context(*s["grid"], s["ka"], s["kb"], s["kc"], s["hmat"], precision=pkg.SDFT_PREC_FP64, max_states=ns)
    c.set_vks(s["vks"])
    c.set_kb(s["kb_desc"])
    emin, emax = -1.0, 45.0
    scale, em = 2.0 / (emax - emin), 0.5 * (emin + emax)
    cr, ci = c.genNoiseOrbitalReal(ns, seed=7.0)
    hr, hi = c.normHCheby(cr.copy(), ci.copy(), None, None, 1, scale, em, cpy_flag=0)
    m0, m1 = np.empty(ns), np.empty(ns)
    for k in range(ns):
        m = c.calcChebyMoments(cr[k * nc:(k + 1) * nc], ci[k * nc:(k + 1) * nc], 2, scale, em)
        m0[k], m1[k] = m[0], m[1]
    c.close()

    dev = torch.device("cuda", torch.cuda.current_device())
    a_re, a_im, h_re, h_im = (torch.tensor(x, dtype=torch.float64, device=dev) for x in (cr, ci, hr, hi))
    out = torch.empty(ns, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    fn = pkg.lib.sdft_half_dots_noalloc
    for _ in range(2):
        for b_re, b_im, ref in ((a_re, a_im, m0), (h_re, h_im, m1)):
            out.fill_(float("nan"))
            rc = fn(a_re.data_ptr(), a_im.data_ptr(), b_re.data_ptr(), b_im.data_ptr(), nc, ns, out.data_ptr(),
                    stream)
            assert rc == 0, pkg.lib.sdft_last_error()
            torch.cuda.synchronize(dev)
            got = out.cpu().numpy()
            assert np.all(np.abs(got - ref) <= TOL * m0), (got, ref)

    # more orbitals than the static scratch holds: rejected before any launch
    rc = fn(a_re.data_ptr(), a_im.data_ptr(), a_re.data_ptr(), a_im.data_ptr(), 1, 1025, out.data_ptr(), stream)
    assert rc == 1 and b"1024" in pkg.lib.sdft_last_error()


def test_half_dots_noalloc_at_the_limit(pkg):
    """1024 orbitals (the whole static scratch) of 5000 coefficients, which is
    not a multiple of the 8 x 256 coefficients one pass of the slices covers,
    so the last slice of every orbital is partial; against the weighted sum
    in numpy, twice in a row."""
    import torch

    ns, nc = 1024, 5000
    rng = np.random.default_rng(11)
    host = [rng.standard_normal(ns * nc) for _ in range(4)]
    ar, ai, br, bi = (h.reshape(ns, nc) for h in host)
    ref = 2.0 * (np.einsum("sg,sg->s", ar, br) + np.einsum("sg,sg->s", ai, bi)) - ar[:, -1] * br[:, -1]
    scale = 2.0 * (np.abs(ar * br).sum(axis=1) + np.abs(ai * bi).sum(axis=1))
    dev = torch.device("cuda", torch.cuda.current_device())
    d = [torch.tensor(h, dtype=torch.float64, device=dev) for h in host]
    out = torch.empty(ns, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for _ in range(2):
        out.fill_(float("nan"))
        rc = pkg.lib.sdft_half_dots_noalloc(d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), d[3].data_ptr(), nc,
                                            ns, out.data_ptr(), stream)
        assert rc == 0, pkg.lib.sdft_last_error()
        torch.cuda.synchronize(dev)
        got = out.cpu().numpy()
        assert np.all(np.abs(got - ref) <= 1e-13 * scale)
