"""Generate tests/golden/cfg1_reference.npz from the reference's own C code.

Runs in the build container, where the reference tree exists and
oracle/build_ref.sh has produced oracle/_ref/libpinyref.so (the reference's
filter.c, normh.c, density.c, gen-noise.c, calc-chempot-chebyshev.c,
coeff.c, ... compiled in place).  The fixture pins the oracle and the CUDA
path on machines without the reference tree (hpsi, the KB atomic forces of
calcNlPseudoPostScf, filters, moments, the chemical potential of
calcChemPotCheby, coefficients, noise and density).

  python tests/golden/make_golden.py

Workload: the 8-atom Si cell (a = 10.26 bohr, 24^3 grid, Ecut = 10 Ha,
Gaussian V_loc, Gaussian s+p KB projectors) built by workload.make_system.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import __graft_entry__ as g  # noqa: E402
from oracle import ref as R  # noqa: E402

EMIN, EMAX = -1.0, 45.0


def main():
    if not R.available():
        raise SystemExit("oracle/_ref/libpinyref.so missing: run oracle/build_ref.sh first")
    pkg = g.load_package()
    wl = g.load_workload()
    s = wl.make_system(1, (24, 24, 24))
    nc = s["ncoef"]
    out = {"grid": np.array(s["grid"]), "ncoef": np.array(nc)}
    ka, kb, kc, b1, b2 = R.gvec(s["hmat"], wl.ECUT_HA, [20, 20, 20], nc)
    out.update(ka=ka, kb=kb, kc=kc, ib1=b1, ib2=b2)
    r = R.RefSys(s, 8)
    rng = np.random.default_rng(2024)
    cr = rng.standard_normal(4 * nc)
    ci = rng.standard_normal(4 * nc)
    ci.reshape(4, nc)[:, -1] = 0.0
    out.update(in_re=cr, in_im=ci)
    fr, fi, e = r.hpsi(cr, ci)
    out.update(hpsi_re=fr, hpsi_im=fi, hpsi_enl=np.array(e))
    fa, ea = r.nl_force(cr, ci)  # calcNlPseudoPostScf: raw KB atomic forces and energy
    out.update(nlforce=fa, nlforce_enl=np.array(ea))
    scale, em = 2.0 / (EMAX - EMIN), 0.5 * (EMAX + EMIN)
    mus = (0.2, 0.35)
    ec = np.stack([pkg.calcChebyCoeff(20, EMAX - EMIN, em, 1000.0, mu) for mu in mus], axis=1).ravel()
    a = r.filter(True, cr, ci, ec, 2, scale, em, moments=True)
    out.update(cheby_ec=ec, cheby_re=np.stack(a[0]), cheby_im=np.stack(a[1]), cheby_mom=a[2])
    nscale = 4.0 / (EMAX - EMIN)
    samp, unsc = pkg.genSampNewtonHermit(24, -2.0, 2.0, nscale, EMIN)
    nec = pkg.genCoeffNewtonHermit(24, 0.2, 1000.0, samp, unsc)
    b = r.filter(False, cr, ci, nec, 1, nscale, em, samp=samp)
    out.update(newton_samp=samp, newton_unscaled=unsc, newton_ec=nec, newton_re=b[0][0], newton_im=b[1][0])
    out.update(moments_L16=r.moments(cr, ci, 16, scale, em))
    nr, ni = r.noise(4, 10.0)
    out.update(noise_re=nr, noise_im=ni, density=r.density(nr, ni))
    out.update(coeff_cheby_L64=R.cheby_coeff(64, 40.0, 19.0, 1000.0, 0.2, 1),
               coeff_cheby_L128_sqrt=R.cheby_coeff(128, 40.0, 19.0, 1000.0, 0.2, 2))
    # mu by the reference's calcChemPotCheby on the moments of 8 noise orbitals
    nr8, ni8 = r.noise(8, 10.0)
    cemin, cemax, cL = -1.2, 42.0, 64
    mu, ne = r.chem_pot(nr8, ni8, cL, cemin, cemax, 1000.0, 2.0, s["num_elec"], 0.2, 0.05)
    out.update(chempot_moments=r.moments(nr8, ni8, cL, 2.0 / (cemax - cemin), 0.5 * (cemin + cemax)) / 8,
               chempot_args=np.array([cL, cemin, cemax, 1000.0, 2.0, s["num_elec"], 0.2, 0.05]),
               chempot_mu=np.array(mu), chempot_ne=np.array(ne))
    gs, q = R.gaussran2(1001, 10.0)
    out.update(gaussran2_seed10=gs, gaussran2_seed10_next=np.array(q),
               round_fft=np.array([[n, R.round_fft(n)] for n in (1000, 2048, 8192, 16384)]))
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cfg1_reference.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
