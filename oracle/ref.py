"""ctypes binding of oracle/_ref/libpinyref.so: the reference's own C
sources driven by oracle/ref_harness.c.  TEST INFRASTRUCTURE ONLY."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libpinyref.so")
# the same reference objects and harness with the product's PINY adapter
# linked in place of the routines it replaces (oracle/build_ref.sh)
LIB_ADAPTER = os.path.join(HERE, "_ref", "libpinyref_adapter.so")
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_libs = {}


def available(adapter=False):
    return os.path.exists(LIB_ADAPTER if adapter else LIB)


def lib(adapter=False):
    path = LIB_ADAPTER if adapter else LIB
    if path not in _libs:
        L = C.CDLL(path)
        L.ref_create.restype = C.c_void_p
        L.ref_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _ip, _ip, _ip, _ip, _ip, _dp, _dp, C.c_int, _dp,
                                 C.c_int, C.c_double, C.c_double, _dp, _dp, C.c_double, C.c_int]
        L.ref_hpsi.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp, _dp, _dp]
        L.ref_nl_force.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp, _dp]
        L.ref_filter.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp, _dp, C.c_int, C.c_int, _dp, _dp, C.c_double,
                                 C.c_double, _dp, _dp, _dp]
        L.ref_moments.argtypes = [C.c_void_p, C.c_int, _dp, _dp, C.c_int, C.c_double, C.c_double, _dp]
        L.ref_gvec.argtypes = [_dp, C.c_double, _ip, C.c_int, _ip, _ip, _ip, _ip, _ip]
        L.ref_round_fft.restype = C.c_int
        L.ref_cheby_coeff.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, _dp]
        L.ref_newton.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, _dp, _dp, _dp]
        L.ref_gaussran2.argtypes = [C.c_int, _dp, _dp]
        L.ref_noise.argtypes = [C.c_void_p, C.c_int, C.c_double, _dp, _dp]
        L.ref_noise_adapter.argtypes = [C.c_void_p, C.c_int, C.c_double, _dp, _dp]
        L.ref_density.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp]
        L.ref_mix_create.restype = C.c_void_p
        L.ref_mix_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double]
        L.ref_mix_step.argtypes = [C.c_void_p, C.c_int, _dp, _dp]
        L.ref_mix_set_rho.argtypes = [C.c_void_p, _dp]
        L.ref_mix_checkpoint.argtypes = [C.c_void_p, C.c_char_p, C.c_double, C.c_double, C.c_double]
        L.ref_mix_checkpoint.restype = C.c_int
        L.ref_xc_lda.argtypes = [C.c_int, C.c_int, _dp, _dp, C.c_double, _dp, _dp]
        L.ref_vks.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_double, C.c_double, _dp, C.c_double, C.c_int, _dp,
                              C.c_int, _ip, _ip, _ip, _ip, _dp, _dp, _dp, _dp, _dp, _dp, _dp, C.c_double, C.c_double,
                              _dp, _dp]
        L.ref_chempot.argtypes = [C.c_void_p, C.c_int, _dp, _dp, C.c_int, C.c_double, C.c_double, C.c_double,
                                  C.c_double, C.c_double, C.c_double, C.c_double, _dp, _dp]
        L.ref_coul_table.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, C.c_double,
                                     _dp, _dp, _dp]
        L.ref_num_elec.restype = C.c_double
        L.ref_num_elec.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, _dp, C.c_double]
        _libs[path] = L
    return _libs[path]


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class RefSys:
    """One system in the reference's own data structures (single type, s+p KB)."""

    def __init__(self, s, nmax, adapter=False):
        """adapter: drive the product's PINY adapter (device path) through
        the same reference structures and callers."""
        self._L = lib(adapter)
        kb = s["kb_desc"]
        self.ncoef = len(s["ka"])
        self.N = int(np.prod(s["grid"]))
        self.natm = int(kb["natm"])
        self.keep = [i32(s["ka"]), i32(s["kb"]), i32(s["kc"]), i32(s["ib1"]), i32(s["ib2"]),
                     f64(np.asarray(s["hmat"], float).T.reshape(9)), f64(s["vks"]), f64(kb["pos"]), f64(kb["vps"]),
                     f64(kb["vpsnorm"])]
        ka, kb_, kc, b1, b2, h, v, pos, vps, vn = self.keep
        self._p = C.c_void_p(self._L.ref_create(*s["grid"], self.ncoef, _i(ka), _i(kb_), _i(kc), _i(b1), _i(b2), _d(h),
                                              _d(v), kb["natm"], _d(pos), kb["nsplin_g"], kb["gmin_spl"],
                                              kb["dg_spl"], _d(vps), _d(vn), float(kb["gzvps0"][0]), nmax))

    def hpsi(self, cre, cim):
        cre, cim = f64(cre), f64(cim)
        fr, fi = np.zeros_like(cre), np.zeros_like(cim)
        e = C.c_double()
        self._L.ref_hpsi(self._p, cre.size // self.ncoef, _d(cre), _d(cim), _d(fr), _d(fi), C.byref(e))
        return fr, fi, e.value

    def nl_force(self, cre, cim):
        """calcNlPseudoPostScf on the given orbitals: KB atomic forces [natm, 3]
        and energy, before calcEnergyForce's occ / numStateStoUp."""
        cre, cim = f64(cre), f64(cim)
        f = np.zeros(3 * self.natm)
        e = C.c_double()
        self._L.ref_nl_force(self._p, cre.size // self.ncoef, _d(cre), _d(cim), _d(f), C.byref(e))
        return f.reshape(self.natm, 3), e.value

    def filter(self, cheby, cre, cim, ec, nmu, scale, emean, samp=None, moments=False):
        cre, cim, ec = f64(cre), f64(cim), f64(ec)
        L = ec.size // nmu
        sr, si = np.zeros(nmu * cre.size), np.zeros(nmu * cre.size)
        m = np.zeros(L + 1) if moments else None
        sp = f64(samp) if samp is not None else None
        self._L.ref_filter(self._p, 1 if cheby else 0, cre.size // self.ncoef, _d(cre), _d(cim), L, nmu, _d(ec),
                         _d(sp) if sp is not None else None, scale, emean, _d(sr), _d(si),
                         _d(m) if m is not None else None)
        out = (sr.reshape(nmu, -1), si.reshape(nmu, -1))
        return out + (m,) if moments else out

    def noise(self, nstate, seed=10.0):
        re = np.zeros(nstate * self.ncoef)
        im = np.zeros(nstate * self.ncoef)
        self._L.ref_noise(self._p, nstate, seed, _d(re), _d(im))
        return re, im

    def noise_adapter(self, nstate, seed=10.0):
        """The product adapter's genNoiseOrbitalReal on these structures
        (adapter library only)."""
        re = np.zeros(nstate * self.ncoef)
        im = np.zeros(nstate * self.ncoef)
        if self._L.ref_noise_adapter(self._p, nstate, seed, _d(re), _d(im)) != 0:
            raise RuntimeError("the adapter's noise is only in the adapter library")
        return re, im

    def density(self, cre, cim):
        cre, cim = f64(cre), f64(cim)
        rho = np.zeros(self.N)
        self._L.ref_density(self._p, cre.size // self.ncoef, _d(cre), _d(cim), _d(rho))
        return rho

    def chem_pot(self, cre, cim, L, emin, emax, beta, occ, num_elec, chem_pot_init, gap_init):
        """calcChemPotCheby on these orbitals as the noise: the reference
        computes their moments itself and bisects N(mu) = num_elec.
        Returns (mu, N(mu))."""
        cre, cim = f64(cre), f64(cim)
        mu, ne = C.c_double(), C.c_double()
        self._L.ref_chempot(self._p, cre.size // self.ncoef, _d(cre), _d(cim), L, emin, emax, beta, occ, num_elec,
                            chem_pot_init, gap_init, C.byref(mu), C.byref(ne))
        return mu.value, ne.value

    def vks(self, ecut, vloc, gmin, dg, gzvps_loc, xc, rho_in, cap=1 << 22, q=None, q_pseud=0.0, alp_ewd=1.0):
        """The reference's density side of the SCF step on this system's
        cell, atoms and grid (ref_vks): the density sphere (ka, kb, kc),
        vext, rho(G), V_KS (filter layout) and [E_H, E_ext, E_xc, mu_xc].
        With atom charges q: also the local-pseudopotential + Ewald
        reciprocal forces [natm, 3] and [vrecip, vself, vbgr]."""
        rho_in = f64(rho_in)
        n = C.c_int(0)
        ka, kb, kc = (np.zeros(cap, np.int32) for _ in range(3))
        vr, vi, rr, ri = (np.zeros(cap) for _ in range(4))
        v = np.zeros(self.N)
        e = np.zeros(4)
        vloc = f64(vloc)
        qa = f64(q) if q is not None else None
        f = np.zeros(3 * self.natm)
        ee = np.zeros(3)
        rc = self._L.ref_vks(self._p, ecut, vloc.size // 4, gmin, dg, _d(vloc), gzvps_loc, int(xc), _d(rho_in), cap,
                             C.byref(n), _i(ka),
                             _i(kb), _i(kc), _d(vr), _d(vi), _d(rr), _d(ri), _d(v), _d(e),
                             _d(qa) if qa is not None else None, q_pseud, alp_ewd,
                             _d(f) if qa is not None else None, _d(ee))
        if rc:
            raise RuntimeError("ref_vks: density sphere larger than cap")
        k = n.value
        out = dict(ka=ka[:k], kb=kb[:k], kc=kc[:k], vext_re=vr[:k], vext_im=vi[:k], rhog_re=rr[:k],
                   rhog_im=ri[:k], vks=v, energies=e)
        if qa is not None:
            out.update(force=f.reshape(self.natm, 3), ewald=ee)
        return out

    def moments(self, cre, cim, L, scale, emean):
        cre, cim = f64(cre), f64(cim)
        m = np.zeros(L + 1)
        self._L.ref_moments(self._p, cre.size // self.ncoef, _d(cre), _d(cim), L, scale, emean, _d(m))
        return m


def gvec(hmat, ecut, kmax, ncoef):
    h = f64(np.asarray(hmat, float).T.reshape(9))
    km = i32(kmax)
    ka, kb, kc = (np.zeros(ncoef, np.int32) for _ in range(3))
    b1, b2 = np.zeros(ncoef, np.int32), np.zeros(ncoef, np.int32)
    lib().ref_gvec(_d(h), ecut, _i(km), ncoef, _i(ka), _i(kb), _i(kc), _i(b1), _i(b2))
    return ka, kb, kc, b1[:ncoef - 1], b2[:ncoef - 1]


def cheby_coeff(L, ediff, emean, beta, mu, fun=2):
    out = np.zeros(L)
    lib().ref_cheby_coeff(L, ediff, emean, beta, mu, fun, _d(out))
    return out


def newton(L, scale, emin, beta, mu):
    s, u, e = np.zeros(L), np.zeros(L), np.zeros(L)
    lib().ref_newton(L, scale, emin, beta, mu, _d(s), _d(u), _d(e))
    return s, u, e


def gaussran2(n, seed):
    q = C.c_double(seed)
    out = np.zeros(max(n, 1))
    lib().ref_gaussran2(n, C.byref(q), _d(out))
    return out[:n], q.value


def round_fft(n):
    return lib().ref_round_fft(n)


class RefMixer:
    """genDensityMix (stodft/diis.c:34) and checkpointOutput
    (stodft/checkpointIO.c:32) of the reference on one rank.  The handle is
    not freed (test use)."""

    def __init__(self, n, num_diis, num_step_mix, mix_ratio_big, mix_ratio_sm, mix_ratio_sm2):
        self.n = int(n)
        self._p = C.c_void_p(lib().ref_mix_create(self.n, num_diis, num_step_mix, mix_ratio_big, mix_ratio_sm,
                                                  mix_ratio_sm2))

    def set_rho(self, rho):
        lib().ref_mix_set_rho(self._p, _d(f64(rho)))

    def step(self, iscf, rho_correct):
        out = np.zeros(self.n)
        lib().ref_mix_step(self._p, int(iscf), _d(f64(rho_correct)), _d(out))
        return out

    def checkpoint(self, directory, cell):
        rc = lib().ref_mix_checkpoint(self._p, str(directory).encode(), *[float(x) for x in cell])
        if rc:
            raise OSError("checkpointOutput harness failed")
        return os.path.join(str(directory), "density-checkpoint")


def xc_lda(kind, rho, vks, vol):
    """excpot_pz_lda (kind 1) / excpot_pw_lda (kind 2) of the reference:
    returns (vks + V_xc, E_xc, mu_xc)."""
    rho = f64(rho).copy()
    v = f64(vks).copy()
    exc, muxc = C.c_double(0.0), C.c_double(0.0)
    lib().ref_xc_lda(int(kind), rho.size, _d(rho), _d(v), float(vol), C.byref(exc), C.byref(muxc))
    return v, exc.value, muxc.value


def num_elec(L, emin, emax, beta, occ, moments_normalised, mu):
    """calcNumElecCheby: occ * sum_{k<L} c_k(mu) m_k with the Chebyshev
    coefficients of F on [emin, emax]."""
    m = f64(moments_normalised)
    return lib().ref_num_elec(L, emin, emax, beta, occ, _d(m), mu)


def coul_table(n, rmin, rmax, alp, qij, ishift=0, rheal=0.0):
    """The reference's real-space Ewald pair table (ref_coul_table): its r
    grid, v and dv = -(dv/dr)/r."""
    r, v, dv = np.zeros(n), np.zeros(n), np.zeros(n)
    lib().ref_coul_table(int(n), rmin, rmax, alp, qij, int(ishift), rheal, _d(r), _d(v), _d(dv))
    return r, v, dv

