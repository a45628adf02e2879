"""ctypes binding of the CPU oracle (sdft_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline leg as the checker; never by the product path."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def _load():
    from . import build as _b  # noqa: PLC0415
    return C.CDLL(_b.build())


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = _load()
        L = _lib
        L.oracle_gvec.restype = C.c_int
        L.oracle_gvec.argtypes = [_dp, C.c_double, _ip, C.c_int, _ip, _ip, _ip, _ip, _ip]
        L.oracle_create.restype = C.c_void_p
        L.oracle_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _ip, _ip, _ip, _ip, _ip, _dp]
        L.oracle_destroy.argtypes = [C.c_void_p]
        L.oracle_set_vks.argtypes = [C.c_void_p, _dp]
        L.oracle_set_kinetic_cap.argtypes = [C.c_void_p, C.c_double]
        L.oracle_set_kb.argtypes = [C.c_void_p, C.c_int, _dp, _ip, C.c_int, C.c_int, _ip, C.c_int, C.c_double,
                                    C.c_double, _dp, _dp, _dp]
        L.oracle_hpsi.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp, _dp, _dp]
        L.oracle_nl_force.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp, _dp]
        L.oracle_normh_cheby.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, _dp, _dp,
                                         _dp, _dp, _dp, _dp]
        L.oracle_normh_newton.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_double, _dp, _dp, _dp,
                                          _dp]
        L.oracle_filter_cheby.argtypes = [C.c_void_p, C.c_int, _dp, _dp, C.c_int, C.c_int, _dp, C.c_double,
                                          C.c_double, _dp, _dp, _dp]
        L.oracle_filter_newton.argtypes = [C.c_void_p, C.c_int, _dp, _dp, C.c_int, C.c_int, _dp, _dp, C.c_double,
                                           C.c_double, _dp, _dp]
        L.oracle_cheby_moments.argtypes = [C.c_void_p, C.c_int, _dp, _dp, C.c_int, C.c_double, C.c_double, _dp]
        L.oracle_density.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp]
        L.oracle_ran_essl.restype = C.c_double
        L.oracle_ran_essl.argtypes = [_dp]
        L.oracle_gaussran2.argtypes = [C.c_int, _dp, _dp]
        L.oracle_noise.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_int, _dp, _dp]
        L.oracle_round_fft.restype = C.c_int
        L.oracle_round_fft.argtypes = [C.c_int]
        L.oracle_cheby_coeff.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
                                         _dp]
        L.oracle_newton_samp.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, _dp, _dp]
        L.oracle_newton_coeff.argtypes = [C.c_int, C.c_int, _dp, C.c_double, _dp, _dp, _dp]
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def gvec(hmat, ecut, kmax):
    h = f64(np.asarray(hmat, float).reshape(3, 3).T.reshape(9))
    km = i32(kmax)
    n = lib().oracle_gvec(_d(h), ecut, _i(km), 0, None, None, None, None, None)
    ka, kb, kc = (np.zeros(n + 1, np.int32) for _ in range(3))
    b1, b2 = np.zeros(n + 1, np.int32), np.zeros(n + 1, np.int32)
    lib().oracle_gvec(_d(h), ecut, _i(km), n + 1, _i(ka), _i(kb), _i(kc), _i(b1), _i(b2))
    return ka, kb, kc, b1[:n], b2[:n]


class OracleSys:
    def __init__(self, sysd):
        self.n = sysd["grid"]
        self.ncoef = len(sysd["ka"])
        h = f64(np.asarray(sysd["hmat"], float).T.reshape(9))
        ib1 = i32(np.append(sysd["ib1"], 0))
        ib2 = i32(np.append(sysd["ib2"], 0))
        self._p = C.c_void_p(lib().oracle_create(*self.n, self.ncoef, _i(i32(sysd["ka"])), _i(i32(sysd["kb"])),
                                                 _i(i32(sysd["kc"])), _i(ib1), _i(ib2), _d(h)))
        lib().oracle_set_vks(self._p, _d(f64(sysd["vks"])))
        kb = sysd.get("kb_desc")
        if kb is not None and kb["natm"] > 0:
            self._keep = [f64(kb["pos"]), i32(kb["type"]), i32(kb["lmax_type"]), f64(kb["vps"]),
                          f64(kb["vpsnorm"]), f64(kb["gzvps0"])]
            pos, typ, lmt, vps, vn, gz = self._keep
            lib().oracle_set_kb(self._p, kb["natm"], _d(pos), _i(typ), kb["ntype"], kb["lmax"], _i(lmt),
                                kb["nsplin_g"], kb["gmin_spl"], kb["dg_spl"], _d(vps), _d(vn), _d(gz))

    def __del__(self):
        try:
            lib().oracle_destroy(self._p)
        except Exception:
            pass

    def hpsi(self, cre, cim, want_enl=False):
        cre, cim = f64(cre), f64(cim)
        fr, fi = np.zeros_like(cre), np.zeros_like(cim)
        e = C.c_double()
        lib().oracle_hpsi(self._p, cre.size // self.ncoef, _d(cre), _d(cim), _d(fr), _d(fi), C.byref(e))
        return (fr, fi, e.value) if want_enl else (fr, fi)

    def nl_force(self, cre, cim):
        """KB nonlocal atomic forces [natm, 3] and energy of the given orbitals
        (raw sums over them, before occ / numStateStoUp)."""
        cre, cim = f64(cre), f64(cim)
        n = self._keep[0].size // 3 if hasattr(self, "_keep") else 0
        f = np.zeros(3 * max(n, 1))
        e = C.c_double()
        lib().oracle_nl_force(self._p, cre.size // self.ncoef, _d(cre), _d(cim), _d(f), C.byref(e))
        return f[:3 * n].reshape(n, 3), e.value

    def filter_cheby(self, cre, cim, ec, nmu, scale, emean, store_moments=False):
        cre, cim, ec = f64(cre), f64(cim), f64(ec)
        L = ec.size // nmu
        sr = np.zeros(nmu * cre.size)
        si = np.zeros(nmu * cre.size)
        m = np.zeros(L + 1) if store_moments else None
        lib().oracle_filter_cheby(self._p, cre.size // self.ncoef, _d(cre), _d(cim), L, nmu, _d(ec), scale, emean,
                                  _d(sr), _d(si), _d(m) if m is not None else None)
        out = (sr.reshape(nmu, -1), si.reshape(nmu, -1))
        return out + (m,) if store_moments else out

    def filter_newton(self, cre, cim, ec, samp, nmu, scale, emean):
        cre, cim, ec, samp = f64(cre), f64(cim), f64(ec), f64(samp)
        L = ec.size // nmu
        sr = np.zeros(nmu * cre.size)
        si = np.zeros(nmu * cre.size)
        lib().oracle_filter_newton(self._p, cre.size // self.ncoef, _d(cre), _d(cim), L, nmu, _d(ec), _d(samp), scale,
                                   emean, _d(sr), _d(si))
        return sr.reshape(nmu, -1), si.reshape(nmu, -1)

    def moments(self, cre, cim, L, scale, emean):
        cre, cim = f64(cre), f64(cim)
        m = np.zeros(L + 1)
        lib().oracle_cheby_moments(self._p, cre.size // self.ncoef, _d(cre), _d(cim), L, scale, emean, _d(m))
        return m

    def density(self, cre, cim):
        cre, cim = f64(cre), f64(cim)
        rho = np.zeros(int(np.prod(self.n)))
        lib().oracle_density(self._p, cre.size // self.ncoef, _d(cre), _d(cim), _d(rho))
        return rho

    def noise(self, nstate, seed=10.0, np_states=1, myid=0):
        cre = np.zeros(nstate * self.ncoef)
        cim = np.zeros(nstate * self.ncoef)
        lib().oracle_noise(self._p, nstate, seed, np_states, myid, _d(cre), _d(cim))
        return cre, cim


def gaussran2(n, seed):
    q = C.c_double(seed)
    out = np.zeros(max(n, 1))
    lib().oracle_gaussran2(n, C.byref(q), _d(out))
    return out[:n], q.value


def round_fft(n):
    return lib().oracle_round_fft(n)


def cheby_coeff(L, ediff, emean, beta, mu, fun=2, ngrid=None):
    ng = round_fft(32 * L) if ngrid is None else ngrid
    c = np.zeros(L)
    lib().oracle_cheby_coeff(L, ng, ediff, emean, beta, mu, fun, _d(c))
    return c


def newton_samp(L, smin, smax, scale, emin):
    s, u = np.zeros(L), np.zeros(L)
    lib().oracle_newton_samp(L, smin, smax, scale, emin, _d(s), _d(u))
    return s, u


def newton_coeff(L, mu, beta, samp, unscale):
    mu = f64(np.atleast_1d(mu))
    ec = np.zeros(L * mu.size)
    lib().oracle_newton_coeff(L, mu.size, _d(mu), beta, _d(f64(samp)), _d(f64(unscale)), _d(ec))
    return ec
