"""B200 stochastic-DFT filter hot path (host-side Python mirror).

The compute path is the CUDA library ``lib/libsdft_b200.so`` behind the C
ABI declared in ``include/sdft_b200.h``; this module binds it with ctypes
and mirrors the reference routines' names and argument meaning
(mingchenPurdueChem/stochastic-density-functional-theory-piny):

=============================  =========================================
this module                    reference routine (file:line)
=============================  =========================================
``Context.calc_coef_force``     calcCoefForceWrapSCF  stodft/reduced-energy/energy-wrapper-scf.c:1066
``Context.normHCheby``          normHCheby            stodft/normh.c:182
``Context.normHNewtonHerm``     normHNewtonHerm       stodft/normh.c:35
``Context.filterChebyPolyHerm`` filterChebyPolyHerm   stodft/filter.c:318
``Context.filterNewtonPolyHerm`` filterNewtonPolyHerm stodft/filter.c:33
``Context.calcChebyMoments``    calcChebyMoments      stodft/calc-chempot-chebyshev.c:596
``Context.rhoCalcRealStoHybrid`` rhoCalcRealStoHybrid stodft/density.c:43
``Context.genNoiseOrbitalReal`` genNoiseOrbitalReal   stodft/gen-noise.c:162
``calcChemPotCheby``            calcChemPotCheby      stodft/calc-chempot-chebyshev.c:30
``calcChebyCoeff``              calcChebyCoeff        stodft/coeff.c:1093
``genSampNewtonHermit``         genSampNewtonHermit   stodft/coeff.c:423
``genCoeffNewtonHermit``        genCoeffNewtonHermit  stodft/coeff.c:199
``setkvec3d_sm``                setkvec3d_sm          interface/cp_ewald/set_cp_ewald.c:685
=============================  =========================================

Errors: every C call returns a status; a non-zero status raises
``SdftError`` carrying ``sdft_last_error()`` (the reference prints an
``@@@ERROR@@@`` banner and exits instead).  There is no CPU fallback: if
the library is missing, importing this package raises ``ImportError``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libsdft_b200.so")

SDFT_PREC_FP64 = 0
SDFT_PREC_MIXED = 1
SDFT_PREC_MIXED_FAST = 2

_ERRNAMES = {1: "ARG", 2: "CUDA", 3: "NOMEM", 4: "STATE", 5: "UNSUPPORTED", 6: "NODEVICE", 7: "TIMEOUT"}
SDFT_ERR_ARG, SDFT_ERR_CUDA, SDFT_ERR_NOMEM, SDFT_ERR_STATE = 1, 2, 3, 4
SDFT_ERR_UNSUPPORTED, SDFT_ERR_NODEVICE, SDFT_ERR_TIMEOUT = 5, 6, 7


class SdftError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"sdft error {code} ({_ERRNAMES.get(code, '?')}): {msg}")
        self.code = code


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} missing: build it with __graft_entry__.build() (no CPU fallback exists)")
    return C.CDLL(LIB_PATH)


lib = _load()

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_vp = C.c_void_p


class KbDesc(C.Structure):
    _fields_ = [
        ("natm", C.c_int), ("pos", _dp), ("type", _ip), ("ntype", C.c_int), ("lmax", C.c_int),
        ("lmax_type", _ip), ("nsplin_g", C.c_int), ("gmin_spl", C.c_double), ("dg_spl", C.c_double),
        ("vps", _dp), ("vpsnorm", _dp), ("gzvps0", _dp),
    ]


def _sig(name, res, args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = args
    return f


# exported symbols (also checked by tests/test_abi.py against include/sdft_b200.h)
_sig("sdft_last_error", C.c_char_p, [])
_sig("sdft_version", C.c_int, [])
_sig("sdft_gvec_count", C.c_int, [_dp, C.c_double, _ip, _ip])
_sig("sdft_gvec_fill", C.c_int, [_dp, C.c_double, _ip, C.c_int, _ip, _ip, _ip, _ip, _ip])
_sig("sdft_fft_maps", C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, _ip, _ip, _ip, _ip, _ip])
_sig("sdft_ak2_kinetic", C.c_int, [_dp, C.c_int, _ip, _ip, _ip, C.c_double, _dp])
_sig("sdft_ctx_create", C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, _ip, _ip, _ip, _dp, C.c_int, C.c_int,
                                  C.c_int, C.POINTER(_vp)])
_sig("sdft_ctx_destroy", C.c_int, [_vp])
_sig("sdft_ctx_set_kinetic_cap", C.c_int, [_vp, C.c_double])
_sig("sdft_ctx_set_vks", C.c_int, [_vp, _dp])
_sig("sdft_ctx_set_kb", C.c_int, [_vp, C.POINTER(KbDesc)])
_sig("sdft_ctx_device_bytes", C.c_longlong, [_vp])
_sig("sdft_ctx_stream", _vp, [_vp])
_sig("sdft_hpsi", C.c_int, [_vp, C.c_int, _dp, _dp, _dp, _dp, _dp])
_sig("sdft_normh_cheby", C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, _dp, _dp, _dp, _dp,
                                   _dp, _dp])
_sig("sdft_normh_newton", C.c_int, [_vp, C.c_int, C.c_double, C.c_double, C.c_double, _dp, _dp, _dp, _dp])
_sig("sdft_filter_cheby", C.c_int, [_vp, C.c_int, _dp, _dp, C.c_int, C.c_int, _dp, C.c_double, C.c_double,
                                    C.POINTER(_dp), C.POINTER(_dp), _dp])
_sig("sdft_filter_newton", C.c_int, [_vp, C.c_int, _dp, _dp, C.c_int, C.c_int, _dp, _dp, C.c_double, C.c_double,
                                     C.POINTER(_dp), C.POINTER(_dp)])
_sig("sdft_cheby_moments", C.c_int, [_vp, C.c_int, _dp, _dp, C.c_int, C.c_double, C.c_double, _dp])
_sig("sdft_density", C.c_int, [_vp, C.c_int, _dp, _dp, _dp])
_sig("sdft_noise_real", C.c_int, [_vp, C.c_int, C.c_double, C.c_int, C.c_int, _dp, _dp])
_sig("sdft_upload_orbitals", C.c_int, [_vp, C.c_int, _dp, _dp])
_sig("sdft_noise_real_dev", C.c_int, [_vp, C.c_int, C.c_double, C.c_int, C.c_int])
_sig("sdft_filter_cheby_dev", C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _dp, C.c_double, C.c_double])
_sig("sdft_filter_newton_dev", C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _dp, _dp, C.c_double, C.c_double])
_sig("sdft_cheby_moments_dev", C.c_int, [_vp, C.c_int, C.c_int, C.c_double, C.c_double, _dp])
_sig("sdft_density_dev", C.c_int, [_vp, C.c_int, C.c_int, C.c_double, _dp])
_sig("sdft_download_filtered", C.c_int, [_vp, C.c_int, C.c_int, _dp, _dp])
_sig("sdft_sync", C.c_int, [_vp])
_sig("sdft_ctx_selftest_wait", C.c_int, [_vp, C.c_longlong])
_sig("sdft_set_device_memory_limit", C.c_int, [C.c_int, C.c_longlong])
_sig("sdft_device_memory_in_use", C.c_longlong, [C.c_int])
_sig("sdft_set_device", C.c_int, [C.c_int])
_sig("sdft_vks_create", C.c_int, [C.c_int, C.c_int, C.c_int, _dp, C.c_int, _ip, _ip, _ip, C.c_int, C.POINTER(_vp)])
_sig("sdft_vks_destroy", C.c_int, [_vp])
_sig("sdft_vks_set_local", C.c_int, [_vp, C.c_int, _dp, C.c_int, _ip, C.c_int, C.c_double, C.c_double, _dp, _dp])
_sig("sdft_vks_from_rho", C.c_int, [_vp, _vp, C.c_int, _vp, _dp, _dp])
_sig("sdft_vks_get_vext", C.c_int, [_vp, _dp, _dp])
_sig("sdft_vks_local_forces", C.c_int, [_vp, _dp, _dp, C.c_double, _dp, _dp])
_sig("sdft_ewald_real", C.c_int, [C.c_int, _dp, _dp, _dp, C.c_double, C.c_double, C.c_int, C.c_double, _dp, _dp,
                                  _vp])
_sig("sdft_event_create", C.c_int, [C.c_int, C.POINTER(C.c_void_p)])
_sig("sdft_event_record", C.c_int, [_vp, _vp])
_sig("sdft_event_query", C.c_int, [_vp, C.POINTER(C.c_int)])
_sig("sdft_event_synchronize", C.c_int, [_vp])
_sig("sdft_event_elapsed_ms", C.c_int, [_vp, _vp, C.POINTER(C.c_float)])
_sig("sdft_event_destroy", C.c_int, [_vp])
_sig("sdft_launch_count", C.c_longlong, [_vp])
_sig("sdft_ctx_set_timing", C.c_int, [_vp, C.c_int])
_sig("sdft_ctx_read_timing", C.c_int, [_vp, _dp, C.POINTER(C.c_longlong)])
_sig("sdft_ctx_set_gemm_split", C.c_int, [_vp, C.c_int])
_sig("sdft_ctx_set_gemm_bn", C.c_int, [_vp, C.c_int])
_sig("sdft_ctx_set_priority", C.c_int, [_vp, C.c_int])
_sig("sdft_ctx_set_plane_threads", C.c_int, [_vp, C.c_int])
_sig("sdft_xc_lda_dev", C.c_int, [C.c_int, C.c_longlong, _vp, _vp, C.c_double, _dp, _dp, _vp])
_sig("sdft_mixer_create", C.c_int, [C.c_int, C.c_longlong, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                    C.POINTER(_vp)])
_sig("sdft_mixer_step", C.c_int, [_vp, C.c_int, _vp, _vp])
_sig("sdft_mixer_state", C.c_int, [_vp, _ip, _ip, _dp])
_sig("sdft_mixer_write_checkpoint", C.c_int, [_vp, C.c_char_p, _vp, C.c_double])
_sig("sdft_mixer_read_checkpoint", C.c_int, [_vp, C.c_char_p, _vp])
_sig("sdft_mixer_destroy", C.c_int, [_vp])
_sig("sdft_lanczos_bounds", C.c_int, [_vp, C.c_int, _dp, _dp, C.c_double, _dp, _dp, _ip, _dp, _dp])
_sig("sdft_energy_chempot_dev", C.c_int, [_vp, C.c_int, C.c_int, C.c_double, C.c_int, _dp, _dp])
_sig("sdft_nl_force_dev", C.c_int, [_vp, C.c_int, C.c_int, C.c_double, C.c_int, _dp, _dp])
_sig("sdft_batch_set_priority", C.c_int, [_vp, C.c_int])
_sig("sdft_download_density", C.c_int, [_vp, _dp])
_sig("sdft_batch_create", C.c_int, [C.c_int, C.POINTER(_vp), _ip, _ip, C.POINTER(_dp), _dp, _dp, _dp, C.POINTER(_vp)])
_sig("sdft_batch_launch", C.c_int, [_vp])
_sig("sdft_batch_sync", C.c_int, [_vp])
_sig("sdft_batch_stream", _vp, [_vp])
_sig("sdft_batch_kernel_count", C.c_longlong, [_vp])
_sig("sdft_batch_destroy", C.c_int, [_vp])
_sig("sdft_half_dots_noalloc", C.c_int, [_vp, _vp, _vp, _vp, C.c_int, C.c_int, _vp, _vp])
KERNEL_KINDS = ("stage_a_pack_cfft", "stage_b_plane_fft_vks", "stage_c_cfft_unpack_recur", "kb_proj_gemm",
                "kb_back_gemm", "density_planes", "noise_planes", "other")
_sig("sdft_round_fft", C.c_int, [C.c_int])
_sig("sdft_cheby_coeff", C.c_int, [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, _dp])
_sig("sdft_num_elec_cheby", C.c_double, [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                         C.c_double, _dp])
_sig("sdft_chempot_cheby", C.c_int, [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, _dp, C.c_double,
                                     C.c_double, C.c_double, _dp, _dp])
_sig("sdft_newton_samp", C.c_int, [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, _dp, _dp])
_sig("sdft_newton_coeff", C.c_int, [C.c_int, C.c_int, _dp, C.c_double, _dp, _dp, _dp])
_sig("sdft_gaussran2", C.c_int, [C.c_int, _dp, _dp])
_sig("sdft_gaussran2_signs_dev", C.c_int, [C.c_longlong, _dp, _vp, _vp])


def _chk(rc):
    if rc != 0:
        raise SdftError(rc, lib.sdft_last_error().decode(errors="replace"))


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


# ---------------------------------------------------------------------------
# host-side setup
# ---------------------------------------------------------------------------
def setkvec3d_sm(hmat, ecut, kmax):
    """Half G-sphere in PINY order, G = 0 last: returns (ka, kb, kc, ibreak1, ibreak2).

    hmat: 3x3 cell matrix with the cell vectors as columns (PINY hmat)."""
    h = _f64(np.asarray(hmat, dtype=np.float64).reshape(3, 3).T.reshape(9))  # column-major
    km = _i32(kmax)
    n = C.c_int()
    _chk(lib.sdft_gvec_count(_d(h), float(ecut), _i(km), C.byref(n)))
    nk = n.value
    ka, kb, kc = (np.zeros(nk + 1, np.int32) for _ in range(3))
    b1, b2 = np.zeros(nk, np.int32), np.zeros(nk, np.int32)
    _chk(lib.sdft_gvec_fill(_d(h), float(ecut), _i(km), nk, _i(ka), _i(kb), _i(kc), _i(b1), _i(b2)))
    return ka, kb, kc, b1, b2


def fft_maps(n1, n2, n3, ka, kb, kc):
    ka, kb, kc = _i32(ka), _i32(kb), _i32(kc)
    m, mc = np.zeros(len(ka), np.int32), np.zeros(len(ka), np.int32)
    _chk(lib.sdft_fft_maps(n1, n2, n3, len(ka), _i(ka), _i(kb), _i(kc), _i(m), _i(mc)))
    return m, mc


def roundFFT(n):
    return int(lib.sdft_round_fft(int(n)))


def calcChebyCoeff(L, energy_diff, energy_mean, beta, chem_pot, fun_flag=2, num_cheby_grid=None):
    """Chebyshev coefficients of F (fun_flag 1) or sqrt(F) (2) on [Emin, Emax]."""
    ng = roundFFT(32 * L) if num_cheby_grid is None else int(num_cheby_grid)
    out = np.zeros(L)
    _chk(lib.sdft_cheby_coeff(L, ng, energy_diff, energy_mean, beta, chem_pot, fun_flag, _d(out)))
    return out


def calcNumElecCheby(L, energy_diff, energy_mean, beta, chem_pot, occ, moments):
    m = _f64(moments)
    return float(lib.sdft_num_elec_cheby(L, roundFFT(32 * L), energy_diff, energy_mean, beta, chem_pot, occ, _d(m)))


def calcChemPotCheby(L, energy_diff, energy_mean, beta, occ, moments_normalised, num_elec_true, chem_pot_init,
                     gap_init):
    """Bisection on N(mu) = occ * sum_k c_k(mu) m_k; moments already divided by N_sto."""
    m = _f64(moments_normalised)
    mu, ne = C.c_double(), C.c_double()
    _chk(lib.sdft_chempot_cheby(L, energy_diff, energy_mean, beta, occ, _d(m), num_elec_true, chem_pot_init,
                                gap_init, C.byref(mu), C.byref(ne)))
    return mu.value, ne.value


def genSampNewtonHermit(L, smin, smax, scale, energy_min):
    s, u = np.zeros(L), np.zeros(L)
    _chk(lib.sdft_newton_samp(L, smin, smax, scale, energy_min, _d(s), _d(u)))
    return s, u


def genCoeffNewtonHermit(L, chem_pot, beta, samp, samp_unscale):
    mu = _f64(np.atleast_1d(chem_pot))
    ec = np.zeros(L * len(mu))
    _chk(lib.sdft_newton_coeff(L, len(mu), _d(mu), beta, _d(_f64(samp)), _d(_f64(samp_unscale)), _d(ec)))
    return ec


def set_device_memory_limit(device, nbytes):
    """Cap (bytes) on the device memory the library allocates on `device`;
    0 removes it.  Allocations past the cap raise SdftError(SDFT_ERR_NOMEM)."""
    _chk(lib.sdft_set_device_memory_limit(int(device), int(nbytes)))


def device_memory_in_use(device=0):
    """Bytes the library holds on `device`."""
    return int(lib.sdft_device_memory_in_use(int(device)))


def set_device(device):
    """Make `device` the calling thread's current CUDA device."""
    _chk(lib.sdft_set_device(int(device)))


class Event:
    """A CUDA event (timing enabled) through the library's C ABI."""

    def __init__(self, device=0):
        p = C.c_void_p()
        _chk(lib.sdft_event_create(int(device), C.byref(p)))
        self._p = p

    def record(self, stream_ptr=0):
        """Record on a stream (an int handle such as Context.stream_ptr; 0 =
        the legacy default stream)."""
        _chk(lib.sdft_event_record(self._p, C.c_void_p(int(stream_ptr or 0))))
        return self

    def query(self):
        done = C.c_int(0)
        _chk(lib.sdft_event_query(self._p, C.byref(done)))
        return bool(done.value)

    def synchronize(self):
        _chk(lib.sdft_event_synchronize(self._p))

    def elapsed_ms(self, later):
        """Device milliseconds from this event to `later`."""
        ms = C.c_float(0.0)
        _chk(lib.sdft_event_elapsed_ms(self._p, later._p, C.byref(ms)))
        return float(ms.value)

    def close(self):
        if getattr(self, "_p", None):
            lib.sdft_event_destroy(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def gaussran2(nran, seed):
    q = C.c_double(seed)
    out = np.zeros(max(nran, 1))
    _chk(lib.sdft_gaussran2(nran, C.byref(q), _d(out)))
    return out[:nran], q.value


SDFT_XC_PZ_LDA = 1
SDFT_XC_PW_LDA = 2


def xc_lda_dev(kind, n, rho_ptr, vks_ptr, vol, stream_ptr=0):
    """vks += V_xc(rho) on the device (pointers of n doubles); returns
    (E_xc, sum V_xc rho) times vol / n (the LDA step of cpGetVksStodft)."""
    exc, muxc = C.c_double(0.0), C.c_double(0.0)
    _chk(lib.sdft_xc_lda_dev(int(kind), int(n), C.c_void_p(rho_ptr), C.c_void_p(vks_ptr), float(vol), C.byref(exc),
                             C.byref(muxc), C.c_void_p(stream_ptr)))
    return exc.value, muxc.value


def gaussran2_signs_dev(nran, seed, out_ptr, stream_ptr=0):
    """Signs of gaussran2(nran, seed) (1 = negative) written as bytes to the
    device buffer at out_ptr (nran bytes) on the device generator; returns the
    generator state gaussran2 leaves."""
    q = C.c_double(seed)
    _chk(lib.sdft_gaussran2_signs_dev(int(nran), C.byref(q), C.c_void_p(out_ptr), C.c_void_p(stream_ptr)))
    return q.value


# ---------------------------------------------------------------------------
# device context
# ---------------------------------------------------------------------------
class Context:
    """One G sphere / FFT grid on one GPU (sdft_ctx)."""

    def __init__(self, n1, n2, n3, ka, kb, kc, hmat, precision=SDFT_PREC_FP64, max_states=1, device=0):
        self.n = (int(n1), int(n2), int(n3))
        self.ka, self.kb, self.kc = _i32(ka), _i32(kb), _i32(kc)
        self.ncoef = len(self.ka)
        self.hmat = np.asarray(hmat, dtype=np.float64).reshape(3, 3)
        h = _f64(self.hmat.T.reshape(9))
        self.precision = precision
        self.device = int(device)
        self.max_states = int(max_states)
        p = _vp()
        _chk(lib.sdft_ctx_create(n1, n2, n3, self.ncoef, _i(self.ka), _i(self.kb), _i(self.kc), _d(h), precision,
                                 self.max_states, device, C.byref(p)))
        self._p = p

    def close(self):
        if getattr(self, "_p", None):
            lib.sdft_ctx_destroy(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- setup
    def set_vks(self, v_filter_layout):
        v = _f64(v_filter_layout).reshape(-1)
        assert v.size == self.n[0] * self.n[1] * self.n[2]
        _chk(lib.sdft_ctx_set_vks(self._p, _d(v)))

    def set_vks_dev_ptr(self, ptr):
        """V_KS from device memory (an address, e.g. a buffer sdft_vks_from_rho filled)."""
        _chk(lib.sdft_ctx_set_vks(self._p, C.cast(C.c_void_p(int(ptr)), _dp)))

    def set_kinetic_cap(self, gcut):
        _chk(lib.sdft_ctx_set_kinetic_cap(self._p, float(gcut)))

    def set_kb(self, kb):
        """kb: dict with natm,pos,type,ntype,lmax,lmax_type,nsplin_g,gmin_spl,dg_spl,vps,vpsnorm,gzvps0"""
        if kb is None or kb["natm"] == 0:
            _chk(lib.sdft_ctx_set_kb(self._p, None))
            self._kb_keep = None
            return
        self._kb_keep = {k: (_f64(v) if k in ("pos", "vps", "vpsnorm", "gzvps0") else
                             (_i32(v) if k in ("type", "lmax_type") else v)) for k, v in kb.items()}
        k = self._kb_keep
        d = KbDesc(k["natm"], _d(k["pos"]), _i(k["type"]), k["ntype"], k["lmax"], _i(k["lmax_type"]),
                   k["nsplin_g"], k["gmin_spl"], k["dg_spl"], _d(k["vps"]), _d(k["vpsnorm"]), _d(k["gzvps0"]))
        _chk(lib.sdft_ctx_set_kb(self._p, C.byref(d)))

    @property
    def device_bytes(self):
        return int(lib.sdft_ctx_device_bytes(self._p))

    @property
    def launches(self):
        return int(lib.sdft_launch_count(self._p))

    def sync(self):
        _chk(lib.sdft_sync(self._p))

    def selftest_wait(self, polls=1000):
        """Queue the bounded-wait self-test (a wait that runs out after
        `polls` polls); the next sync() raises SdftError(SDFT_ERR_TIMEOUT)."""
        _chk(lib.sdft_ctx_selftest_wait(self._p, int(polls)))

    def set_timing(self, on=True):
        _chk(lib.sdft_ctx_set_timing(self._p, 1 if on else 0))

    def read_timing(self):
        """{kind: (total_ms, launches)} since the last read (synchronises)."""
        ms = np.zeros(8)
        n = (C.c_longlong * 8)()
        _chk(lib.sdft_ctx_read_timing(self._p, _d(ms), n))
        return {k: (float(ms[i]), int(n[i])) for i, k in enumerate(KERNEL_KINDS)}

    def _ns(self, cre):
        ns = cre.size // self.ncoef
        assert ns * self.ncoef == cre.size
        return ns

    # -- hot path (host buffers)
    def calc_coef_force(self, cre, cim, want_enl=False):
        cre, cim = _f64(cre), _f64(cim)
        fr, fi = np.zeros_like(cre), np.zeros_like(cim)
        e = C.c_double(0.0)
        _chk(lib.sdft_hpsi(self._p, self._ns(cre), _d(cre), _d(cim), _d(fr), _d(fi), C.byref(e) if want_enl else None))
        return (fr, fi, e.value) if want_enl else (fr, fi)

    def normHCheby(self, cre, cim, wf1re, wf1im, ipoly, scale, energy_mean, cpy_flag=1):
        """In place like normHCheby: returns (fcre, fcim); with cpy_flag cre/cim/wf1 rotate."""
        fr, fi = np.zeros_like(cre), np.zeros_like(cim)
        _chk(lib.sdft_normh_cheby(self._p, self._ns(cre), ipoly, cpy_flag, scale, energy_mean, _d(cre), _d(cim),
                                  _d(wf1re) if wf1re is not None else None, _d(wf1im) if wf1im is not None else None,
                                  _d(fr), _d(fi)))
        return fr, fi

    def normHNewtonHerm(self, cre, cim, scale, energy_mean, zn):
        fr, fi = np.zeros_like(cre), np.zeros_like(cim)
        _chk(lib.sdft_normh_newton(self._p, self._ns(cre), scale, energy_mean, zn, _d(cre), _d(cim), _d(fr), _d(fi)))
        return fr, fi

    def filterChebyPolyHerm(self, cre, cim, expan_coeff, num_chem_pot, scale, energy_mean, store_moments=False):
        cre, cim = _f64(cre), _f64(cim)
        ec = _f64(expan_coeff)
        L = ec.size // num_chem_pot
        ns = self._ns(cre)
        sre = [np.zeros_like(cre) for _ in range(num_chem_pot)]
        sim = [np.zeros_like(cim) for _ in range(num_chem_pot)]
        pr = (_dp * num_chem_pot)(*[_d(a) for a in sre])
        pi = (_dp * num_chem_pot)(*[_d(a) for a in sim])
        mom = np.zeros(L + 1) if store_moments else None
        _chk(lib.sdft_filter_cheby(self._p, ns, _d(cre), _d(cim), L, num_chem_pot, _d(ec), scale, energy_mean, pr, pi,
                                   _d(mom) if mom is not None else None))
        return (sre, sim, mom) if store_moments else (sre, sim)

    def filterNewtonPolyHerm(self, cre, cim, expan_coeff, samp_point, num_chem_pot, scale, energy_mean):
        cre, cim = _f64(cre), _f64(cim)
        ec, sp = _f64(expan_coeff), _f64(samp_point)
        L = ec.size // num_chem_pot
        ns = self._ns(cre)
        sre = [np.zeros_like(cre) for _ in range(num_chem_pot)]
        sim = [np.zeros_like(cim) for _ in range(num_chem_pot)]
        pr = (_dp * num_chem_pot)(*[_d(a) for a in sre])
        pi = (_dp * num_chem_pot)(*[_d(a) for a in sim])
        _chk(lib.sdft_filter_newton(self._p, ns, _d(cre), _d(cim), L, num_chem_pot, _d(ec), _d(sp), scale,
                                    energy_mean, pr, pi))
        return sre, sim

    def calcChebyMoments(self, cre, cim, L, scale, energy_mean):
        cre, cim = _f64(cre), _f64(cim)
        m = np.zeros(L + 1)
        _chk(lib.sdft_cheby_moments(self._p, self._ns(cre), _d(cre), _d(cim), L, scale, energy_mean, _d(m)))
        return m

    def rhoCalcRealStoHybrid(self, cre, cim):
        """sum_s |psi_s(r)|^2 in package layout (a fastest), unscaled."""
        cre, cim = _f64(cre), _f64(cim)
        rho = np.zeros(self.n[0] * self.n[1] * self.n[2])
        _chk(lib.sdft_density(self._p, self._ns(cre), _d(cre), _d(cim), _d(rho)))
        return rho

    def genNoiseOrbitalReal(self, nstate, seed=10.0, np_states=1, myid=0):
        cre = np.zeros(nstate * self.ncoef)
        cim = np.zeros(nstate * self.ncoef)
        _chk(lib.sdft_noise_real(self._p, nstate, seed, np_states, myid, _d(cre), _d(cim)))
        return cre, cim

    # -- hot path (device resident)
    def upload(self, cre, cim):
        cre, cim = _f64(cre), _f64(cim)
        _chk(lib.sdft_upload_orbitals(self._p, self._ns(cre), _d(cre), _d(cim)))

    def noise_dev(self, nstate, seed=10.0, np_states=1, myid=0):
        _chk(lib.sdft_noise_real_dev(self._p, nstate, seed, np_states, myid))

    def filter_cheby_dev(self, nstate, expan_coeff, num_chem_pot, scale, energy_mean):
        ec = _f64(expan_coeff)
        _chk(lib.sdft_filter_cheby_dev(self._p, nstate, ec.size // num_chem_pot, num_chem_pot, _d(ec), scale,
                                       energy_mean))

    def filter_newton_dev(self, nstate, expan_coeff, samp_point, num_chem_pot, scale, energy_mean):
        ec, sp = _f64(expan_coeff), _f64(samp_point)
        _chk(lib.sdft_filter_newton_dev(self._p, nstate, ec.size // num_chem_pot, num_chem_pot, _d(ec), _d(sp), scale,
                                        energy_mean))

    def moments_dev(self, nstate, L, scale, energy_mean):
        m = np.zeros(L + 1)
        _chk(lib.sdft_cheby_moments_dev(self._p, nstate, L, scale, energy_mean, _d(m)))
        return m

    def density_dev(self, nstate, imu=0, scale=1.0, want=True, out_ptr=None):
        """Density of the filtered orbitals; returned as a host array (want),
        or copied to the device address out_ptr (e.g. a torch tensor's
        data_ptr()), or left on the device."""
        if out_ptr is not None:
            _chk(lib.sdft_density_dev(self._p, nstate, imu, scale, C.cast(C.c_void_p(out_ptr), _dp)))
            return None
        rho = np.zeros(self.n[0] * self.n[1] * self.n[2]) if want else None
        _chk(lib.sdft_density_dev(self._p, nstate, imu, scale, _d(rho) if want else None))
        return rho

    def download_density(self):
        """The last density computed on this context (no recomputation)."""
        rho = np.zeros(self.n[0] * self.n[1] * self.n[2])
        _chk(lib.sdft_download_density(self._p, _d(rho)))
        return rho

    def set_gemm_split(self, split):
        """Split-K of the nonlocal projection GEMM (0 = cost model)."""
        _chk(lib.sdft_ctx_set_gemm_split(self._p, int(split)))

    def set_gemm_bn(self, bn):
        """Orbital columns per tile of the mixed-precision KB GEMMs: 0 (per
        call, 64 where it pads the orbital count less), 64 or 128."""
        _chk(lib.sdft_ctx_set_gemm_bn(self._p, int(bn)))

    def set_plane_threads(self, nt):
        """Threads per CTA of the FP32 plane stage: 128, 256, or 0 = the
        library's default (128 for 48 x 48 to 72 x 72 planes, 256 otherwise)."""
        _chk(lib.sdft_ctx_set_plane_threads(self._p, int(nt)))

    def set_priority(self, priority):
        """CUDA priority of the context's stream (lower = more urgent); idle only."""
        _chk(lib.sdft_ctx_set_priority(self._p, int(priority)))

    def lanczos_bounds(self, nstep=20, seed=15, margin=0.1, v0=None):
        """Spectral bounds (Emin - margin, Emax + margin) from `nstep` Lanczos
        steps on the device.  The start vector is the seeded standard normal
        orbital of workload.lanczos_bounds (Im G0 = 0) unless v0 = (re, im)
        is given.  Returns (emin, emax, alphas, betas)."""
        if v0 is None:
            rng = np.random.default_rng(seed)
            cr = rng.standard_normal(self.ncoef)
            ci = rng.standard_normal(self.ncoef)
            ci[-1] = 0.0
        else:
            cr, ci = _f64(v0[0]), _f64(v0[1])
        al = np.zeros(nstep)
        be = np.zeros(nstep)
        k = C.c_int(0)
        lo, hi = C.c_double(0.0), C.c_double(0.0)
        _chk(lib.sdft_lanczos_bounds(self._p, int(nstep), _d(cr), _d(ci), float(margin), _d(al), _d(be), C.byref(k),
                                     C.byref(lo), C.byref(hi)))
        return lo.value, hi.value, al[:k.value], be[:k.value]

    def energy_chempot_dev(self, nstate, imu=0, occ=2.0, nsto_total=None):
        """(energy_ke, energy_pnl) of the filtered orbitals for chemical
        potential imu, as calcEnergyChemPot stores them."""
        ek, ep = C.c_double(0.0), C.c_double(0.0)
        _chk(lib.sdft_energy_chempot_dev(self._p, int(nstate), int(imu), float(occ),
                                         int(nsto_total or nstate), C.byref(ek), C.byref(ep)))
        return ek.value, ep.value

    def nl_force_dev(self, nstate, imu=0, occ=2.0, nsto_total=None):
        """(forces [natm, 3], energy_pnl): the nonlocal atomic forces of the
        filtered orbitals for chemical potential imu, as calcEnergyForce forms
        them (occ / nsto_total times the calcNlPseudoPostScf sums)."""
        kb = getattr(self, "_kb_keep", None)
        natm = int(kb["natm"]) if kb else 0
        f = np.zeros(3 * max(natm, 1))
        ep = C.c_double(0.0)
        _chk(lib.sdft_nl_force_dev(self._p, int(nstate), int(imu), float(occ), int(nsto_total or nstate), _d(f),
                                   C.byref(ep)))
        return f[:3 * natm].reshape(natm, 3), ep.value

    @property
    def stream_ptr(self):
        return int(lib.sdft_ctx_stream(self._p) or 0)

    def download_filtered(self, nstate, imu=0):
        re = np.zeros(nstate * self.ncoef)
        im = np.zeros(nstate * self.ncoef)
        _chk(lib.sdft_download_filtered(self._p, nstate, imu, _d(re), _d(im)))
        return re, im


def ewald_real(hmat, pos, q, alp_ewd, rmax, ishift=0, rheal=0.0, stream=None):
    """Real-space ion-ion Ewald forces [natm, 3] and energy on the device
    (the pair term of PINY's energy_control_inter_real, vcoul_bin's fitted
    erfc; ishift 0 plain, 1 shifted to 0 at rmax, 2 switched over rheal)."""
    pos = _f64(pos).reshape(-1)
    q = _f64(q)
    h = _f64(np.asarray(hmat, dtype=np.float64).reshape(3, 3).T.reshape(9))  # column-major, as the library takes it
    f = np.zeros(3 * q.size)
    e = C.c_double(0.0)
    _chk(lib.sdft_ewald_real(int(q.size), _d(pos), _d(q), _d(h), float(alp_ewd), float(rmax), int(ishift),
                             float(rheal), _d(f), C.byref(e), stream))
    return f.reshape(-1, 3), e.value


class DensityGrid:
    """The density side of the SCF step on one grid (sdft_vks): the density
    in G space (calcRhoStoRecipFullg), the Hartree and local-pseudopotential
    parts of V_KS with the LDA exchange-correlation (cpGetVksStodft), and the
    local pseudopotential on the density sphere (controlEwdLocPreScf).

    ka, kb, kc: the half sphere of the density cutoff in PINY order with
    G = 0 last (setkvec3d_sm(hmat, 4 * Ecut, kmax) gives it); the grid must
    hold it."""

    def __init__(self, n1, n2, n3, hmat, ka, kb, kc, device=0):
        self.n = (int(n1), int(n2), int(n3))
        self.ka, self.kb, self.kc = _i32(ka), _i32(kb), _i32(kc)
        self.ncoef = len(self.ka)
        h = _f64(np.asarray(hmat, dtype=np.float64).reshape(3, 3).T.reshape(9))
        p = _vp()
        _chk(lib.sdft_vks_create(n1, n2, n3, _d(h), self.ncoef, _i(self.ka), _i(self.kb), _i(self.kc), int(device),
                                 C.byref(p)))
        self._p = p

    def set_local(self, pos, table, gmin, dg, gzvps, types=None):
        """Local pseudopotential: per-type Taylor-knot tables table[ntype][4][nsplin]
        (or one [4][nsplin] table), knots gmin + k dg, G = 0 values gzvps[ntype]."""
        pos = _f64(np.asarray(pos, dtype=np.float64).reshape(-1, 3))
        tab = _f64(table)
        nsplin = tab.shape[-1]
        ntype = tab.size // (4 * nsplin)
        types = _i32(np.zeros(len(pos), np.int32) if types is None else types)
        gz = _f64(np.atleast_1d(gzvps))
        _chk(lib.sdft_vks_set_local(self._p, len(pos), _d(pos), ntype, _i(types), nsplin, float(gmin), float(dg),
                                    _d(tab), _d(gz)))

    def vks_from_rho(self, rho, xc_kind=SDFT_XC_PZ_LDA, out_ptr=None):
        """rho: the density times the volume, package layout (a fastest), a
        host array or a device address (int).  Returns (V_KS in the filter
        layout -- None if out_ptr, a device address, received it --,
        rho(G) re, rho(G) im, [E_H, E_ext, E_xc, mu_xc])."""
        N = self.n[0] * self.n[1] * self.n[2]
        if isinstance(rho, (int, np.integer)):
            rp = C.c_void_p(int(rho))
        else:
            rho = _f64(rho)
            assert rho.size == N
            rp = C.c_void_p(rho.ctypes.data)
        v = None
        if out_ptr is None:
            v = np.zeros(N)
            vp = C.c_void_p(v.ctypes.data)
        else:
            vp = C.c_void_p(int(out_ptr))
        rg = np.zeros(2 * self.ncoef)
        e = np.zeros(4)
        _chk(lib.sdft_vks_from_rho(self._p, rp, int(xc_kind), vp, _d(rg), _d(e)))
        return v, rg[:self.ncoef], rg[self.ncoef:], e

    def vext(self):
        re, im = np.zeros(self.ncoef), np.zeros(self.ncoef)
        _chk(lib.sdft_vks_get_vext(self._p, _d(re), _d(im)))
        return re, im

    def local_forces(self, q, q_pseud, alp_ewd):
        """Local-pseudopotential + Ewald reciprocal forces [natm, 3] from the
        last vks_from_rho density, and [vrecip, vself, vbgr] (calcLocExtPostScf,
        ewald3d_selfbgr_cp).  q: per-atom charges; q_pseud: per-type."""
        q = _f64(q)
        qp = _f64(np.atleast_1d(q_pseud))
        f = np.zeros(3 * q.size)
        e = np.zeros(3)
        _chk(lib.sdft_vks_local_forces(self._p, _d(q), _d(qp), float(alp_ewd), _d(f), _d(e)))
        return f.reshape(-1, 3), e

    def close(self):
        if getattr(self, "_p", None):
            lib.sdft_vks_destroy(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DensityMixer:
    """genDensityMix (stodft/diis.c:34) on the device (sdft_mixer_*), with
    checkpointOutput / checkpointInput files (stodft/checkpointIO.c).
    step() takes and returns numpy arrays, or device pointers (ints)."""

    def __init__(self, n, num_diis, num_step_mix, mix_ratio_big, mix_ratio_sm, mix_ratio_sm2, device=0):
        self.n = int(n)
        p = _vp()
        _chk(lib.sdft_mixer_create(int(device), self.n, int(num_diis), int(num_step_mix), float(mix_ratio_big),
                                   float(mix_ratio_sm), float(mix_ratio_sm2), C.byref(p)))
        self._p = p

    @staticmethod
    def _ptr(a):
        return C.c_void_p(a) if isinstance(a, int) else a.ctypes.data_as(_vp)

    def step(self, iscf, rho_correct, rho=None):
        """One SCF step; returns rho (the mixed density; unchanged at iscf 0)."""
        if isinstance(rho_correct, int):
            if not isinstance(rho, int):
                raise TypeError("device rho_correct needs a device rho pointer")
            _chk(lib.sdft_mixer_step(self._p, int(iscf), C.c_void_p(rho_correct), C.c_void_p(rho)))
            return rho
        rc = _f64(rho_correct)
        out = np.zeros(self.n) if rho is None else rho
        _chk(lib.sdft_mixer_step(self._p, int(iscf), self._ptr(rc), self._ptr(out)))
        return out

    def state(self):
        it, nd = C.c_int(0), C.c_int(0)
        coef = np.zeros(16)
        _chk(lib.sdft_mixer_state(self._p, C.byref(it), C.byref(nd), _d(coef)))
        return it.value, nd.value, coef[:nd.value]

    def write_checkpoint(self, path, rho, vol):
        r = rho if isinstance(rho, int) else _f64(rho)
        _chk(lib.sdft_mixer_write_checkpoint(self._p, str(path).encode(), self._ptr(r), float(vol)))

    def read_checkpoint(self, path):
        rho = np.zeros(self.n)
        _chk(lib.sdft_mixer_read_checkpoint(self._p, str(path).encode(), self._ptr(rho)))
        return rho

    def close(self):
        if getattr(self, "_p", None):
            lib.sdft_mixer_destroy(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Filters + densities of several contexts (systems) captured as one CUDA
    graph (sdft_batch_*): every context is a concurrent branch and
    launch() replays the whole batch with one graph launch."""

    def __init__(self, ctxs, nstate, L, coeffs, scale, emean, occ_over_nsto):
        n = len(ctxs)
        self._ctxs = list(ctxs)
        self._coeffs = [_f64(c) for c in coeffs]
        arr = (_vp * n)(*[c._p for c in ctxs])
        cptr = (_dp * n)(*[_d(c) for c in self._coeffs])
        ns, Ls = _i32(nstate), _i32(L)
        sc, em, oc = _f64(scale), _f64(emean), _f64(occ_over_nsto)
        p = _vp()
        _chk(lib.sdft_batch_create(n, arr, _i(ns), _i(Ls), cptr, _d(sc), _d(em), _d(oc), C.byref(p)))
        self._p = p

    def launch(self):
        _chk(lib.sdft_batch_launch(self._p))

    def sync(self):
        _chk(lib.sdft_batch_sync(self._p))

    def set_plane_threads(self, nt):
        """Threads per CTA of the FP32 plane stage: 128, 256, or 0 = the
        library's default (128 for 48 x 48 to 72 x 72 planes, 256 otherwise)."""
        _chk(lib.sdft_ctx_set_plane_threads(self._p, int(nt)))

    def set_priority(self, priority):
        """CUDA priority of the stream the graph is launched into; idle only."""
        _chk(lib.sdft_batch_set_priority(self._p, int(priority)))

    @property
    def stream_ptr(self):
        return int(lib.sdft_batch_stream(self._p) or 0)

    @property
    def kernels_per_launch(self):
        return int(lib.sdft_batch_kernel_count(self._p))

    def close(self):
        if getattr(self, "_p", None):
            lib.sdft_batch_destroy(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
