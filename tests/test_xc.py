"""LDA exchange-correlation (excpot_pz_lda / excpot_pw_lda,
energy/cp/xc_functionals.c:268,378): the device kernel against the
reference's own functions compiled in oracle/_ref, and those against a
numpy statement of the published PZ81 / PW92 formulas."""
import numpy as np
import pytest

from oracle import ref as R

pytestmark = pytest.mark.skipif(not R.available(), reason="reference-compiled oracle (oracle/_ref) not built")


def _density(n, seed=2):
    rng = np.random.default_rng(seed)
    rho = np.abs(0.02 + 0.03 * rng.standard_normal(n)) ** 1.5  # rs from ~1e-1 to ~1e1
    rho[::97] = 0.0        # clamped to 1e-10
    rho[5::211] = -1e-6    # clamped too
    rho[7::13] = 2.0       # rs < 1 branch of PZ81
    return rho


def _pz_numpy(rho):
    r = np.where(rho <= 0.0, 1e-10, rho)
    rs = (3.0 / (4.0 * np.pi * r)) ** (1.0 / 3.0)
    x = -(3.0 * r / np.pi) ** (1.0 / 3.0)
    g, b1, b2, a, b, c, d = -0.14230, 1.05290, 0.33340, 0.03110, -0.0480, 0.00200, -0.01160
    f1 = 1.0 + b1 * np.sqrt(rs) + b2 * rs
    f2 = 1.0 + 7.0 / 6.0 * b1 * np.sqrt(rs) + 4.0 / 3.0 * b2 * rs
    lr = np.log(rs)
    cf = np.where(rs >= 1.0, g / f1, a * lr + b + c * rs * lr + d * rs)
    mu = np.where(rs >= 1.0, g / f1 * f2 / f1, a * lr + (b - a / 3.0) + 2.0 / 3.0 * c * rs * lr + (2.0 * d - c) / 3.0 * rs)
    return x + mu, 0.75 * np.sum(x * r) + np.sum(cf * r), np.sum((x + mu) * r)


@pytest.mark.parametrize("n", [1000, 13824])
def test_reference_pz_lda_matches_formula(n):
    rho = _density(n)
    v, exc, muxc = R.xc_lda(1, rho, np.zeros(n), vol=float(n))  # vol = n: energies are plain sums
    vf, ef, mf = _pz_numpy(rho)
    assert np.max(np.abs(v - vf)) < 1e-13 * np.max(np.abs(vf))
    assert abs(exc - ef) < 1e-12 * abs(ef) and abs(muxc - mf) < 1e-12 * abs(mf)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", [1, 2])
@pytest.mark.parametrize("n", [1000, 96 ** 3])
def test_device_xc_matches_reference(pkg, kind, n):
    import torch
    rho = _density(n)
    v0 = np.linspace(-1.0, 1.0, n)
    vref, eref, mref = R.xc_lda(kind, rho, v0, vol=1234.5)
    rho_d = torch.from_numpy(rho).cuda()
    v_d = torch.from_numpy(v0.copy()).cuda()
    exc, muxc = pkg.xc_lda_dev(kind, n, rho_d.data_ptr(), v_d.data_ptr(), 1234.5)
    v = v_d.cpu().numpy()
    assert np.max(np.abs(v - vref)) < 1e-13 * np.max(np.abs(vref))
    assert abs(exc - eref) < 1e-12 * abs(eref) and abs(muxc - mref) < 1e-12 * abs(mref)
