"""Restatement of the density side of the reference's SCF step in numpy.

TEST INFRASTRUCTURE ONLY (the checker of sdft_vks_*; never called by the
product path).  Follows, on one grid (cp_dual_grid_opt 0), periodic cell,
spin-unpolarised:
* controlEwdLocPreScf (stodft/reduced-energy/cp-energy-eext-stodft.c:340-470):
  vext(G) = (1/vol) sum_a v(|G|) (cos, -sin)(2 pi k.s_a), s_a = h^-1 r_a,
  v by get_vpsnow's cubic (energy/cp/cp_energy_eext.c:2139), vext(0) =
  (1/vol) sum_a gzvps;
* calcRhoStoRecipFullg (stodft/density.c:699): rho(G) = (1/N) sum_r rho(r)
  e^{-iG.r} (para_fft_gen3d_bck_to_g with its 1/N: the sign its code applies,
  pinned against the reference run), on the half sphere;
* cpGetVksStodft (stodft/reduced-energy/cp-energy-ee-rho-stodft.c:644-1007):
  E_H, E_ext, V(G) = vext + 4 pi rho/(|G|^2 vol), V(r) = sum over G and -G of
  V(G) e^{+iG.r}, + V_xc of rho/vol (PZ81, energy/cp/xc_functionals.c:268),
  transposed to the filter layout (c fastest).
Grids are in the package layout, a fastest: index ia + n1 (ib + n2 ic)."""
from __future__ import annotations

import math

import numpy as np


def _hinv(hmat):
    return np.linalg.inv(np.asarray(hmat, dtype=np.float64).reshape(3, 3))


def gvec_cart(hmat, ka, kb, kc):
    """G = 2 pi h^-T k (the xk, yk, zk of the reference's loops)."""
    hi = _hinv(hmat)
    k = np.stack([ka, kb, kc], axis=1).astype(np.float64)
    return 2.0 * math.pi * k @ hi


def spline(tab, nsplin, gmin, dg, g):
    """get_vpsnow on one Taylor-knot table tab[4][nsplin]."""
    tab = np.asarray(tab, dtype=np.float64).reshape(4, nsplin)
    iii = np.floor((g - gmin) / dg).astype(np.int64) + 1
    iii = np.clip(iii, 1, nsplin)
    h = g - ((iii - 1) * dg + gmin)
    k = iii - 1
    return ((tab[3, k] * h + tab[2, k]) * h + tab[1, k]) * h + tab[0, k]


def vext(hmat, ka, kb, kc, pos, vtab, nsplin, gmin, dg, gzvps):
    """vext on the half sphere (G = 0 last), one atom type."""
    vol = abs(np.linalg.det(np.asarray(hmat, dtype=np.float64).reshape(3, 3)))
    g = np.linalg.norm(gvec_cart(hmat, ka[:-1], kb[:-1], kc[:-1]), axis=1)
    v = spline(vtab, nsplin, gmin, dg, g)
    s = np.asarray(pos, dtype=np.float64) @ _hinv(hmat).T  # s_a = h^-1 r_a
    k = np.stack([ka[:-1], kb[:-1], kc[:-1]], axis=1).astype(np.float64)
    cs, sn = np.zeros(len(k)), np.zeros(len(k))
    for a in range(0, len(k), 4096):  # blocks of G: the phases of one block at a time
        arg = 2.0 * math.pi * (k[a:a + 4096] @ s.T)  # [G, atom]
        cs[a:a + 4096] = np.cos(arg).sum(axis=1)
        sn[a:a + 4096] = np.sin(arg).sum(axis=1)
    re = np.append(cs * v / vol, len(pos) * gzvps / vol)
    im = np.append(-sn * v / vol, 0.0)
    return re, im


def pz_lda(rho):
    """PZ81 exchange-correlation: (V_xc, sum e_xc rho, sum V_xc rho) per point."""
    r = np.where(rho <= 0.0, 1e-10, rho)
    rs = (3.0 / (4.0 * np.pi * r)) ** (1.0 / 3.0)
    x = -(3.0 * r / np.pi) ** (1.0 / 3.0)
    g, b1, b2, a, b, c, d = -0.14230, 1.05290, 0.33340, 0.03110, -0.0480, 0.00200, -0.01160
    f1 = 1.0 + b1 * np.sqrt(rs) + b2 * rs
    f2 = 1.0 + 7.0 / 6.0 * b1 * np.sqrt(rs) + 4.0 / 3.0 * b2 * rs
    lr = np.log(rs)
    cf = np.where(rs >= 1.0, g / f1, a * lr + b + c * rs * lr + d * rs)
    mu = np.where(rs >= 1.0, g / f1 * f2 / f1,
                  a * lr + (b - a / 3.0) + 2.0 / 3.0 * c * rs * lr + (2.0 * d - c) / 3.0 * rs)
    return x + mu, 0.75 * np.sum(x * r) + np.sum(cf * r), np.sum((x + mu) * r)


def vks_from_rho(grid, hmat, ka, kb, kc, vre, vim, rho_in, xc=True):
    """Returns (V_KS in the filter layout, rho(G) re, im, [E_H, E_ext, E_xc, mu_xc])."""
    n1, n2, n3 = grid
    N = n1 * n2 * n3
    vol = abs(np.linalg.det(np.asarray(hmat, dtype=np.float64).reshape(3, 3)))
    z = np.asarray(rho_in, dtype=np.float64).reshape(n3, n2, n1)  # [ic, ib, ia]
    zg = np.fft.fftn(z) / N  # (1/N) sum_r z e^{-2 pi i k.r}
    ia, ib, ic = np.mod(ka, n1), np.mod(kb, n2), np.mod(kc, n3)
    rg = zg[ic, ib, ia]
    rre, rim = rg.real.copy(), rg.imag.copy()
    rim[-1] = 0.0
    g2 = (gvec_cart(hmat, ka, kb, kc) ** 2).sum(axis=1)
    gh = 4.0 * math.pi / (g2[:-1] * vol)
    eh = 2.0 * np.sum(0.5 * gh * (rre[:-1] ** 2 + rim[:-1] ** 2))
    eext = 2.0 * np.sum(vre[:-1] * rre[:-1] + vim[:-1] * rim[:-1]) + vre[-1] * rre[-1]
    Vr = np.append(vre[:-1] + gh * rre[:-1], vre[-1])
    Vi = np.append(vim[:-1] + gh * rim[:-1], 0.0)
    vg = np.zeros((n3, n2, n1), dtype=np.complex128)
    vg[np.mod(-kc[:-1], n3), np.mod(-kb[:-1], n2), np.mod(-ka[:-1], n1)] = Vr[:-1] - 1j * Vi[:-1]
    vg[ic, ib, ia] = Vr + 1j * Vi
    v = (np.fft.ifftn(vg) * N).real  # sum_G V(G) e^{+2 pi i k.r}
    exc = muxc = 0.0
    if xc:
        vx, ex, mx = pz_lda(np.asarray(rho_in, dtype=np.float64).reshape(n3, n2, n1) / vol)
        v = v + vx
        exc, muxc = ex * vol / N, mx * vol / N
    vf = np.ascontiguousarray(np.transpose(v, (2, 1, 0))).reshape(-1)  # [ia][ib][ic], c fastest
    return vf, rre, rim, np.array([eh, eext, exc, muxc])


def local_forces(hmat, ka, kb, kc, pos, q, q_pseud, vtab, nsplin, gmin, dg, rre, rim, alp):
    """control_ewd_loc (energy/cp/cp_energy_eext.c:646-1290) for a periodic
    cell, one atom type, ewaldLocalOpt 0, with ewald3d_selfbgr_cp (:2200):
    over the half sphere (G != 0),
      vtemp_a = v(|G|) - 4 pi (q_a - q_pseud) / G^2,
      S = sum_b q_b e^{i 2 pi k.s_b},  preg = exp(-G^2 / 4 alp^2) 4 pi / (G^2 vol),
      F_a += G [(2 preg Re S q_a + 2 rho_r vtemp_a / vol) sin(2 pi k.s_a)
              - (2 preg Im S q_a - 2 rho_i vtemp_a / vol) cos(2 pi k.s_a)],
      vrecip = sum preg |S|^2;
    vself = -alp / sqrt(pi) sum q^2, vbgr = -pi (sum q)^2 / (2 alp^2 vol).
    Returns (F [natm, 3], [vrecip, vself, vbgr])."""
    h = np.asarray(hmat, dtype=np.float64).reshape(3, 3)
    vol = abs(np.linalg.det(h))
    q = np.asarray(q, dtype=np.float64)
    s = np.asarray(pos, dtype=np.float64) @ _hinv(hmat).T
    k = np.stack([ka[:-1], kb[:-1], kc[:-1]], axis=1).astype(np.float64)
    G = gvec_cart(hmat, ka[:-1], kb[:-1], kc[:-1])
    g2 = (G ** 2).sum(axis=1)
    v = spline(vtab, nsplin, gmin, dg, np.sqrt(g2))
    preg = np.exp(-g2 / (4.0 * alp * alp)) * 4.0 * math.pi / (g2 * vol)
    rre, rim = np.asarray(rre)[:-1], np.asarray(rim)[:-1]  # G != 0
    F = np.zeros((len(q), 3))
    vrec = 0.0
    for a0 in range(0, len(k), 4096):
        sl = slice(a0, a0 + 4096)
        arg = 2.0 * math.pi * (k[sl] @ s.T)  # [G, atom]
        cs, sn = np.cos(arg), np.sin(arg)
        sr_, si_ = cs @ q, sn @ q
        vrec += np.sum(preg[sl] * (sr_ * sr_ + si_ * si_))
        vt = v[sl, None] - 4.0 * math.pi * (q[None, :] - q_pseud) / g2[sl, None]
        pr = 2.0 * preg[sl, None] * sr_[:, None] * q[None, :] + 2.0 * rre[sl, None] * vt / vol
        pi_ = 2.0 * preg[sl, None] * si_[:, None] * q[None, :] - 2.0 * rim[sl, None] * vt / vol
        w = pr * sn - pi_ * cs  # [G, atom]
        F += w.T @ G[sl]
    vself = -np.dot(q, q) * alp / math.sqrt(math.pi)
    vbgr = -0.5 * q.sum() ** 2 * math.pi / (alp * alp * vol)
    return F, np.array([vrec, vself, vbgr])


# The reference's fit of erfc(x) (vcoul_bin, interface/inter_params/
# spline_fit.c:371-380): erfc(x) ~ sum_i e_i t^i exp(-x^2), t = 1/(1 + p x),
# within 2.3e-9 of erfc on [0, 6].
_GERFC_P = 0.3614
_GERFC_E = (0.2041422096422003, 0.1997535956961481, 0.2213176596405576, 0.03360430734640255,
            0.4732592578721755, -0.509078520069735, 0.6772631491947646, -0.369912979092217,
            0.06965131976970335)


def coul_pair(r, qij, alp, rmax, ishift=0, rheal=0.0):
    """vcoul_bin's real-space Ewald pair term (spline_fit.c:415-437, iperd >
    0) with spline_vdv's switch and shift (:61-72, :87-92), evaluated at r
    instead of tabulated:
      v  = qij gerfc(alp r) / r,
      dv = (gerfc/r^2 + dgerfc/r) qij / r = -(dv/dr) / r,
    ishift 2: v sw, dv sw + v dsw, sw = 1 + rp^2 (2 rp - 3), rp =
    clip((r - rmax + rheal)/rheal, 0, 1), dsw = -6 (rp/rheal)(rp - 1)/r;
    ishift 1: v - v(rmax).  Returns (v, dv)."""
    r = np.asarray(r, dtype=np.float64)

    def g_dg(rr):
        x = rr * alp
        ex = np.exp(-x * x)
        t = 1.0 / (1.0 + _GERFC_P * x)
        poly = np.zeros_like(rr)
        dpoly = np.zeros_like(rr)
        for i in range(len(_GERFC_E), 0, -1):
            poly = poly * t + _GERFC_E[i - 1]
            dpoly = dpoly * t + i * _GERFC_E[i - 1]
        g = poly * t * ex
        dg = dpoly * t * t * ex * _GERFC_P * alp + 2.0 * alp * alp * g * rr
        return g, dg

    g, dg = g_dg(r)
    v = qij * g / r
    dv = (g / (r * r) + dg / r) * qij / r
    if ishift == 2:
        rp = np.clip((r - rmax + rheal) / rheal, 0.0, 1.0)
        sw = 1.0 + rp * rp * (2.0 * rp - 3.0)
        dsw = -6.0 * (rp / rheal) * (rp - 1.0) / r
        v, dv = v * sw, dv * sw + v * dsw
    elif ishift == 1:
        gm, _ = g_dg(np.array([rmax], dtype=np.float64))
        v = v - qij * gm[0] / rmax
    return v, dv


def ewald_images(hmat, rmax):
    """Lattice translations h n that can bring a pair (fractional offsets in
    (-1, 1)) within rmax: |n_i| <= ceil(rmax / w_i) + 1, w_i the cell's
    width across face i.  Returns [nimg, 3] with n = 0 first."""
    h = np.asarray(hmat, dtype=np.float64).reshape(3, 3)
    cols = [h[:, j] for j in range(3)]
    vol = abs(np.linalg.det(h))
    nmax = [int(math.ceil(rmax / (vol / np.linalg.norm(np.cross(cols[(j + 1) % 3], cols[(j + 2) % 3]))))) + 1
            for j in range(3)]
    ns = [(0, 0, 0)] + [(i, j, k) for i in range(-nmax[0], nmax[0] + 1) for j in range(-nmax[1], nmax[1] + 1)
                        for k in range(-nmax[2], nmax[2] + 1) if (i, j, k) != (0, 0, 0)]
    return np.array(ns, dtype=np.float64) @ h.T


def ewald_real(hmat, pos, q, alp, rmax, ishift=0, rheal=0.0):
    """The real-space ion-ion Ewald sum that calc-nuclei-force.c:605/635 gets
    from energy_control_inter_real (PINY's pair engine over the vcoul_bin
    table), summed directly over all pairs and periodic images with r <
    rmax: E = 1/2 sum_a sum_{b, n; (b, n) != (a, 0)} v(|r_a - r_b - h n|),
    F_a = sum dv (r_a - r_b - h n).  Positions are wrapped into the cell
    first.  Returns (F [natm, 3], E)."""
    h = np.asarray(hmat, dtype=np.float64).reshape(3, 3)
    q = np.asarray(q, dtype=np.float64)
    s = np.asarray(pos, dtype=np.float64).reshape(-1, 3) @ _hinv(hmat).T
    s -= np.floor(s)
    x = s @ h.T
    img = ewald_images(hmat, rmax)
    n = len(q)
    F = np.zeros((n, 3))
    E = 0.0
    for a in range(n):
        d = (x[a] - x)[:, None, :] - img[None, :, :]  # [b, image, 3]
        r = np.sqrt((d * d).sum(axis=2))
        m = r < rmax
        m[a, 0] = False
        v, dv = coul_pair(r[m], q[a] * q[np.nonzero(m)[0]], alp, rmax, ishift, rheal)
        E += 0.5 * v.sum()
        F[a] = (dv[:, None] * d[m]).sum(axis=0)
    return F, E
