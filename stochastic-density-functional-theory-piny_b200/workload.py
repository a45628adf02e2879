"""Synthetic diamond-Si workloads for the filter hot path.

Inputs are generated, not read: seeded diamond-cubic Si supercells with a
Gaussian local potential and Gaussian s+p Kleinman-Bylander projectors
(no pseudopotential files exist for this path).

* Cell: conventional cubic cell a0 = 10.26 bohr, 8 atoms at the fcc sites
  plus the (1/4,1/4,1/4) shifted copies; supercells n x n x n.
* V_loc(r) = sum_atoms -4 exp(-|r-R|^2 / (2*0.9^2)) Ha, periodic images,
  sampled on the FFT grid in the filter layout (c fastest).  V_KS := V_loc.
* KB projectors: beta_l(r) ~ r^l exp(-r^2/(2 rc^2)), rc = 1.2 bohr,
  normalised in real space; radial form factors
      v_0(g) = 4 pi N_0 sqrt(pi/2) rc^3 exp(-g^2 rc^2/2)
      v_1(g) = 4 pi N_1 sqrt(pi/2) rc^5 g exp(-g^2 rc^2/2)
  tabulated for get_vpsnow as per-knot Taylor coefficients
  (vps0..vps3 = f, f', f''/2, f'''/6).  E_KB: s = +0.5 Ha, p = -0.5 Ha.
* Plane waves 0.5|G|^2 <= Ecut = 10 Ha (20 Ry).
"""
from __future__ import annotations

import math

import numpy as np

A0_SI = 10.26
ECUT_HA = 10.0
SIGMA_LOC = 0.9
V0_LOC = -4.0
RC_KB = 1.2
EKB = (0.5, -0.5)  # s, p

CONFIGS = {
    # name: (supercell n, grid, n_orbitals, L, polynomial)
    "cfg1": dict(nrep=1, grid=(24, 24, 24), nsto=16, L=64, poly="newton", mu=0.2),
    "cfg2": dict(nrep=2, grid=(48, 48, 48), nsto=128, L=256, poly="cheby", mu=None),
    "cfg3": dict(nrep=4, grid=(96, 96, 96), nsto=512, L=512, poly="cheby", mu=None),
}
# Batched uneven systems: supercells of 1..3 conventional cells per axis
# (8..216 atoms), uniform +-2 % strain per axis, N(0, 0.05 bohr) displacements,
# grid 24 per cell and axis (24..72), 16..256 orbitals, order 128..512.
BATCH = dict(nsys=32, seed=4, strain=0.02, disp=0.05, nsto=(16, 256), L=(128, 512))
BETA = 1000.0          # 1/Ha
ELEC_PER_8 = 32.0      # electrons per 8 Si atoms (4 e/atom)
OCC = 2.0              # spin-unpolarised occupation


def _reps(nrep):
    return (int(nrep),) * 3 if np.isscalar(nrep) else tuple(int(x) for x in nrep)


def diamond_positions(nrep, a0=A0_SI):
    """Fractional coordinates of an n1 x n2 x n3 (or n^3) diamond supercell."""
    r = _reps(nrep)
    base = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0]], dtype=np.float64)
    basis = np.concatenate([base, base + 0.25])
    cells = np.array([[i, j, k] for i in range(r[0]) for j in range(r[1]) for k in range(r[2])], dtype=np.float64)
    frac = (cells[:, None, :] + basis[None, :, :]).reshape(-1, 3) / np.array(r, dtype=np.float64)
    return frac


def make_system(nrep=1, grid=(24, 24, 24), a0=A0_SI, strain=(0.0, 0.0, 0.0), disp_sigma=0.0, seed=0,
                ecut=ECUT_HA, with_kb=True, gvec=None):
    """Orthorhombic Si supercell (nrep: n or (n1, n2, n3) conventional cells).
    Returns a dict with the cell, G sphere, V_KS (filter layout), KB
    description and electron count.

    gvec(hmat, ecut, kmax) -> (ka, kb, kc, ibreak1, ibreak2) lists the half
    G sphere in PINY order; the default is the library's setkvec3d_sm.  This
    module needs nothing else from the package, so a caller that must not
    load the library (the reference's CPU arm of the benchmark) can load it
    on its own and pass its own G-vector routine."""
    if gvec is None:
        from . import setkvec3d_sm as gvec  # noqa: PLC0415  (package-relative)
    rng = np.random.default_rng(seed)
    r = _reps(nrep)
    L = np.array([a0 * r[i] * (1.0 + strain[i]) for i in range(3)])
    hmat = np.diag(L)
    frac = diamond_positions(nrep, a0)
    pos = frac * L
    if disp_sigma > 0:
        pos = pos + rng.normal(0.0, disp_sigma, size=pos.shape)
    n1, n2, n3 = grid
    kmax = [int(math.ceil(math.sqrt(2 * ecut) * Li / (2 * math.pi))) + 1 for Li in L]
    ka, kb, kc, ib1, ib2 = gvec(hmat, ecut, kmax)
    v = local_potential(pos, L, grid)
    kbd = kb_projectors(pos, ecut, L) if with_kb else None
    return dict(hmat=hmat, L=L, pos=pos, natm=len(pos), grid=tuple(grid), ka=ka, kb=kb, kc=kc, ib1=ib1, ib2=ib2,
                vks=v, kb_desc=kbd, num_elec=ELEC_PER_8 * len(pos) / 8.0, ncoef=len(ka))


def local_potential(pos, L, grid):
    """V(r) in the filter layout (ia*n2 + ib)*n3 + ic; separable periodic Gaussians."""
    n1, n2, n3 = grid
    s2 = 2.0 * SIGMA_LOC ** 2

    def axis(n, Lx, X):
        x = np.arange(n) * (Lx / n)
        d = x[None, :] - X[:, None]
        d -= Lx * np.round(d / Lx)
        g = np.zeros_like(d)
        for img in (-2, -1, 0, 1, 2):
            g += np.exp(-((d + img * Lx) ** 2) / s2)
        return g

    gx, gy, gz = axis(n1, L[0], pos[:, 0]), axis(n2, L[1], pos[:, 1]), axis(n3, L[2], pos[:, 2])
    v = V0_LOC * np.einsum("ai,aj,ak->ijk", gx, gy, gz, optimize=True)
    return np.ascontiguousarray(v.reshape(-1))


def _ff(l, g):
    """form factor f and its first three derivatives at g (arrays)."""
    a = RC_KB ** 2 / 2.0
    e = np.exp(-a * g * g)
    if l == 0:
        n0 = math.sqrt(4.0 / (math.sqrt(math.pi) * RC_KB ** 3))
        A = 4.0 * math.pi * n0 * math.sqrt(math.pi / 2.0) * RC_KB ** 3
        f = A * e
        f1 = A * (-2 * a * g) * e
        f2 = A * (4 * a * a * g * g - 2 * a) * e
        f3 = A * (-8 * a ** 3 * g ** 3 + 12 * a * a * g) * e
    else:
        n1 = math.sqrt(8.0 / (3.0 * math.sqrt(math.pi) * RC_KB ** 5))
        B = 4.0 * math.pi * n1 * math.sqrt(math.pi / 2.0) * RC_KB ** 5
        f = B * g * e
        f1 = B * (1 - 2 * a * g * g) * e
        f2 = B * (-6 * a * g + 4 * a * a * g ** 3) * e
        f3 = B * (-6 * a + 24 * a * a * g * g - 8 * a ** 3 * g ** 4) * e
    return f, f1, f2, f3


def local_table(ecut=ECUT_HA, nsplin=4096):
    """The local potential of local_potential() in G space, as the reference
    tabulates a local channel: v(g) = V0 (2 pi sigma^2)^(3/2) exp(-g^2
    sigma^2 / 2), the Fourier transform of one atom's Gaussian, on knots
    gmin + k dg up to past the density cutoff (|G| <= 2 sqrt(2 Ecut)), as
    per-knot Taylor coefficients (f and its first three derivatives over
    0!, 1!, 2!, 3!).  Returns (table [4][nsplin], gmin, dg, v(0)) for
    sdft_vks_set_local."""
    gmax = 2.0 * math.sqrt(2.0 * ecut) * 1.05 + 0.5
    dg = gmax / (nsplin - 1)
    g = np.arange(nsplin) * dg
    s2 = SIGMA_LOC ** 2
    A = V0_LOC * (2.0 * math.pi * s2) ** 1.5
    e = np.exp(-0.5 * s2 * g * g)
    f = A * e
    f1 = A * (-s2 * g) * e
    f2 = A * (s2 * s2 * g * g - s2) * e
    f3 = A * (-(s2 ** 3) * g ** 3 + 3.0 * s2 * s2 * g) * e
    return np.stack([f, f1, f2 / 2.0, f3 / 6.0]), 0.0, dg, A


def density_grid(L, ecut=ECUT_HA):
    """Per axis, the smallest 2^a 3^b edge that holds the density sphere
    0.5 |G|^2 <= 4 Ecut of an orthorhombic cell of edges L (2 kmax + 1
    points, kmax = the sphere's largest |k| on that axis)."""
    def ok(n):
        while n % 2 == 0:
            n //= 2
        while n % 3 == 0:
            n //= 3
        return n == 1
    out = []
    for Li in L:
        kmax = int(math.floor(2.0 * math.sqrt(2.0 * ecut) * Li / (2.0 * math.pi)))
        n = 2 * kmax + 1
        while not ok(n):
            n += 1
        out.append(n)
    return tuple(out)


def kb_projectors(pos, ecut, L, nsplin=2048):
    gmax = math.sqrt(2 * ecut) * 1.05 + 0.5
    dg = gmax / (nsplin - 1)
    g = np.arange(nsplin) * dg
    vps = np.zeros((1, 2, 4, nsplin))
    for l in (0, 1):
        f, f1, f2, f3 = _ff(l, g)
        vps[0, l] = np.stack([f, f1, f2 / 2.0, f3 / 6.0])
    return dict(natm=len(pos), pos=np.ascontiguousarray(pos, dtype=np.float64), type=np.zeros(len(pos), np.int32),
                ntype=1, lmax=1, lmax_type=np.array([1], np.int32), nsplin_g=nsplin, gmin_spl=0.0, dg_spl=dg,
                vps=vps.reshape(-1), vpsnorm=np.array(EKB, dtype=np.float64),
                gzvps0=np.array([_ff(0, np.zeros(1))[0][0]], dtype=np.float64))


def half_dot(ncoef, ar, ai, br, bi):
    """<a|b> over the half sphere: 2 sum (re re + im im) - re(G0) re(G0)."""
    return 2.0 * (np.dot(ar, br) + np.dot(ai, bi)) - ar[ncoef - 1] * br[ncoef - 1]


def lanczos_bounds(hpsi, ncoef, nstep=20, seed=15, margin=0.1):
    """Spectral bounds from `nstep` Lanczos steps on one random real orbital.

    hpsi(cr, ci) -> raw PINY force (f = -4 H c for G != 0, -2 H c at G = 0).
    Returns (Emin - margin, Emax + margin) like calc-spectral-range.c's +-0.1."""
    rng = np.random.default_rng(seed)
    cr = rng.standard_normal(ncoef)
    ci = rng.standard_normal(ncoef)
    ci[-1] = 0.0
    nrm = math.sqrt(half_dot(ncoef, cr, ci, cr, ci))
    cr /= nrm
    ci /= nrm
    alphas, betas = [], []
    pr = np.zeros(ncoef); pi = np.zeros(ncoef)
    beta = 0.0
    for _ in range(nstep):
        fr, fi = hpsi(cr, ci)
        hr = -0.25 * fr; hi = -0.25 * fi
        hr[-1] = -0.5 * fr[-1]; hi[-1] = 0.0
        alpha = half_dot(ncoef, cr, ci, hr, hi)
        wr = hr - alpha * cr - beta * pr
        wi = hi - alpha * ci - beta * pi
        alphas.append(alpha)
        beta = math.sqrt(max(half_dot(ncoef, wr, wi, wr, wi), 0.0))
        betas.append(beta)
        if beta < 1e-12:
            break
        pr, pi = cr, ci
        cr, ci = wr / beta, wi / beta
    k = len(alphas)
    T = np.diag(alphas) + np.diag(betas[:k - 1], 1) + np.diag(betas[:k - 1], -1)
    ev = np.linalg.eigvalsh(T)
    return float(ev[0] - margin), float(ev[-1] + margin)


def batch_specs(nsys=BATCH["nsys"], seed=BATCH["seed"], big_fraction=0.0, big_nsto=256, big_L=512):
    """Seeded specs of uneven systems: dicts with nrep (per axis), grid,
    strain, disp_seed, nsto (even), L (even).  The supercell shape is drawn
    uniformly from the 27 shapes with 1..3 cells per axis (8..216 atoms).
    With big_fraction > 0 that fraction of specs is the 512-atom 4x4x4 cell
    on the 96^3 grid with big_nsto orbitals and order big_L."""
    rng = np.random.default_rng(seed)
    shapes = [(a, b, c) for a in (1, 2, 3) for b in (1, 2, 3) for c in (1, 2, 3)]
    out = []
    for i in range(nsys):
        if big_fraction > 0 and rng.random() < big_fraction:
            rep = (4, 4, 4)
            nsto, L = big_nsto, big_L
        else:
            rep = shapes[int(rng.integers(len(shapes)))]
            nsto = 2 * int(rng.integers(BATCH["nsto"][0] // 2, BATCH["nsto"][1] // 2 + 1))
            L = 2 * int(rng.integers(BATCH["L"][0] // 2, BATCH["L"][1] // 2 + 1))
        strain = tuple(float(x) for x in rng.uniform(-BATCH["strain"], BATCH["strain"], size=3))
        out.append(dict(nrep=rep, grid=tuple(24 * r for r in rep), strain=strain, disp_seed=int(rng.integers(1 << 30)),
                        nsto=nsto, L=L))
    return out


def build_spec(spec):
    """The system of one batch spec."""
    return make_system(spec["nrep"], spec["grid"], strain=spec["strain"], disp_sigma=BATCH["disp"],
                       seed=spec["disp_seed"])
