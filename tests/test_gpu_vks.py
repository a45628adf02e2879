"""The density side of the SCF step on the GPU (sdft_vks_*): the local
pseudopotential on the density sphere, the density in G space, the Hartree
and local parts of V_KS with PZ81 exchange-correlation, against the numpy
restatement (oracle/vks.py), which tests/test_oracle_pin.py pins to the
reference's own controlEwdLocPreScf / calcRhoStoRecipFullg / cpGetVksStodft.

Grids hold the density sphere (0.5 |G|^2 <= 4 Ecut): 32^3 for the 8-atom
cell, 128^3 for the 512-atom cell.  Tolerances: vext and rho(G) 1e-13,
V_KS and the energies 1e-12 (relative)."""
import numpy as np
import pytest

from conftest import rel_l2
from oracle import oracle as O
from oracle import vks as V

pytestmark = pytest.mark.gpu


def _grid_for(pkg, wl, s):
    ka, kb, kc, _, _ = pkg.setkvec3d_sm(s["hmat"], 4 * wl.ECUT_HA, list(s["grid"]))
    g = pkg.DensityGrid(*s["grid"], s["hmat"], ka, kb, kc)
    vtab, gmin, dg, gz = wl.local_table()
    g.set_local(s["pos"], vtab, gmin, dg, gz)
    return g, (ka, kb, kc), (vtab, gmin, dg, gz)


def _check(pkg, wl, s, rho_in):
    g, (ka, kb, kc), (vtab, gmin, dg, gz) = _grid_for(pkg, wl, s)
    try:
        vre, vim = V.vext(s["hmat"], ka, kb, kc, s["pos"], vtab, vtab.shape[1], gmin, dg, gz)
        gre, gim = g.vext()
        assert rel_l2(gre, vre) < 1e-13 and rel_l2(gim, vim) < 1e-13
        v, rre, rim, e = g.vks_from_rho(rho_in, pkg.SDFT_XC_PZ_LDA)
        ov, orr, ori, oe = V.vks_from_rho(s["grid"], s["hmat"], ka, kb, kc, vre, vim, rho_in)
        assert rel_l2(rre, orr) < 1e-13 and rel_l2(rim, ori) < 1e-13
        assert rel_l2(v, ov) < 1e-12
        assert np.all(np.abs(e - oe) <= 1e-12 * np.abs(oe))
        # without xc: the Hartree and local parts alone
        v2, _, _, e2 = g.vks_from_rho(rho_in, 0)
        ov2, _, _, oe2 = V.vks_from_rho(s["grid"], s["hmat"], ka, kb, kc, vre, vim, rho_in, xc=False)
        assert rel_l2(v2, ov2) < 1e-12 and e2[2] == 0.0
    finally:
        g.close()


def test_vks_8_atoms_32(pkg, wl):
    s = wl.make_system(1, (32, 32, 32))
    o = O.OracleSys(s)
    cr, ci = o.noise(4, 10.0)
    rho = o.density(cr, ci)
    _check(pkg, wl, s, rho * (s["num_elec"] / rho.mean()))


def test_vks_512_atoms_128(pkg, wl):
    """The 512-atom cell on the grid of its density sphere (128-point lines)."""
    s = wl.make_system(4, (128, 128, 128), with_kb=False)
    rng = np.random.default_rng(3)
    rho = 1.0 + 0.5 * rng.random(128 ** 3)
    _check(pkg, wl, s, rho * (s["num_elec"] / rho.mean()))


def test_scf_step_on_device(pkg, wl):
    """One device-resident step: noise -> filter -> density (device buffer)
    -> V_KS from it (device in, device out) -> the next H.psi on the new
    potential, against the oracle given the same density."""
    import torch
    s = wl.make_system(1, (32, 32, 32))
    nsto, L = 8, 24
    c = pkg.Context(*s["grid"], s["ka"], s["kb"], s["kc"], s["hmat"], max_states=nsto)
    g, (ka, kb, kc), (vtab, gmin, dg, gz) = _grid_for(pkg, wl, s)
    try:
        c.set_vks(s["vks"])
        c.set_kb(s["kb_desc"])
        emin, emax = -1.0, 45.0
        scale, em = 2.0 / (emax - emin), 0.5 * (emin + emax)
        ec = pkg.calcChebyCoeff(L, emax - emin, em, wl.BETA, 0.2)
        c.noise_dev(nsto, seed=10.0)
        c.filter_cheby_dev(nsto, ec, 1, scale, em)
        dev = torch.device("cuda", 0)
        rho_d = torch.empty(int(np.prod(s["grid"])), dtype=torch.float64, device=dev)
        v_d = torch.empty_like(rho_d)
        c.density_dev(nsto, 0, wl.OCC / nsto, out_ptr=rho_d.data_ptr())
        _, _, _, e = g.vks_from_rho(rho_d.data_ptr(), pkg.SDFT_XC_PZ_LDA, out_ptr=v_d.data_ptr())
        rho = rho_d.cpu().numpy()
        vre, vim = V.vext(s["hmat"], ka, kb, kc, s["pos"], vtab, vtab.shape[1], gmin, dg, gz)
        ov, _, _, oe = V.vks_from_rho(s["grid"], s["hmat"], ka, kb, kc, vre, vim, rho)
        v = v_d.cpu().numpy()
        assert rel_l2(v, ov) < 1e-12
        assert np.all(np.abs(e - oe) <= 1e-12 * np.abs(oe))
        c.set_vks_dev_ptr(v_d.data_ptr())  # V_KS straight from the device buffer
        s2 = dict(s, vks=v)
        cr, ci = O.OracleSys(s).noise(3, seed=4.0)
        fr, fi = c.calc_coef_force(cr, ci)
        orr, oi = O.OracleSys(s2).hpsi(cr, ci)
        assert rel_l2(np.concatenate([fr, fi]), np.concatenate([orr, oi])) < 1e-12
    finally:
        g.close()
        c.close()


@pytest.mark.parametrize("nrep,grid,q_pseud", [(1, (32, 32, 32), 4.0), (1, (32, 32, 32), 3.5),
                                               (4, (128, 128, 128), 4.0)])
def test_local_forces(pkg, wl, nrep, grid, q_pseud):
    """Local-pseudopotential + Ewald reciprocal forces and the Ewald energies
    (calcLocExtPostScf / ewald3d_selfbgr_cp) on displaced atoms, against the
    numpy restatement (pinned to the reference's control_ewd_loc), relative
    to the largest force component: 1e-12."""
    s = wl.make_system(nrep, grid, disp_sigma=0.05, seed=2, with_kb=nrep == 1)
    if nrep == 1:
        o = O.OracleSys(s)
        cr, ci = o.noise(4, 10.0)
        rho = o.density(cr, ci)
    else:
        rho = 1.0 + 0.5 * np.random.default_rng(5).random(int(np.prod(grid)))
    rho_in = rho * (s["num_elec"] / rho.mean())
    q = np.full(s["natm"], 4.0)
    g, (ka, kb, kc), (vtab, gmin, dg, gz) = _grid_for(pkg, wl, s)
    try:
        g.vks_from_rho(rho_in, pkg.SDFT_XC_PZ_LDA)
        F, e = g.local_forces(q, [q_pseud], 1.2)
    finally:
        g.close()
    vre, vim = V.vext(s["hmat"], ka, kb, kc, s["pos"], vtab, vtab.shape[1], gmin, dg, gz)
    _, rre, rim, _ = V.vks_from_rho(s["grid"], s["hmat"], ka, kb, kc, vre, vim, rho_in)
    oF, oe = V.local_forces(s["hmat"], ka, kb, kc, s["pos"], q, q_pseud, vtab, vtab.shape[1], gmin, dg, rre, rim, 1.2)
    assert np.abs(F - oF).max() < 1e-12 * np.abs(oF).max()
    assert np.all(np.abs(e - oe) <= 1e-12 * np.abs(oe))


@pytest.mark.parametrize("nrep,grid,ishift", [(1, (32, 32, 32), 0), (1, (32, 32, 32), 2), (4, (96, 96, 96), 1)])
def test_ewald_real_device(pkg, wl, nrep, grid, ishift):
    """The device real-space ion-ion Ewald sum against the numpy restatement
    (pinned to the reference's vcoul_bin table): 8 atoms with a cutoff past
    the cell (many images) and 512 atoms; forces and energy at 1e-12.  With
    the device's reciprocal, self and background terms from
    sdft_vks_local_forces, the full Ewald energy does not depend on the
    splitting parameter (8 atoms, alp 0.4 and 0.5: the real-space part moves
    by 0.6 hartree)."""
    s = wl.make_system(nrep, grid, disp_sigma=0.05, seed=2, with_kb=False)
    q = np.full(s["natm"], 4.0)
    rmax = 20.0 if nrep == 1 else 12.0
    alp = 0.4 if nrep == 1 else 0.6
    F, E = pkg.ewald_real(s["hmat"], s["pos"], q, alp, rmax, ishift, 2.0)
    Fo, Eo = V.ewald_real(s["hmat"], s["pos"], q, alp, rmax, ishift, 2.0)
    assert np.abs(F - Fo).max() <= 1e-12 * np.abs(Fo).max()
    assert abs(E - Eo) <= 1e-12 * abs(Eo)
    if nrep != 1 or ishift != 0:
        return
    rho_in = np.full(int(np.prod(grid)), s["num_elec"] / np.prod(grid))
    tot, real = [], []
    for a in (0.4, 0.5):
        g = _grid_for(pkg, wl, s)[0]
        try:
            g.vks_from_rho(rho_in, pkg.SDFT_XC_PZ_LDA)
            _, ew = g.local_forces(q, [4.0], a)
        finally:
            g.close()
        real.append(pkg.ewald_real(s["hmat"], s["pos"], q, a, 20.0)[1])
        tot.append(real[-1] + ew.sum())
    assert real[0] - real[1] > 0.5
    assert abs(tot[0] - tot[1]) < 1e-9 * abs(tot[1])
