"""State-parallel host logic (states.py) with world_size 2 over gloo on CPU.

Each rank draws its own noise (np_states = 2, myid = rank), takes moments
and the stochastic density of its orbitals with the CPU oracle, and sums
them over the ranks with StateGroup; rank 0 checks the sums, the chemical
potential and the KB atomic forces (each rank's orbitals, summed as
calcEnergyForce reduces them over comm_states) against a single-process run
over both ranks' orbitals.
"""
import os
import socket

import numpy as np
import pytest

from conftest import ROOT

L, NLOC = 12, 3
EMIN, EMAX = -1.0, 45.0


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out_path):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import __graft_entry__ as g
        from oracle import oracle as O
        pkg = g.load_package()
        wl = g.load_workload()
        states = __import__(pkg.__name__ + ".states", fromlist=["StateGroup"])
        s = wl.make_system(1, (24, 24, 24))
        o = O.OracleSys(s)
        grp = states.StateGroup(dist)
        n = states.local_count(2 * NLOC, world, rank)
        cr, ci = o.noise(n, 10.0, np_states=world, myid=rank)
        scale, em = 2.0 / (EMAX - EMIN), 0.5 * (EMAX + EMIN)
        mom = o.moments(cr, ci, L, scale, em)
        mu, ne = grp.chem_pot(pkg, mom, 2 * NLOC, L, EMAX - EMIN, em, wl.BETA, wl.OCC, s["num_elec"], 0.2, 0.05)
        rho = grp.sum_array(o.density(cr, ci))
        fa, _ = o.nl_force(cr, ci)
        fa = grp.sum_array(fa * wl.OCC / (2 * NLOC))
        if rank == 0:
            np.savez(out_path, mom=grp.sum_array(mom), mu=mu, ne=ne, rho=rho, force=fa)
        else:
            grp.sum_array(mom)
    finally:
        dist.destroy_process_group()


def test_two_state_ranks_match_one_process(tmp_path, pkg, wl):
    import torch.multiprocessing as mp
    out = str(tmp_path / "r0.npz")
    mp.start_processes(_rank_main, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    from oracle import oracle as O
    s = wl.make_system(1, (24, 24, 24))
    o = O.OracleSys(s)
    scale, em = 2.0 / (EMAX - EMIN), 0.5 * (EMAX + EMIN)
    mom = np.zeros(L + 1)
    rho = np.zeros(int(np.prod(s["grid"])))
    crs, cis = [], []
    for r in range(2):
        cr, ci = o.noise(NLOC, 10.0, np_states=2, myid=r)
        mom += o.moments(cr, ci, L, scale, em)
        rho += o.density(cr, ci)
        crs.append(cr)
        cis.append(ci)
    force = o.nl_force(np.concatenate(crs), np.concatenate(cis))[0] * wl.OCC / (2 * NLOC)
    assert np.abs(got["force"] - force).max() < 1e-13 * np.abs(force).max()
    mu, ne = pkg.calcChemPotCheby(L, EMAX - EMIN, em, wl.BETA, wl.OCC, mom / (2 * NLOC), s["num_elec"], 0.2, 0.05)
    assert np.allclose(got["mom"], mom, rtol=1e-13, atol=0)
    assert np.allclose(got["rho"], rho, rtol=1e-13, atol=1e-13 * np.abs(rho).max())
    assert abs(float(got["mu"]) - mu) < 1e-10 and abs(float(got["ne"]) - ne) < 1e-8


def test_local_count(pkg):
    states = __import__(pkg.__name__ + ".states", fromlist=["local_count"])
    assert [states.local_count(10, 4, r) for r in range(4)] == [3, 3, 2, 2]
    with pytest.raises(ValueError):
        states.local_count(1, 2, 0)
