"""State-parallel decomposition of the filter (the reference's comm_states).

Stochastic orbitals are independent, so ranks split them and never exchange
orbital data.  The reference's exchanges, reproduced here over
torch.distributed (NCCL between GPUs, gloo on CPU):

* each rank draws its own noise with np_states = world size and
  myid = rank (gen-noise.c:229-239 derives every rank's seed on rank 0 and
  broadcasts them);
* the Chebyshev moments are summed over ranks before the chemical-potential
  bisection, which normalises by the total orbital count
  (calc-chempot-chebyshev.c:144 reduces chebyMomentsUp to rank 0; here every
  rank receives the sum and runs the same deterministic bisection);
* the stochastic density of every rank's orbitals is summed over ranks
  (density.c:1444 reduces rhoUpChemPot to rank 0; here every rank receives
  it).

All ranks must call these helpers in the same order.
"""
from __future__ import annotations

import numpy as np


def local_count(nsto_total: int, world: int, rank: int) -> int:
    """Orbitals of `rank` when nsto_total orbitals are split as evenly as
    possible (the first nsto_total % world ranks take one more)."""
    if world < 1 or not 0 <= rank < world or nsto_total < world:
        raise ValueError("local_count: need 0 <= rank < world <= nsto_total")
    base, extra = divmod(nsto_total, world)
    return base + (1 if rank < extra else 0)


class StateGroup:
    """Sums over the state ranks of a torch.distributed process group
    (None = single rank, every sum is the identity)."""

    def __init__(self, dist=None, group=None, device=None):
        self.dist = dist
        self.group = group
        self.device = device
        self.world = dist.get_world_size(group) if dist else 1
        self.rank = dist.get_rank(group) if dist else 0

    def sum_tensor_(self, t):
        """In-place sum of a torch tensor over the ranks."""
        if self.dist:
            self.dist.all_reduce(t, group=self.group)
        return t

    def sum_array(self, a):
        """Sum of a numpy array over the ranks (returns a new float64 array)."""
        a = np.ascontiguousarray(a, dtype=np.float64)
        if not self.dist:
            return a.copy()
        import torch
        t = torch.from_numpy(a.copy())
        if self.device is not None:
            t = t.to(self.device)
        self.dist.all_reduce(t, group=self.group)
        return t.cpu().numpy()

    def chem_pot(self, pkg, moments_local, nsto_total, L, energy_diff, energy_mean, beta, occ, num_elec,
                 chem_pot_init, gap_init):
        """calcChemPotCheby on the moments of all ranks' orbitals."""
        mom = self.sum_array(moments_local) / float(nsto_total)
        return pkg.calcChemPotCheby(L, energy_diff, energy_mean, beta, occ, mom, num_elec, chem_pot_init, gap_init)
