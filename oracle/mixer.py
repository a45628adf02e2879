"""Density mixing and checkpoint files, restated in numpy.  TEST
INFRASTRUCTURE ONLY (the oracle of the device mixer).

Follows genDensityMix / updateBank / updateErr / calcDensityDiis /
matrixInvSVD (stodft/diis.c:34-464) and checkpointOutput / checkpointInput
(stodft/checkpointIO.c:32-533), spin-unpolarised, one rank:

- bank: the last num_diis + 1 corrected densities (newest first);
  err: the last num_diis differences rho_correct - rho_old;
- iscf == 0: bank the density, rho_old = rho_correct (the output density is
  left as it was);
- 1 <= iscf <= num_step_mix: rho = rho_correct (1 - r) + bank[0] r with
  r = mix_ratio_big (bank[0] is rho_correct itself after the banking, as in
  the reference);
- iscf > num_step_mix: DIIS.  B_ij = <err_i|err_j> for i, j < n = min(iscf,
  num_diis); the bordered matrix [[B, -m], [-m^T, 0]] with m = max |B_ij|
  and right side (0, ..., 0, -m) is solved by an SVD pseudo-inverse
  (singular values below 1e-10 of the largest dropped); the density is
  sum_i c_i (bank_i + (alpha - 1) err_i), alpha = mix_ratio_sm for
  iscf <= 10, else mix_ratio_sm2;
- rho_old = the output density.
"""
from __future__ import annotations

import numpy as np


class DensityMixer:
    def __init__(self, n, num_diis, num_step_mix, mix_ratio_big, mix_ratio_sm, mix_ratio_sm2):
        self.n, self.num_diis, self.num_step_mix = int(n), int(num_diis), int(num_step_mix)
        self.r_big, self.r_sm, self.r_sm2 = float(mix_ratio_big), float(mix_ratio_sm), float(mix_ratio_sm2)
        self.bank = [None] * (self.num_diis + 1)
        self.err = [None] * self.num_diis
        self.old = np.zeros(self.n)
        self.rho = np.zeros(self.n)
        self.num_diis_now = 0
        self.iscf = 0
        self.coef = None

    def _bank(self, rho):  # updateBank (stodft/diis.c:134)
        self.bank = [np.array(rho, dtype=np.float64)] + self.bank[:self.num_diis]

    def _err(self, rho):  # updateErr (stodft/diis.c:161)
        self.err = [np.asarray(rho, dtype=np.float64) - self.old] + self.err[:self.num_diis - 1]

    @staticmethod
    def svd_solve(a, b):  # matrixInvSVD (stodft/diis.c:383)
        u, s, vt = np.linalg.svd(a)
        sinv = np.where(s / s.max() > 1e-10, 1.0 / np.where(s > 0, s, 1.0), 0.0)
        return vt.T @ (sinv * (u.T @ b))

    def step(self, iscf, rho_correct):
        rho_correct = np.asarray(rho_correct, dtype=np.float64)
        n = min(iscf, self.num_diis)
        self.num_diis_now = n
        self.iscf = iscf
        if iscf == 0:
            self._bank(rho_correct)
            self.old = rho_correct.copy()
        elif iscf <= self.num_step_mix:
            self._err(rho_correct)
            self._bank(rho_correct)
            self.rho = rho_correct * (1.0 - self.r_big) + self.bank[0] * self.r_big
            self.old = self.rho.copy()
        else:
            self._err(rho_correct)
            self._bank(rho_correct)
            B = np.array([[float(np.dot(self.err[i], self.err[j])) for j in range(n)] for i in range(n)])
            m = max(abs(B[i, j]) for i in range(n) for j in range(i, n))
            A = np.zeros((n + 1, n + 1))
            A[:n, :n] = B
            A[n, :n] = -m
            A[:n, n] = -m
            b = np.zeros(n + 1)
            b[n] = -m
            x = self.svd_solve(A, b)
            self.coef = x[:n]
            pre = (self.r_sm if iscf <= 10 else self.r_sm2) - 1.0
            out = np.zeros(self.n)
            for i in range(n):
                out += x[i] * (self.bank[i] + pre * self.err[i])
            self.rho = out
            self.old = self.rho.copy()
        return self.rho.copy()

    def checkpoint_text(self, rho, vol):
        """The density-checkpoint file checkpointOutput writes for rho_up =
        rho: "iscf num_diis_now", rho * vol, the banks and the errors, one
        "%.16lg" value per line."""
        nout = self.num_diis_now + 1 if self.num_diis_now < self.num_diis else self.num_diis_now
        lines = [f"{self.iscf} {self.num_diis_now}"]
        lines += ["%.16g" % v for v in np.asarray(rho, dtype=np.float64) * vol]
        for i in range(nout):
            lines += ["%.16g" % v for v in self.bank[i]]
        for i in range(self.num_diis_now):
            lines += ["%.16g" % v for v in self.err[i]]
        return "\n".join(lines) + "\n"
