"""Autotuner for the per-system launch shapes of the filter.

Three shapes are tuned per problem shape:
* the orbital columns per tile of the mixed-precision KB GEMMs, 128 or 64:
  the orbital count is padded to the tile width, so 64 wastes less on small
  or just-over-128 counts, while 128 reads each projector tile fewer times
  (timed first, at the cost model's split);
* the split-K factor of the nonlocal projection GEMM (Z = Pj C: M =
  projectors, N = orbitals, K = 2 ncoef): few-orbital, small systems have
  only a handful of output tiles, so the K range per CTA decides how many of
  the 148 SMs work.  The built-in wave-quantisation cost model (choice 0) is
  one candidate; fixed splits are the others;
* the CTA size of the FP32 plane FFT stage (one CTA per plane and orbital
  pair): 256 threads, or 128, which fits twice the CTAs per SM and can be
  faster on small planes (mixed contexts on the fast FFT path).
Each candidate is timed (best of two) on a short Chebyshev filter of the
context's resident orbitals: the filter kernels themselves, device time by
CUDA events on the context stream, through the library's own event calls.
The library's own choice (0) is a candidate in each list, and another is set
only when it is more than 2 % faster, so timing noise cannot pick a slower
shape.  Results are cached per problem shape (grid, projectors, orbital
tiles of 64, precision), in memory and optionally in a JSON file.

Tuning overwrites the context's filter accumulators: run it before the real
filter.
"""
from __future__ import annotations

import json
import os

import numpy as np

CANDIDATES = (0, 1, 2, 4, 8, 16, 32)
# 0 first in each list: the library's own choice (the split cost model, the
# per-call tile width, the default CTA size), which another candidate must
# beat by more than MARGIN to be taken, so timing noise cannot pick a worse one
PLANE_THREADS = (0, 256, 128)
GEMM_BN = (0, 128, 64)
MARGIN = 0.02


def _pick(times):
    """The candidate to set: the fastest, unless the library's choice ("0")
    is within MARGIN of it."""
    best = min(times, key=times.get)
    if "0" in times and times["0"] <= times[best] * (1.0 + MARGIN):
        return 0
    return int(best)


class Tuner:
    def __init__(self, pkg, path=None, steps=6, candidates=CANDIDATES):
        self.pkg = pkg
        self.path = path
        self.steps = int(steps)
        self.candidates = tuple(candidates)
        self.cache = {}
        if path and os.path.exists(path):
            with open(path) as f:
                self.cache = json.load(f)

    @staticmethod
    def key(ctx, nstate, nproj):
        # the GEMM tile grid depends on the projector count and the orbitals
        # in 64-wide tiles; K (2 ncoef) follows from the grid
        return f"{ctx.n[0]}x{ctx.n[1]}x{ctx.n[2]}/P{nproj}/N{(nstate + 63) // 64}/prec{ctx.precision}"

    def _time(self, ctx, nstate, split, scale, emean, reps=2):
        """Device time of a short filter under split-K `split`: the best of
        `reps` runs after a warm-up run."""
        ctx.set_gemm_split(split)
        ec = np.full(self.steps + 1, 1.0 / (self.steps + 1))
        ctx.filter_cheby_dev(nstate, ec, 1, scale, emean)  # warm (buffers, caches)
        a, b = self.pkg.Event(ctx.device), self.pkg.Event(ctx.device)
        try:
            best = float("inf")
            for _ in range(reps):
                a.record(ctx.stream_ptr)
                ctx.filter_cheby_dev(nstate, ec, 1, scale, emean)
                b.record(ctx.stream_ptr)
                ctx.sync()
                best = min(best, a.elapsed_ms(b))
            return best
        finally:
            a.close()
            b.close()

    def tune(self, ctx, nstate, nproj, scale=0.1, emean=0.0):
        """Pick and set the KB GEMM tile width, the projection split-K and
        the plane-stage CTA size for (ctx, nstate); returns the split."""
        k = self.key(ctx, nstate, nproj)
        if k not in self.cache:
            bn = {}
            if ctx.precision != self.pkg.SDFT_PREC_FP64:  # the FP64 GEMM has one tile shape
                for w in GEMM_BN:
                    ctx.set_gemm_bn(w)
                    bn[str(w)] = self._time(ctx, nstate, 0, scale, emean)
                ctx.set_gemm_bn(_pick(bn))
            times = {str(c): self._time(ctx, nstate, c, scale, emean) for c in self.candidates}
            best = _pick(times)
            entry = {"split": best, "ms": times}
            if bn:
                entry["gemm_bn"] = _pick(bn)
                entry["gemm_bn_ms"] = bn
            plane = {}
            for nt in PLANE_THREADS:
                try:
                    ctx.set_plane_threads(nt)
                except self.pkg.SdftError:  # FP64 or the generic FFT path: one plane shape only
                    continue
                plane[str(nt)] = self._time(ctx, nstate, best, scale, emean)
            if len(plane) > 1:
                entry["plane_threads"] = _pick(plane)
                entry["plane_ms"] = plane
            self.cache[k] = entry
            if self.path:
                with open(self.path, "w") as f:
                    json.dump(self.cache, f, indent=1, sort_keys=True)
        entry = self.cache[k]
        split = int(entry["split"])
        ctx.set_gemm_split(split)
        if "gemm_bn" in entry:
            ctx.set_gemm_bn(int(entry["gemm_bn"]))
        try:
            ctx.set_plane_threads(int(entry.get("plane_threads", 0)))
        except self.pkg.SdftError:  # one plane shape only (FP64, generic FFT path)
            pass
        return split
