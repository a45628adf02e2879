"""Filter + density requests served with continuous batching on one GPU.

A request names a system (a batch spec from workload.batch_specs), its
number of stochastic orbitals, the polynomial order and a noise seed.  For
every request the server

1. waits until a slot is free and its device memory fits in the HBM budget
   (admission); memory is reserved from an estimate and corrected to the
   context's measured footprint once it exists; a request that could not
   fit even on an idle device is refused;
2. prepares it on its own context: V_KS, KB projectors, 20-step Lanczos
   bounds (device resident), noise orbitals generated on the device, Chebyshev moments, mu by
   the FP64 bisection (calcChemPotCheby) and the filter coefficients;
3. issues its Chebyshev filter + density on the request's own stream as a
   captured one-context CUDA graph (sdft_batch; graph=False issues the
   kernels directly, which measured slower: thousands of launches from
   concurrent host threads), so requests admitted while others run overlap
   on the device; the request's streams get a CUDA priority by its work
   (request_priority: cheaper = more urgent), so short requests are not
   queued behind 512-atom ones;
4. when the graph's completion event fires, downloads the density, frees the
   context and returns its memory to the budget.

Requests are independent and every kernel is deterministic, so a request's
result does not depend on what else runs beside it.
"""
from __future__ import annotations

import time
from collections import deque

import numpy as np


def request_priority(grid, nsto, L, levels=6, ref_cost=1e11):
    """CUDA stream priority of a request by its filter work nsto * L * grid
    points: 0 (least urgent) at ref_cost and above, one level more urgent per
    factor 4 less work, down to -(levels - 1) (clamped to the device range by
    the library)."""
    import math
    cost = float(nsto) * L * grid[0] * grid[1] * grid[2]
    return -min(levels - 1, max(0, int(math.log(ref_cost / cost, 4)))) if cost < ref_cost else 0


def prepare(pkg, wl, s, nsto, L, precision, seed, device=0, tuner=None, mu=None, priority=None):
    """Context with resident noise orbitals and filter coefficients for one
    system (steps 2 of the request life cycle).  mu, if given, replaces the
    bisection result (the moments are still computed); priority, if given,
    is the CUDA priority of the context's stream."""
    t = [time.perf_counter()]
    ctx = pkg.Context(*s["grid"], s["ka"], s["kb"], s["kc"], s["hmat"], precision=precision, max_states=nsto,
                      device=device)
    if priority is not None:
        ctx.set_priority(priority)
    ctx.set_vks(s["vks"])
    ctx.set_kb(s["kb_desc"])
    t.append(time.perf_counter())
    emin, emax = ctx.lanczos_bounds(20, seed=15, margin=0.1)[:2]  # device Lanczos, same start vector as the host one
    ediff, emean = emax - emin, 0.5 * (emin + emax)
    scale = 2.0 / ediff
    t.append(time.perf_counter())
    ctx.noise_dev(nsto, seed=seed)
    t.append(time.perf_counter())
    mom = ctx.moments_dev(nsto, L, scale, emean)
    t.append(time.perf_counter())
    mu_b, ne = pkg.calcChemPotCheby(L, ediff, emean, wl.BETA, wl.OCC, mom / nsto, s["num_elec"], 0.2, 0.05)
    mu = mu_b if mu is None else mu
    ec = pkg.calcChebyCoeff(L, ediff, emean, wl.BETA, mu, fun_flag=2)
    if tuner is not None:  # times short filters of the resident noise (accumulators only)
        tuner.tune(ctx, nsto, 4 * s["natm"], scale, emean)
    phases = dict(context_s=t[1] - t[0], lanczos_s=t[2] - t[1], noise_s=t[3] - t[2], moments_s=t[4] - t[3])
    return dict(ctx=ctx, ec=ec, scale=scale, emean=emean, mu=mu, num_elec=ne, occ_over=wl.OCC / nsto, nsto=nsto, L=L,
                phases=phases, priority=priority)


def estimate_spec_bytes(spec, nsto, ecut=10.0, a0=10.26):
    """estimate_bytes before the system is built: G-sphere and sphere-column
    counts from the cell volume and cutoff (x 1.15 margin)."""
    import math
    rep = spec["nrep"]
    Lc = [a0 * rep[i] * (1.0 + spec["strain"][i]) for i in range(3)]
    vol = Lc[0] * Lc[1] * Lc[2]
    gmax = math.sqrt(2.0 * ecut)
    ncoef = int(vol * gmax ** 3 / (6.0 * math.pi ** 2) / 2.0) + 1
    area = Lc[0] * Lc[1]
    cols = int(area * gmax ** 2 / (4.0 * math.pi)) + 1
    natm = 8 * rep[0] * rep[1] * rep[2]
    return int(1.15 * _bytes(spec["grid"], ncoef, cols, natm, nsto))


def _bytes(grid, ncoef, cols, natm, nsto):
    n1, n2, n3 = grid
    spad = (nsto + 127) // 128 * 128
    vec = spad * 2 * ncoef * 8
    npairs = (nsto + 1) // 2
    P = 4 * natm
    ppad = (P + 127) // 128 * 128
    kp = (2 * ncoef + 63) // 64 * 64
    mpad = (2 * ncoef + 127) // 128 * 128
    return int(5 * vec + npairs * n3 * cols * 8 + npairs * n1 * n2 * n3 * 8 + 4 * (ppad * kp + mpad * ppad)
               + 4 * spad * (kp + ppad) + 32 * spad * ppad * 8 + 64 * 2 ** 20)


def estimate_bytes(s, nsto):
    """Device footprint of one request's context (mixed precision), from the
    sizes the library allocates: orbital blocks, FFT column scratch, density
    partials, KB digit arrays and split-K partials."""
    cols = len(set(zip(s["ka"][:-1].tolist(), s["kb"][:-1].tolist()))) * 2 + 1
    return _bytes(s["grid"], s["ncoef"], cols, s["natm"], nsto)


def admission(est, used, budget, busy):
    """Admission decision for the request at the head of the queue:
    'refuse' if its estimated footprint alone exceeds the budget (it could
    never run), 'wait' while it does not fit beside the requests already
    holding memory, else 'admit'.  An idle device admits whatever fits the
    budget on its own."""
    if est > budget:
        return "refuse"
    if used + est > budget and busy:
        return "wait"
    return "admit"


class Server:
    """Continuous-batching loop over a list of timed requests.  Admission and
    completion run on the calling thread; preparation (host set-up, moments,
    capture, launch) runs on a pool of `workers` threads, so the host work of
    new requests overlaps the device work of running ones (the library's calls
    release the interpreter lock).  Device events and the calling threads'
    device come from the library's C ABI; nothing here needs another CUDA
    binding.

    While it runs, the library's device memory on the server's device is
    capped at what it held at the start plus the HBM budget
    (sdft_set_device_memory_limit), so a request whose footprint was
    underestimated fails alone with SDFT_ERR_NOMEM instead of taking memory
    from the others.  Requests whose estimate exceeds the whole budget are
    refused at admission; both outcomes are recorded per request."""

    def __init__(self, pkg, wl, precision, hbm_budget=150e9, slots=16, device=0, tuner=None, workers=4,
                 priorities=True, graph=True):
        self.pkg, self.wl = pkg, wl
        self.priorities = bool(priorities)
        self.graph = bool(graph)
        self.precision = precision
        self.budget = float(hbm_budget)
        self.slots = int(slots)
        self.device = device
        self.tuner = tuner
        self.workers = int(workers)

    def _start(self, i, r, t0):
        pkg = self.pkg
        pkg.set_device(self.device)
        t_adm = time.perf_counter() - t0
        tb = time.perf_counter()
        s = self.wl.build_spec(r["spec"])
        build_s = time.perf_counter() - tb
        prio = request_priority(s["grid"], r["nsto"], r["L"]) if self.priorities else None
        p = prepare(pkg, self.wl, s, r["nsto"], r["L"], self.precision, r["seed"], self.device, self.tuner,
                    mu=r.get("mu"), priority=prio)
        ctx = p["ctx"]
        try:
            tc = time.perf_counter()
            if self.graph:  # one captured graph per request, replayed once
                b = pkg.Batch([ctx], [r["nsto"]], [r["L"]], [p["ec"]], [p["scale"]], [p["emean"]], [p["occ_over"]])
                if prio is not None:
                    b.set_priority(prio)
                st = b.stream_ptr
                b.launch()
            else:  # the same kernels issued directly on the context's stream (no capture / instantiation)
                b = None
                st = ctx.stream_ptr
                ctx.filter_cheby_dev(r["nsto"], p["ec"], 1, p["scale"], p["emean"])
                ctx.density_dev(r["nsto"], 0, p["occ_over"], want=False)
            p["phases"].update(build_s=build_s, launch_s=time.perf_counter() - tc)
            ev = pkg.Event(self.device).record(st)
        except BaseException:
            ctx.close()
            raise
        return dict(i=i, ctx=ctx, batch=b, ev=ev, mem=ctx.device_bytes, t_adm=t_adm, prep=p, natm=s["natm"])

    def run(self, requests, keep_density=True):
        """requests: list of dicts with arrival (s), spec, nsto, L, seed and
        optionally mu.  Returns per-request records and a summary.  A record
        has status 'done' (latency, orbitals, density ...), 'refused' (its
        estimate exceeds the budget) or 'failed' (the library refused it, e.g.
        SDFT_ERR_NOMEM under the cap; error holds the message).  Times are
        seconds from the start of the run: arrivals and admissions on the
        host clock, completions from CUDA events."""
        from concurrent.futures import ThreadPoolExecutor
        pkg = self.pkg
        pkg.set_device(self.device)
        order = sorted(range(len(requests)), key=lambda i: requests[i]["arrival"])
        pending = deque(order)
        waiting = deque()
        starting, active = [], []
        used = 0.0
        rec = [None] * len(requests)
        t0_ev = pkg.Event(self.device)
        t0 = time.perf_counter()
        t0_ev.record(0)
        held0 = pkg.device_memory_in_use(self.device)
        pkg.set_device_memory_limit(self.device, int(held0 + self.budget))
        peak_active, peak_used = 0, 0.0
        pool = ThreadPoolExecutor(max_workers=self.workers)
        try:
            while pending or waiting or starting or active:
                now = time.perf_counter() - t0
                while pending and requests[pending[0]]["arrival"] <= now:
                    waiting.append(pending.popleft())
                # admission: FIFO while a slot and memory are free
                while waiting and len(active) + len(starting) < self.slots:
                    i = waiting[0]
                    r = requests[i]
                    est = estimate_spec_bytes(r["spec"], r["nsto"])
                    d = admission(est, used, self.budget, bool(active or starting))
                    if d == "wait":
                        break
                    waiting.popleft()
                    if d == "refuse":
                        rec[i] = dict(status="refused", arrival=r["arrival"], nsto=r["nsto"], L=r["L"],
                                      reason=f"estimated {est / 1e9:.2f} GB > budget {self.budget / 1e9:.2f} GB")
                        continue
                    used += est
                    starting.append((i, est, pool.submit(self._start, i, r, t0)))
                # started requests become active (reservation -> measured footprint)
                keep = []
                for i, est, fut in starting:
                    if fut.done():
                        try:
                            a = fut.result()
                        except pkg.SdftError as e:
                            used -= est
                            r = requests[i]
                            rec[i] = dict(status="failed", arrival=r["arrival"], nsto=r["nsto"], L=r["L"],
                                          error=str(e), code=e.code)
                            continue
                        used += a["mem"] - est
                        active.append(a)
                    else:
                        keep.append((i, est, fut))
                starting = keep
                peak_active = max(peak_active, len(active))
                peak_used = max(peak_used, used)
                # completions
                still = []
                for a in active:
                    if a["ev"].query():
                        if a["batch"] is not None:
                            a["batch"].sync()
                        else:
                            a["ctx"].sync()
                        i = a["i"]
                        rho = a["ctx"].download_density() if keep_density else None
                        t_done = t0_ev.elapsed_ms(a["ev"]) / 1e3
                        a["ev"].close()
                        r = requests[i]
                        rec[i] = dict(status="done", arrival=r["arrival"], admitted=a["t_adm"], done=t_done,
                                      latency=t_done - r["arrival"], nsto=r["nsto"], L=r["L"], natm=a["natm"],
                                      mu=a["prep"]["mu"],
                                      num_elec=float(rho.sum() / rho.size) if rho is not None else None, density=rho,
                                      phases=a["prep"]["phases"])
                        if a["batch"] is not None:
                            a["batch"].close()
                        a["ctx"].close()
                        used -= a["mem"]
                    else:
                        still.append(a)
                active = still
                time.sleep(0.0005)
        finally:
            pool.shutdown(wait=True)
            pkg.set_device_memory_limit(self.device, 0)
            t0_ev.close()
        return rec, summarize(rec, peak_active, peak_used, self.workers, self.slots)


def summarize(rec, peak_active=0, peak_used=0.0, workers=None, slots=None):
    """Throughput and latency percentiles over the completed requests, with
    the counts of refused and failed ones."""
    done = [r for r in rec if r and r.get("status") == "done"]
    out = dict(requests=len(rec), completed=len(done),
               refused=sum(1 for r in rec if r and r.get("status") == "refused"),
               failed=sum(1 for r in rec if r and r.get("status") == "failed"),
               peak_active=peak_active, peak_reserved_gb=peak_used / 1e9, workers=workers, slots=slots)
    if not done:
        return out
    lat = np.array([r["latency"] for r in done])
    span = max(r["done"] for r in done) - min(r["arrival"] for r in done)
    out.update(orbitals=int(sum(r["nsto"] for r in done)),
               orbitals_per_s=float(sum(r["nsto"] for r in done) / span), span_s=float(span),
               requests_per_s=float(len(done) / span),
               p50_ms=float(np.percentile(lat, 50) * 1e3), p99_ms=float(np.percentile(lat, 99) * 1e3),
               mean_ms=float(lat.mean() * 1e3),
               prep_mean_s={k: float(np.mean([r["phases"][k] for r in done])) for k in done[0]["phases"]})
    return out


def poisson_requests(wl, n, rate, seed=5, big_fraction=0.1):
    """n requests with seeded Poisson arrivals at `rate` per second drawn from
    the batch distribution with `big_fraction` 512-atom systems."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=n))
    specs = wl.batch_specs(nsys=n, seed=seed + 1, big_fraction=big_fraction)
    return [dict(arrival=float(t[i]), spec=specs[i], nsto=specs[i]["nsto"], L=specs[i]["L"], seed=10.0 + i)
            for i in range(n)]
