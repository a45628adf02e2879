"""Batched systems (one CUDA graph over several contexts) and the serving
loop, on small uneven systems: every result equals the same system filtered
alone and eagerly."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

SPECS = [dict(nrep=(1, 1, 1), grid=(24, 24, 24), strain=(0.01, -0.02, 0.005), disp_seed=11, nsto=6, L=24),
         dict(nrep=(2, 1, 1), grid=(48, 24, 24), strain=(-0.01, 0.0, 0.02), disp_seed=12, nsto=10, L=32),
         dict(nrep=(1, 2, 1), grid=(24, 48, 24), strain=(0.0, 0.015, -0.01), disp_seed=13, nsto=4, L=20)]


def _serve_mod(pkg):
    return __import__(pkg.__name__ + ".serve", fromlist=["prepare"])


@pytest.mark.parametrize("prec", [0, 1])
def test_batch_graph_matches_eager(pkg, wl, prec):
    serve = _serve_mod(pkg)
    preps, eager = [], []
    for i, sp in enumerate(SPECS):
        s = wl.build_spec(sp)
        p = serve.prepare(pkg, wl, s, sp["nsto"], sp["L"], prec, seed=20.0 + i)
        c = p["ctx"]
        c.filter_cheby_dev(sp["nsto"], p["ec"], 1, p["scale"], p["emean"])
        eager.append((c.density_dev(sp["nsto"], 0, p["occ_over"]), c.download_filtered(sp["nsto"])))
        preps.append(p)
    b = pkg.Batch([p["ctx"] for p in preps], [sp["nsto"] for sp in SPECS], [sp["L"] for sp in SPECS],
                  [p["ec"] for p in preps], [p["scale"] for p in preps], [p["emean"] for p in preps],
                  [p["occ_over"] for p in preps])
    assert b.kernels_per_launch > 0
    for _ in range(2):  # replays recompute from the resident noise
        b.launch()
        b.sync()
        for p, sp, (rho, (fr, fi)) in zip(preps, SPECS, eager):
            assert rel_l2(p["ctx"].download_density(), rho) < 1e-14
            gr, gi = p["ctx"].download_filtered(sp["nsto"])
            assert rel_l2(np.concatenate([gr, gi]), np.concatenate([fr, fi])) < 1e-14
    b.close()
    for p in preps:
        p["ctx"].close()


@pytest.mark.parametrize("graph", [False, True])
def test_serving_same_result_alone_and_in_mix(pkg, wl, graph):
    serve = _serve_mod(pkg)
    reqs = [dict(arrival=0.0 + 0.001 * i, spec=sp, nsto=sp["nsto"], L=sp["L"], seed=30.0 + i)
            for i, sp in enumerate(SPECS)]
    srv = serve.Server(pkg, wl, pkg.SDFT_PREC_MIXED, hbm_budget=150e9, slots=8, graph=graph)
    mix, summ = srv.run(reqs)
    assert summ["requests"] == 3 and summ["p99_ms"] >= summ["p50_ms"] > 0
    for i, r in enumerate(reqs):
        alone, _ = srv.run([dict(r, arrival=0.0)])
        assert rel_l2(mix[i]["density"], alone[0]["density"]) < 1e-14
        assert abs(mix[i]["num_elec"] - alone[0]["num_elec"]) < 1e-12 * abs(alone[0]["num_elec"])


def test_serving_refuses_oversize_and_serves_the_rest(pkg, wl):
    """Under a 0.5 GB budget the 512-atom request can never fit: it is
    refused at admission, the small ones complete, and their densities equal
    the same requests served under the full budget."""
    serve = _serve_mod(pkg)
    big = dict(nrep=(4, 4, 4), grid=(96, 96, 96), strain=(0.0, 0.0, 0.0), disp_seed=1, nsto=64, L=16)
    reqs = [dict(arrival=0.0, spec=SPECS[0], nsto=6, L=24, seed=40.0),
            dict(arrival=0.0, spec=big, nsto=64, L=16, seed=41.0),
            dict(arrival=0.001, spec=SPECS[2], nsto=4, L=20, seed=42.0)]
    assert serve.estimate_spec_bytes(big, 64) > 0.5e9 > serve.estimate_spec_bytes(SPECS[0], 6)
    small = serve.Server(pkg, wl, pkg.SDFT_PREC_MIXED, hbm_budget=0.5e9, slots=4)
    rec, summ = small.run(reqs)
    assert [r["status"] for r in rec] == ["done", "refused", "done"]
    assert (summ["completed"], summ["refused"], summ["failed"]) == (2, 1, 0)
    assert "budget" in rec[1]["reason"]
    assert pkg.device_memory_in_use(0) < 0.5e9  # every completed request released its context
    full = serve.Server(pkg, wl, pkg.SDFT_PREC_MIXED, hbm_budget=150e9, slots=4)
    ref, _ = full.run([reqs[0], reqs[2]])
    assert rel_l2(rec[0]["density"], ref[0]["density"]) < 1e-14
    assert rel_l2(rec[2]["density"], ref[1]["density"]) < 1e-14
