"""Host-side logic of the serving loop and the batch workload (no GPU):
request priorities, the device-memory estimate used for admission, the
seeded request stream and the uneven-system specs."""
import importlib

import numpy as np
import pytest


@pytest.fixture(scope="module")
def serve(pkg):
    return importlib.import_module(pkg.__name__ + ".serve")


def test_request_priority_orders_by_work(serve):
    small = serve.request_priority((24, 24, 24), 16, 128)
    mid = serve.request_priority((48, 48, 48), 128, 256)
    big = serve.request_priority((96, 96, 96), 256, 512)
    assert small <= mid <= big <= 0
    assert small == -5 and big == 0  # cheapest gets the most urgent level, 512 atoms the default


def test_memory_estimate_grows_with_work(serve, wl):
    specs = wl.batch_specs(nsys=12, seed=4, big_fraction=0.25)
    est = [serve.estimate_spec_bytes(s, s["nsto"]) for s in specs]
    assert all(e > 64 * 2 ** 20 for e in est)
    # more orbitals of the same system never need less memory
    s = specs[0]
    assert serve.estimate_spec_bytes(s, 2 * s["nsto"]) > serve.estimate_spec_bytes(s, s["nsto"])


def test_spec_estimate_close_to_built_estimate(serve, wl):
    # the pre-build estimate (cell volume and cutoff) brackets the exact one
    specs = wl.batch_specs(nsys=4, seed=9, big_fraction=0.0)
    for sp in specs:
        s = wl.build_spec(sp)
        exact = serve.estimate_bytes(s, sp["nsto"])
        pre = serve.estimate_spec_bytes(sp, sp["nsto"])
        assert 0.9 * exact <= pre <= 1.5 * exact


def test_poisson_requests_are_seeded_and_ordered(serve, wl):
    a = serve.poisson_requests(wl, 20, 50.0, seed=5, big_fraction=0.1)
    b = serve.poisson_requests(wl, 20, 50.0, seed=5, big_fraction=0.1)
    t = np.array([r["arrival"] for r in a])
    assert np.all(np.diff(t) > 0) and [r["seed"] for r in a] == [r["seed"] for r in b]
    assert [r["nsto"] for r in a] == [r["nsto"] for r in b]
    assert all(r["nsto"] % 2 == 0 and r["L"] % 2 == 0 for r in a)


def test_admission_refuses_what_never_fits(serve):
    gb = 1e9
    assert serve.admission(151 * gb, 0.0, 150 * gb, busy=False) == "refuse"
    assert serve.admission(151 * gb, 10 * gb, 150 * gb, busy=True) == "refuse"
    assert serve.admission(100 * gb, 60 * gb, 150 * gb, busy=True) == "wait"
    assert serve.admission(100 * gb, 60 * gb, 150 * gb, busy=False) == "admit"  # idle: whatever fits alone
    assert serve.admission(10 * gb, 60 * gb, 150 * gb, busy=True) == "admit"


def test_summary_counts_refused_and_failed(serve):
    rec = [dict(status="done", arrival=0.0, done=2.0, latency=2.0, nsto=16, phases={"x": 1.0}),
           dict(status="done", arrival=1.0, done=3.0, latency=2.0, nsto=32, phases={"x": 3.0}),
           dict(status="refused", arrival=1.5, nsto=256, L=512, reason="too big"),
           dict(status="failed", arrival=1.7, nsto=64, L=128, error="nomem", code=3)]
    s = serve.summarize(rec)
    assert (s["requests"], s["completed"], s["refused"], s["failed"]) == (4, 2, 1, 1)
    assert s["orbitals"] == 48 and abs(s["orbitals_per_s"] - 16.0) < 1e-12
    assert s["p50_ms"] == 2000.0 and s["prep_mean_s"] == {"x": 2.0}
    assert serve.summarize([rec[2]])["completed"] == 0


@pytest.mark.parametrize("mod", ["serve", "tuner"])
def test_serving_and_tuning_need_no_torch(pkg, mod):
    """The serving loop and the autotuner time and order device work through
    the library's own event calls: neither imports torch."""
    import ast
    import os
    src = open(os.path.join(os.path.dirname(pkg.__file__), mod + ".py")).read()
    names = set()
    for node in ast.walk(ast.parse(src)):
        if isinstance(node, ast.Import):
            names.update(a.name.split(".")[0] for a in node.names)
        elif isinstance(node, ast.ImportFrom) and node.module:
            names.add(node.module.split(".")[0])
    assert "torch" not in names
