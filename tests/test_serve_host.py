"""Host logic of the solve server (no GPU): arrival-order admission, one request
per mesh entry at a time, slots running in parallel, HBM-budget eviction (least
recently used, never an entry with queued requests), failure propagation."""
import threading
import time

import numpy as np
import pytest

from exfem_b200 import elements, mesh, serve
from exfem_b200.materials import LinearElastic


class _FakeEntry:
    def __init__(self, spec):
        self.spec, self.bytes, self.busy, self.last_used = spec, spec.device_bytes_estimate(), False, 0.0


def _spec(key, n=2):
    X, c = mesh.box_hex(1.0, 1.0, 1.0, n, n, n)
    fixed = np.zeros(3 * len(X), bool)
    return serve.MeshSpec(key, X, c, elements.HEX8, LinearElastic(1.0, 0.3), fixed)


def _server(slots, budget, solve_time=0.02, log=None):
    lock = threading.Lock()
    active = {"now": 0, "max": 0, "per_key": {}}

    def setup_fn(spec):
        if log is not None:
            log.append(("setup", spec.key))
        return _FakeEntry(spec)

    def solve_fn(entry, req):
        with lock:
            active["now"] += 1
            active["max"] = max(active["max"], active["now"])
            k = entry.spec.key
            active["per_key"][k] = active["per_key"].get(k, 0) + 1
            assert active["per_key"][k] == 1, "two requests on one entry at once"
        time.sleep(solve_time)
        with lock:
            active["now"] -= 1
            active["per_key"][entry.spec.key] -= 1
        return np.asarray(req.rhs) * 2.0, dict(iters=1)

    s = serve.SolveServer(slots=slots, hbm_budget=budget, setup_workers=0, solve_fn=solve_fn, setup_fn=setup_fn)
    return s, active


def test_requests_run_in_parallel_and_one_per_entry():
    specs = [_spec(f"m{i}") for i in range(4)]
    s, active = _server(slots=4, budget=1e12)
    try:
        futs = []
        for i in range(16):
            sp = specs[i % 4]
            futs.append(s.submit(serve.SolveRequest(sp, rhs=np.full(sp.ndof, float(i)))))
        for i, f in enumerate(futs):
            x, info = f.result(timeout=30)
            np.testing.assert_array_equal(x, np.full(specs[i % 4].ndof, 2.0 * i))
        assert active["max"] >= 2
        st = serve.latency_stats(s.completed)
        assert st["n"] == 16 and st["p99_s"] >= st["p50_s"] > 0
    finally:
        s.close()


def test_budget_evicts_least_recently_used_idle_entry():
    log = []
    one = _spec("a").device_bytes_estimate()
    s, _ = _server(slots=1, budget=2.5 * one, log=log)
    try:
        for key in ["a", "b", "a", "c", "a"]:
            sp = _spec(key)
            s.submit(serve.SolveRequest(sp, rhs=np.zeros(sp.ndof))).result(timeout=30)
        # c evicts b (a was used more recently); the last a needs no new set-up
        assert [k for _, k in log] == ["a", "b", "c"]
        assert s.evictions == 1
        assert s.entry("b") is None and s.entry("a") is not None and s.entry("c") is not None
        assert s.resident_bytes <= 2.5 * one
    finally:
        s.close()


def test_requests_start_in_arrival_order_per_entry():
    s, _ = _server(slots=1, budget=1e12, solve_time=0.01)
    try:
        sp = _spec("x")
        futs = [s.submit(serve.SolveRequest(sp, rhs=np.full(sp.ndof, float(i)))) for i in range(6)]
        for f in futs:
            f.result(timeout=30)
        starts = [r.t_start for r in sorted(s.completed, key=lambda r: r.id)]
        assert starts == sorted(starts)
    finally:
        s.close()


def test_solve_failure_reaches_the_future():
    def bad(entry, req):
        raise RuntimeError("not converged")
    s = serve.SolveServer(slots=2, setup_workers=0, solve_fn=bad, setup_fn=lambda sp: _FakeEntry(sp))
    try:
        sp = _spec("f")
        with pytest.raises(RuntimeError, match="not converged"):
            s.submit(serve.SolveRequest(sp, rhs=np.zeros(sp.ndof))).result(timeout=30)
    finally:
        s.close()


def test_request_kind_must_match_entry():
    sp = _spec("k")
    with pytest.raises(ValueError):
        serve.SolveRequest(sp)
    with pytest.raises(ValueError):
        serve.SolveRequest(sp, step=object())


def test_request_records_for_latency_reports():
    """Per-request records (the raw data behind p50 / p99): one JSON-serialisable
    record per finished request with its queue, service and total times and the
    solver's info, consistent with the latency statistics."""
    import json
    specs = [_spec(f"m{i}") for i in range(2)]
    s, _ = _server(slots=2, budget=1e12, solve_time=0.01)
    try:
        futs = [s.submit(serve.SolveRequest(specs[i % 2], rhs=np.ones(specs[i % 2].ndof))) for i in range(6)]
        for f in futs:
            f.result(timeout=30)
        recs = serve.request_records(list(s.completed))
    finally:
        s.close()
    assert len(recs) == 6 and len({r["id"] for r in recs}) == 6
    json.dumps(recs)
    for r in recs:
        assert r["kind"] == "linear" and r["mesh"] in ("m0", "m1") and r["iters"] == 1
        assert r["queue_s"] >= 0 and r["service_s"] >= 0.01
        assert abs(r["latency_s"] - (r["queue_s"] + r["service_s"])) < 1e-9
    st = serve.latency_stats(list(s.completed))
    assert abs(st["p50_s"] - float(np.percentile([r["latency_s"] for r in recs], 50))) < 1e-12


def test_pending_requests_can_be_withdrawn():
    """Requests that have not started can be withdrawn (one by one or the whole
    backlog); their futures report cancellation, running ones still finish."""
    sp = _spec("m0")
    s, _ = _server(slots=1, budget=1e12, solve_time=0.2)
    try:
        futs = [s.submit(serve.SolveRequest(sp, rhs=np.full(sp.ndof, float(i)))) for i in range(6)]
        time.sleep(0.05)                                   # the first request is running
        reqs = list(s._pending)
        assert s.cancel(reqs[0]) and not s.cancel(reqs[0])
        n = s.cancel_pending()
        assert n == len(reqs) - 1
        x, _ = futs[0].result(timeout=30)
        np.testing.assert_array_equal(x, np.zeros(sp.ndof))
        assert all(f.cancelled() for f in futs[1:])
    finally:
        s.close()
