"""Host logic of the request server (no GPU): request generation and the
device-memory admission ledger."""
import numpy as np

from conftest import ensure_library  # noqa: F401  (package path setup)

from cudolfinx import serve


def test_problem_sizes_match_formulas():
    from oracle import fem_oracle as fo
    for n in (2, 3, 4):
        s1 = serve.problem_sizes("p1", n)
        s2 = serve.problem_sizes("p2", n)
        sv = serve.problem_sizes("vp2", n)
        assert s1["nnz"] == fo.nnz_formula("p1", n)
        assert s2["nnz"] == fo.nnz_formula("p2", n)
        assert sv["nnz"] == 9 * s2["nnz"] and sv["rows"] == 3 * s2["rows"]
        assert s1["cells"] == 6 * n ** 3


def test_make_requests_mix_and_arrivals():
    reqs = serve.make_requests(4000, rate=500.0, seed=1, nmin=8, nmax=96, mix=(0.35, 0.35, 0.30),
                               materialize=False)
    kinds = np.array([r.kind for r in reqs])
    for k, p in zip(serve.FAMILIES, (0.35, 0.35, 0.30)):
        assert abs(np.mean(kinds == k) - p) < 0.03
    ns = np.array([r.n for r in reqs])
    assert ns.min() >= 8 and ns.max() <= 96
    # log-uniform: the median of log n sits midway
    assert abs(np.median(np.log(ns)) - 0.5 * (np.log(8) + np.log(96))) < 0.1
    arr = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(arr) >= 0) and arr[0] == 0.0
    assert abs(len(reqs) / arr[-1] - 500.0) / 500.0 < 0.1
    small = serve.make_requests(20, rate=500.0, seed=2, nmin=2, nmax=6)
    for r in small:
        C = 6 * r.n ** 3
        assert all(c.shape == (C,) and np.all(c > 0) for c in r.coef)
        assert len(r.coef) == (2 if r.kind == "vp2" else 1)


def test_ledger_reuse_evict_wait_never():
    L = serve.SlotLedger(1000)
    st, obj = L.reserve(("p1", 4), 300, 100)
    assert st == "new" and obj is None and L.used == 400
    a = object()
    L.register(("p1", 4), a, 300)
    # same key while busy: another slot, shared bytes not charged again
    st, _ = L.reserve(("p1", 4), 300, 100)
    assert st == "new" and L.used == 700
    b = object()
    L.register(("p1", 4), b, 300)
    # no room now and nothing idle: wait
    st, _ = L.reserve(("p2", 4), 250, 100)
    assert st == "wait" and L.used == 700
    # more than the whole budget: never
    st, _ = L.reserve(("vp2", 9), 2000, 10)
    assert st == "never"
    # releasing keeps the slot idle for reuse
    L.release(("p1", 4), a)
    st, obj = L.reserve(("p1", 4), 300, 100)
    assert st == "reuse" and obj is a and L.used == 700
    L.release(("p1", 4), a)
    L.release(("p1", 4), b)
    # a new size evicts idle slots least recently released first
    st, _ = L.reserve(("p2", 4), 250, 100)
    assert st == "new"
    ev = L.take_evicted()
    assert [o for _, o in ev] == [a]
    assert L.used == 300 + 100 + 250 + 100 and L.used <= L.budget
    assert L.peak <= L.budget
    # dropping the last slot of a size frees its shared bytes too
    c = object()
    L.register(("p2", 4), c, 250)
    L.release(("p2", 4), c, keep=False)
    assert L.used == 400 and ("p2", 4) not in L.shared


def test_ledger_cancel_new_restores():
    L = serve.SlotLedger(1000)
    st, _ = L.reserve(("p1", 3), 200, 50)
    assert st == "new" and L.used == 250
    L.cancel_new(("p1", 3), 200)
    assert L.used == 0 and not L.shared


def test_summarize_percentiles():
    rs = [serve.Result(i, "p1", 4, np.zeros(3), 5, 1e-9, arrival=0.1 * i, admitted=0.1 * i,
                       done=0.1 * i + 0.01 * (i + 1)) for i in range(100)]
    s = serve.summarize(rs)
    assert s["completed"] == 100 and s["errors"] == 0
    lat = [r.latency for r in rs]
    assert abs(s["p50_ms"] - 1e3 * np.percentile(lat, 50)) < 1e-9
    assert abs(s["p99_ms"] - 1e3 * np.percentile(lat, 99)) < 1e-9
