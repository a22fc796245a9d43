"""Scheduler of the serving loop (cq_server_*) in dry-run mode: no device work, each request holds
its slot and its memory estimate for a fixed time.  Checks slot concurrency, admission by HBM
budget, the bypass bound and the latency bookkeeping."""
import pytest

import cq_b200
from cq_b200 import inputs


def _overlaps(res):
    """Largest number of requests holding a slot at the same time."""
    ev = sorted([(r["t_admit"], 1) for r in res] + [(r["t_done"], -1) for r in res], key=lambda e: (e[0], e[1]))
    cur = best = 0
    for _, d in ev:
        cur += d
        best = max(best, cur)
    return best


@pytest.fixture(scope="module")
def small():
    c, cell = inputs.diamond_si(1, sigma=0.1, seed=1)
    return c, cell


def test_slots_bound_concurrency(small):
    c, cell = small
    s = cq_b200.Server(n_slots=3, hbm_budget=1 << 40, dry_run=True, dry_run_seconds=0.05)
    ids = [s.submit(c, cell, 4, 5, 6, 8, 5, 8.0, seed=k) for k in range(9)]
    res = [s.wait(i) for i in ids]
    s.close()
    assert all(r["status"] == 0 for r in res)
    assert _overlaps(res) <= 3
    assert sorted({r["slot"] for r in res}) == [0, 1, 2]
    for r in res:
        assert r["t_arrival"] <= r["t_admit"] <= r["t_done"]
        assert r["latency"] >= 0.05 * 0.9


def test_budget_serialises(small):
    c, cell = small
    est = cq_b200.request_estimate(c, cell, 4, 5, 6, 8, 5)
    s = cq_b200.Server(n_slots=4, hbm_budget=int(1.5 * est), dry_run=True, dry_run_seconds=0.03)
    ids = [s.submit(c, cell, 4, 5, 6, 8, 5, 8.0) for _ in range(5)]
    res = [s.wait(i) for i in ids]
    s.close()
    assert _overlaps(res) == 1
    assert all(r["bytes_estimate"] == est for r in res)


def test_oversized_request_runs_alone(small):
    c, cell = small
    est = cq_b200.request_estimate(c, cell, 4, 5, 6, 8, 5)
    s = cq_b200.Server(n_slots=2, hbm_budget=est // 2, dry_run=True, dry_run_seconds=0.02)
    ids = [s.submit(c, cell, 4, 5, 6, 8, 5, 8.0) for _ in range(3)]
    res = [s.wait(i) for i in ids]
    s.close()
    assert all(r["status"] == 0 for r in res)
    assert _overlaps(res) == 1


def test_bypass_bound(small):
    """A large request waiting for memory is overtaken by at most max_bypass later small ones."""
    c, cell = small
    big_c, big_cell = inputs.diamond_si(2, sigma=0.1, seed=2)
    e_small = cq_b200.request_estimate(c, cell, 4, 5, 6, 8, 5)
    e_big = cq_b200.request_estimate(big_c, big_cell, 13, 10, 12, 16, 10)
    assert e_big > 2 * e_small
    budget = e_big + e_small // 2        # the big one fits only when nothing else runs
    s = cq_b200.Server(n_slots=2, hbm_budget=budget, max_bypass=2, dry_run=True, dry_run_seconds=0.05)
    first = s.submit(c, cell, 4, 5, 6, 8, 5, 8.0)
    big = s.submit(big_c, big_cell, 13, 10, 12, 16, 10, 64.0)
    later = [s.submit(c, cell, 4, 5, 6, 8, 5, 8.0) for _ in range(5)]
    r_first = s.wait(first)
    r_big = s.wait(big)
    r_later = [s.wait(i) for i in later]
    s.close()
    overtook = [r for r in r_later if r["t_admit"] < r_big["t_admit"]]
    assert len(overtook) <= 2
    assert r_big["t_admit"] >= r_first["t_done"] - 1e-6


def test_wait_timeout(small):
    c, cell = small
    s = cq_b200.Server(n_slots=1, hbm_budget=1 << 40, dry_run=True, dry_run_seconds=0.3)
    i = s.submit(c, cell, 4, 5, 6, 8, 5, 8.0)
    with pytest.raises(cq_b200.CQError) as e:
        s.wait(i, timeout=0.01)
    assert e.value.code == cq_b200.CQ_ERR_TIMEOUT
    assert s.wait(i)["status"] == 0
    s.close()


def test_estimate_grows_with_size_and_precision(small):
    c, cell = small
    c2, cell2 = inputs.diamond_si(2, sigma=0.1, seed=1)
    e1 = cq_b200.request_estimate(c, cell, 4, 10, 12, 16, 10)
    e2 = cq_b200.request_estimate(c2, cell2, 4, 10, 12, 16, 10)
    e3 = cq_b200.request_estimate(c2, cell2, 13, 10, 12, 16, 10)
    e4 = cq_b200.request_estimate(c2, cell2, 13, 10, 12, 16, 10, mixed=True)
    assert e1 < e2 < e3 < e4


def test_bad_request_rejected(small):
    c, cell = small
    s = cq_b200.Server(n_slots=1, dry_run=True)
    with pytest.raises(cq_b200.CQError):
        s.submit(c, cell, 0, 5, 6, 8, 5, 8.0)
    with pytest.raises(cq_b200.CQError):
        s.submit(c, cell, 4, 5, 6, 8, 5, -1.0)
    s.close()
