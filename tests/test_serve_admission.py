"""Host logic of the server: which queued request is admitted next, and the
seeded request stream (no GPU)."""
from activechi4_b200.serve import RunRequest, next_admissible, poisson_requests


def _q(*ns):
    return [RunRequest(k, n, 1000) for k, n in enumerate(ns)]


def test_arrival_order_without_limit():
    assert next_admissible(_q(50000, 3000), [90000, 60000]) == 0
    assert next_admissible([], []) == -1


def test_large_request_waits_behind_the_limit():
    q = _q(50000, 60000, 3000, 70000)
    # one run above 20000 active: the large requests wait, the small one goes
    assert next_admissible(q, [88000, 4000], max_big=1) == 2
    # none active: arrival order
    assert next_admissible(q, [4000], max_big=1) == 0
    # two allowed, one active
    assert next_admissible(q, [88000], max_big=2) == 0
    # only large requests queued and the limit reached: nothing
    assert next_admissible(_q(50000, 70000), [88000], max_big=1) == -1
    # the bound is strict: exactly big_n particles is not large
    assert next_admissible(_q(20000), [88000], max_big=1, big_n=20000) == 0


def test_request_stream_is_seeded():
    a = poisson_requests(16, seed=5)
    b = poisson_requests(16, seed=5)
    assert [(r.n, r.steps, r.arrival) for r in a] == [(r.n, r.steps, r.arrival) for r in b]
    assert all(1000 <= r.n <= 256000 and r.steps >= 64 for r in a)
    assert all(a[k].arrival < a[k + 1].arrival for k in range(15))
