"""The served leg's latency summary (bench.py served_summary), on synthetic
request results: a request still running when the loop stops is censored,
counts at its lower bound (stop - arrival), and a percentile that reaches
into the censored requests is flagged as a lower bound; time to nucleation
only counts nucleated requests (done == 1, chk-nucleation.f:35-56)."""
import os
import sys

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)

import bench  # noqa: E402
import clmd  # noqa: E402


def results(rows):
    out = []
    for arrival, admitted, finished, done, clbrkt in rows:
        r = clmd.RequestResult()
        r.arrival, r.admitted, r.finished = arrival, admitted, finished
        r.done, r.clbrkt, r.natom = done, clbrkt, 1000
        out.append(r)
    return out


def stats(wall, completed):
    st = clmd.ServeStats()
    st.wall, st.completed, st.admitted = wall, completed, completed
    return st


def test_all_finished_is_uncensored():
    # 100 requests: latencies 1..100 s; every 4th nucleated at step 1000 k
    rows = [(0.0, 0.1, float(k), 1 if k % 4 == 0 else 2, 1000 * k) for k in range(1, 101)]
    s = bench.served_summary(results(rows), stats(100.0, 100), 100, 120.0)
    lat = s["latency_s"]
    assert not lat["p50_is_lower_bound"] and not lat["p99_is_lower_bound"]
    assert lat["p50"] == np.percentile(np.arange(1, 101), 50)
    assert lat["p99"] == np.percentile(np.arange(1, 101), 99)
    assert lat["time_to_nucleation_p50"] == np.percentile(np.arange(4, 101, 4), 50)
    assert lat["nucleation_step_p50"] == np.percentile(1000 * np.arange(4, 101, 4), 50)
    assert s["requests"]["censored"] == 0 and s["requests"]["nucleated"] == 25


def test_censored_requests_count_at_their_lower_bound():
    # 60 finished at 1..60 s, 40 still running when the loop stopped at 90 s
    rows = [(0.0, 0.1, float(k), 2, 0) for k in range(1, 61)]
    rows += [(10.0, 10.1, -1.0, 0, 0) for _ in range(40)]
    s = bench.served_summary(results(rows), stats(90.0, 60), 100, 90.0)
    lat = s["latency_s"]
    everyone = np.array(list(range(1, 61)) + [80.0] * 40)
    assert lat["p50"] == np.percentile(everyone, 50)
    assert lat["p99"] == 80.0
    assert not lat["p50_is_lower_bound"] and lat["p99_is_lower_bound"]
    assert lat["completed_p50"] == np.percentile(np.arange(1, 61), 50)
    assert s["requests"]["censored"] == 40
    assert lat["time_to_nucleation_p50"] is None


def test_majority_censored_flags_the_median():
    rows = [(0.0, 0.1, 5.0, 1, 200)] * 10 + [(0.0, 0.1, -1.0, 0, 0)] * 90
    s = bench.served_summary(results(rows), stats(30.0, 10), 100, 30.0)
    lat = s["latency_s"]
    assert lat["p50_is_lower_bound"] and lat["p99_is_lower_bound"]
    assert lat["p50"] == 30.0 and lat["time_to_nucleation_p50"] == 5.0
