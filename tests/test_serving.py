"""The request loop's scheduling on a host-only backend with the batch's
admission rules: every request completes, the byte budget and slot count
are never exceeded, requests run concurrently and finished ones release
their memory, and a request larger than the whole budget is rejected without
stopping the others."""
import numpy as np

from enscdynamics_b200 import serving as S
from enscdynamics_b200 import workloads as W


class _Mesh:
    def __init__(self, ne):
        self.n_elements = ne


class _Problem:
    def __init__(self, ne, cycles):
        self.mesh = _Mesh(ne)
        self.cycles = cycles


def stream(n, rate=50.0, seed=5):
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        ne = int(np.exp(rng.uniform(np.log(1000), np.log(500000))))
        out.append(W.Request(i, t, _Problem(ne, int(rng.integers(1000, 10001)))))
    return out


def run(reqs, **kw):
    be = S.FakeBackend(**kw)
    srv = S.Server(be, clock=be.now, sleep=be.sleep)
    return be, srv.serve(reqs)


def test_all_complete_within_budget_and_slots():
    reqs = stream(200)
    budget = 200_000 * 400 * 3   # about three large requests at a time
    be, out = run(reqs, budget_bytes=budget, max_instances=16)
    assert all(o.status == 0 and o.cycles == r.problem.cycles for o, r in zip(out, reqs))
    assert be.peak <= budget and be.peak_instances <= 16
    assert be.peak_instances > 1          # requests overlap on the device
    assert be.used == 0 and not be.slots  # everything retired and freed
    for o in out:
        assert o.arrival <= o.admitted <= o.finished
    s = S.summarize(out)
    assert s["requests"] == 200 and s["failed"] == 0
    assert s["p99_latency_s"] >= s["p50_latency_s"] > 0


def test_backfill_admits_small_requests_past_a_blocked_large_one():
    reqs = [W.Request(0, 0.0, _Problem(900, 5000)), W.Request(1, 0.001, _Problem(900, 100)),
            W.Request(2, 0.002, _Problem(100, 100))]
    be, out = run(reqs, budget_bytes=1000 * 400, max_instances=8)
    # request 1 waits for request 0; request 2 fits beside request 0 and finishes first
    assert out[2].admitted < out[1].admitted
    assert out[2].finished < out[0].finished
    assert out[1].admitted >= out[0].finished


def test_oversized_request_is_rejected_and_others_finish():
    reqs = [W.Request(0, 0.0, _Problem(10_000, 100)), W.Request(1, 0.5, _Problem(10, 100)),
            W.Request(2, 0.6, _Problem(20, 200))]
    be, out = run(reqs, budget_bytes=1000 * 400, max_instances=8)
    assert out[0].status == S.ERR_OOM
    assert out[1].status == 0 and out[2].status == 0 and out[2].cycles == 200


def test_quantum_follows_the_earliest_finishing_instance():
    reqs = [W.Request(0, 0.0, _Problem(100, 1000)), W.Request(1, 0.0, _Problem(100, 70))]
    be, out = run(reqs, budget_bytes=10 ** 9, max_instances=8)
    # the short request retires after one 70-cycle quantum, not after 1024
    assert out[1].finished <= out[0].finished
    assert be.cycles_run < 1000 + 64


def test_prepare_on_threads_matches_inline_prepare():
    reqs = stream(120, seed=9)
    budget = 200_000 * 400 * 3
    outs = []
    for workers in (0, 3):
        be = S.FakeBackend(budget_bytes=budget, max_instances=16)
        srv = S.Server(be, clock=be.now, sleep=be.sleep, prepare_workers=workers, prepare_ahead=4)
        out = srv.serve(reqs)
        assert all(o.status == 0 for o in out) and be.used == 0
        assert srv.stats["quanta"] > 0 and srv.stats["cycles"] >= max(r.problem.cycles for r in reqs)
        outs.append(out)
    # threads change only when a request's host part is ready, not what runs
    for a, b in zip(*outs):
        assert a.cycles == b.cycles and a.arrival <= a.admitted <= a.finished and b.arrival <= b.admitted


def test_a_request_whose_host_part_fails_is_reported_and_others_finish():
    reqs = [W.Request(0, 0.0, _Problem(500, 300)), W.Request(1, 0.1, _Problem(0, 100)),
            W.Request(2, 0.2, _Problem(300, 200))]
    for workers in (0, 2):
        be = S.FakeBackend(budget_bytes=10 ** 9, max_instances=8)
        out = S.Server(be, clock=be.now, sleep=be.sleep, prepare_workers=workers).serve(reqs)
        assert out[1].status == S.ERR_ARG and out[1].finished >= out[1].arrival
        assert out[0].status == 0 and out[2].status == 0 and out[2].cycles == 200


def test_request_admitted_during_a_quantum_joins_the_next_with_all_its_cycles():
    # request 1 arrives while the first quantum runs: it is admitted then (the
    # device part beside the running cycles), takes no part in that quantum,
    # and the next quantum is sized by its full cycle count
    reqs = [W.Request(0, 0.0, _Problem(1000, 1000)), W.Request(1, 1e-6, _Problem(1000, 300))]
    be = S.FakeBackend(budget_bytes=10 ** 9, max_instances=8)
    srv = S.Server(be, clock=be.now, sleep=be.sleep)
    out = srv.serve(reqs)
    assert [o.status for o in out] == [0, 0]
    assert out[1].cycles == 300 and out[0].cycles == 1000
    assert out[1].admitted <= out[0].finished
    assert srv.stats["quanta"] == 2 and be.cycles_run == 1300


def test_request_refused_during_a_quantum_is_admitted_after_the_retire():
    # request 1 arrives while request 0 holds the whole budget: the admission
    # tried during the quantum is refused, and the one after request 0
    # retires takes it
    reqs = [W.Request(0, 0.0, _Problem(1000, 200)), W.Request(1, 1e-6, _Problem(1000, 100))]
    be = S.FakeBackend(budget_bytes=1000 * 400, max_instances=8)
    srv = S.Server(be, clock=be.now, sleep=be.sleep)
    out = srv.serve(reqs)
    assert [o.status for o in out] == [0, 0]
    assert out[1].cycles == 100 and out[1].admitted >= out[0].finished
    assert be.peak <= 1000 * 400 and be.used == 0
