"""Continuous-batching request loop (host logic, fake backend; no GPU)."""
import threading
import time

import pytest

from difftetvr_b200.serve import Request, Result, ServingEngine


class FakeBackend:
    """Completes a batch `delay` seconds after launch; records what it saw."""

    def __init__(self, slots=2, delay=0.02, fpp=10.0):
        self.slots = slots
        self.delay = delay
        self.fpp = fpp
        self.launched = []
        self.max_concurrent = 0
        self.active = 0
        self.lock = threading.Lock()

    def fragments_per_pixel(self, mesh):
        return self.fpp

    def launch(self, slot, reqs):
        with self.lock:
            self.active += 1
            self.max_concurrent = max(self.max_concurrent, self.active)
        self.launched.append((slot, [r.id for r in reqs]))
        return {"t": time.perf_counter() + self.delay, "reqs": reqs}

    def done(self, h):
        return time.perf_counter() >= h["t"]

    def finish(self, h):
        with self.lock:
            self.active -= 1
        return [Result(r.id, image=("img", r.id)) for r in h["reqs"]]


def req(w=16, h=16, mode="forward"):
    return Request(mesh="m", view_matrix=[0.0] * 16, width=w, height=h, mode=mode)


def test_all_requests_complete_in_arrival_order_within_budget():
    be = FakeBackend(delay=0.005)
    eng = ServingEngine(be, budget_fragments=10 * 16 * 16 * 3, max_batch=8)  # 3 requests per batch
    eng.start()
    futs = [eng.submit(req()) for _ in range(20)]
    res = [f.result(timeout=10) for f in futs]
    eng.stop()
    assert [r.request_id for r in res] == list(range(20))
    launched = [i for _, ids in be.launched for i in ids]
    assert launched == list(range(20))  # FIFO admission
    assert max(len(ids) for _, ids in be.launched) <= 3  # memory budget respected
    st = eng.latency_stats()
    assert st["requests"] == 20 and st["p99_ms"] >= st["p50_ms"] > 0
    # Latency = queueing + service; the slowest requests come with their batch.
    assert st["queue_p50_ms"] >= 0 and st["service_p50_ms"] > 0
    assert st["service_p99_ms"] <= st["p99_ms"] + 1e-9
    slow = st["slowest"]
    assert len(slow) == 3 and slow[0]["ms"] >= slow[1]["ms"] >= slow[2]["ms"]
    assert all(0 <= x["queue_ms"] <= x["ms"] and 1 <= x["batch_size"] <= 3 for x in slow)


def test_requests_arriving_during_a_batch_start_on_the_free_slot():
    be = FakeBackend(slots=2, delay=0.05)
    eng = ServingEngine(be, budget_fragments=10 * 16 * 16, max_batch=1)
    eng.start()
    f1 = eng.submit(req())
    time.sleep(0.01)
    f2 = eng.submit(req())  # arrives while the first batch is on the "GPU"
    f1.result(timeout=5)
    f2.result(timeout=5)
    eng.stop()
    assert be.max_concurrent == 2
    assert {s for s, _ in be.launched} == {0, 1}


def test_over_budget_request_is_rejected_and_others_proceed():
    be = FakeBackend(delay=0.001)
    eng = ServingEngine(be, budget_fragments=10 * 32 * 32)
    eng.start()
    bad = eng.submit(req(64, 64))
    good = eng.submit(req(32, 32))
    with pytest.raises(RuntimeError):
        bad.result(timeout=5)
    assert good.result(timeout=5).request_id == good_id(good, eng)
    eng.stop()
    assert eng.rejected == 1


def good_id(fut, eng):
    return [r.id for r in eng.completed][-1]


def test_cancel_pending_requests():
    be = FakeBackend(slots=1, delay=0.05)
    eng = ServingEngine(be, budget_fragments=10 * 16 * 16, max_batch=1)
    eng.start()
    futs = [eng.submit(req()) for _ in range(5)]
    time.sleep(0.01)
    n = eng.cancel_pending()
    eng.stop()
    assert n >= 3
    assert sum(f.cancelled() for f in futs) == n
    assert all(f.done() for f in futs)


def test_sjf_admits_small_requests_first_and_aged_ones_before_them():
    """Shortest-estimate-first admission with an age bound: among fresh
    requests the smallest go first; a request queued longer than the age
    bound goes before all fresh ones."""
    be = FakeBackend(slots=1, delay=0.0)
    eng = ServingEngine(be, budget_fragments=10 * 64 * 64 * 4, max_batch=2, policy="sjf", age_ms=1e6)
    big, small1, small2 = req(64, 64), req(16, 16), req(16, 16)
    for i, r in enumerate((big, small1, small2)):
        r.id, r.t_arrival = i, time.perf_counter()
        eng.queue.append(r)
    first = eng.admit()
    assert [r.id for r in first] == [1, 2]
    assert [r.id for r in eng.queue] == [0]
    # The same queue with the big request aged past the bound.
    eng2 = ServingEngine(be, budget_fragments=10 * 64 * 64 * 4, max_batch=2, policy="sjf", age_ms=5.0)
    big2, small3 = req(64, 64), req(16, 16)
    big2.id, big2.t_arrival = 0, time.perf_counter() - 1.0
    small3.id, small3.t_arrival = 1, time.perf_counter()
    eng2.queue.extend([small3, big2])
    assert [r.id for r in eng2.admit()] == [0, 1]
    with pytest.raises(ValueError):
        ServingEngine(be, budget_fragments=1, policy="lifo")


def test_sjf_completes_every_request():
    be = FakeBackend(slots=2, delay=0.002)
    eng = ServingEngine(be, budget_fragments=10 * 32 * 32 * 3, max_batch=4, policy="sjf", age_ms=5.0)
    eng.start()
    futs = [eng.submit(req(16 if i % 3 else 32, 16 if i % 3 else 32)) for i in range(30)]
    assert sorted(f.result(timeout=10).request_id for f in futs) == list(range(30))
    eng.stop()


def test_priority_slot_takes_the_largest_request_alone():
    """With a high-priority slot the largest queued request goes there alone
    and the other slots take the rest in the engine's policy."""
    be = FakeBackend(slots=2, delay=0.05)
    be.priority_slots = 1
    eng = ServingEngine(be, budget_fragments=10 * 64 * 64 * 4, max_batch=8, policy="sjf", age_ms=1e6)
    reqs = [req(16, 16), req(64, 64), req(16, 16), req(32, 32)]
    for i, r in enumerate(reqs):
        r.id, r.t_arrival = i, time.perf_counter()
        eng.queue.append(r)
    eng.step()
    by_slot = dict(be.launched)
    assert by_slot[0] == [1]              # the 64 x 64 request, alone, on the priority slot
    assert sorted(by_slot[1]) == [0, 2, 3]
    eng.running = False
    while eng.busy:
        eng.step()
        time.sleep(0.005)


def test_batch_fragments_caps_the_batch_but_not_a_single_request():
    be = FakeBackend(slots=1, delay=0.0)
    eng = ServingEngine(be, budget_fragments=10 * 64 * 64 * 4, max_batch=8, batch_fragments=10 * 32 * 32 * 2)
    for i, r in enumerate([req(32, 32), req(32, 32), req(32, 32), req(64, 64)]):
        r.id, r.t_arrival = i, time.perf_counter()
        eng.queue.append(r)
    assert [r.id for r in eng.admit()] == [0, 1]   # two 32 x 32 fill the batch target
    assert [r.id for r in eng.admit()] == [2]      # the 64 x 64 would overflow it
    assert [r.id for r in eng.admit()] == [3]      # over the target, alone
