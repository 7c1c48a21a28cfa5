"""Replica router of the serving layer (one process, several GPUs, every
request whole on one GPU) tested on the CPU with fake contexts and a fake
solve: slot and HBM-budget admission, the most-room placement rule, oversize
requests running alone, and failure handling (a GPU whose solve fails at the
CUDA level is taken out and the request is routed once more)."""
import threading
import time

import pytest

from hicma_parsec_b200 import serving, tlr


class FakeCtx:
    def __init__(self, device):
        self.device = device
        self.closed = False

    def close(self):
        self.closed = True


class FakeGPUs:
    """Solve stand-in: tracks in-flight requests and held bytes per device."""

    def __init__(self, budgets, fail_devices=(), sleep=0.01, raise_on_fail=False):
        self.lock = threading.Lock()
        self.inflight = {}
        self.max_inflight = {}
        self.held = {}
        self.max_held = {}
        self.alone_violations = 0
        self.budgets = budgets
        self.fail_devices = set(fail_devices)
        self.sleep = sleep
        self.raise_on_fail = raise_on_fail
        self.calls = []

    def footprint(self, req):
        return req.n

    def solve(self, ctx, req):
        d = ctx.device
        with self.lock:
            self.calls.append((req.rid, d))
            self.inflight[d] = self.inflight.get(d, 0) + 1
            self.max_inflight[d] = max(self.max_inflight.get(d, 0), self.inflight[d])
            self.held[d] = self.held.get(d, 0) + req.n
            self.max_held[d] = max(self.max_held.get(d, 0), self.held[d])
            if req.n > self.budgets[d] and self.inflight[d] > 1:
                self.alone_violations += 1
        time.sleep(self.sleep[d] if isinstance(self.sleep, dict) else self.sleep)
        with self.lock:
            self.inflight[d] -= 1
            self.held[d] -= req.n
        if d in self.fail_devices:
            if self.raise_on_fail:
                raise RuntimeError("device lost")
            return serving.MLEResult(rid=req.rid, n=req.n, status=tlr.ERR_CUDA, error="cuda failure")
        return serving.MLEResult(rid=req.rid, n=req.n, logdet=float(req.rid))


def reqs(sizes, spacing=0.0):
    return [serving.MLERequest(rid=i, kind=2, n=n, nb=10, beta=0.1, sigma=1.0, noise=1e-3, acc=1e-8, seed=i,
                               arrival=i * spacing) for i, n in enumerate(sizes)]


def router(budgets, gpus, slots=2):
    devs = list(range(len(budgets)))
    return serving.ReplicaRouter(devices=devs, slots=slots, hbm_budgets=budgets, make_context=FakeCtx,
                                 solve=gpus.solve, footprint=gpus.footprint)


def run_bounded(rt, rq, realtime=False, limit=60.0):
    out = {}
    th = threading.Thread(target=lambda: out.setdefault("res", rt.run(rq, realtime=realtime)), daemon=True)
    th.start()
    th.join(limit)
    assert not th.is_alive(), "router did not finish"
    return out["res"]


def test_every_request_served_once_within_slots_and_budgets():
    budgets = [200, 200, 200]
    g = FakeGPUs(budgets)
    rt = router(budgets, g, slots=2)
    res = run_bounded(rt, reqs([40 + (7 * i) % 50 for i in range(30)]))
    assert [r.rid for r in res] == list(range(30))
    assert all(r.status == 0 and r.logdet == r.rid for r in res)
    assert sorted(rid for rid, _ in g.calls) == list(range(30))
    assert set(r.device for r in res) == {0, 1, 2}
    assert max(g.max_inflight.values()) <= 2
    assert all(g.max_held[d] <= budgets[d] for d in g.max_held)
    rt.close()


def test_placement_prefers_the_most_room():
    budgets = [100, 1000]
    g = FakeGPUs(budgets, sleep={0: 0.6, 1: 0.1})
    rt = router(budgets, g, slots=1)
    res = run_bounded(rt, reqs([50, 50, 50]))
    # first to device 1 (950 left vs 50); device 1 then busy, so the second goes to device 0;
    # the third waits for a slot and again prefers device 1
    assert [r.device for r in res] == [1, 0, 1]


def test_oversize_requests_run_alone():
    budgets = [10]
    g = FakeGPUs(budgets, sleep=0.02)
    rt = router(budgets, g, slots=3)
    res = run_bounded(rt, reqs([50, 60, 70]))
    assert all(r.status == 0 for r in res)
    assert g.alone_violations == 0 and g.max_inflight[0] == 1
    order = sorted(res, key=lambda r: r.t_admit)
    for prev, nxt in zip(order, order[1:]):
        assert nxt.t_admit >= prev.t_done - 1e-3


@pytest.mark.parametrize("raise_on_fail", [False, True])
def test_failed_gpu_is_taken_out_and_requests_rerouted(raise_on_fail):
    budgets = [1000, 1000]
    g = FakeGPUs(budgets, fail_devices={0}, raise_on_fail=raise_on_fail)
    rt = router(budgets, g, slots=2)
    res = run_bounded(rt, reqs([10] * 12))
    assert all(r.status == 0 and r.device == 1 for r in res)
    assert rt.failed == {0}
    # at most the requests in flight on device 0 when it failed ran there
    assert sum(1 for _, d in g.calls if d == 0) <= 2
    rt.close()


def test_all_gpus_failing_ends_every_request_with_an_error():
    budgets = [1000, 1000]
    g = FakeGPUs(budgets, fail_devices={0, 1})
    rt = router(budgets, g, slots=1)
    res = run_bounded(rt, reqs([10] * 6))
    assert all(r.status == tlr.ERR_CUDA for r in res)
    assert rt.failed == {0, 1}
    assert len(g.calls) <= 4          # each device failed once per in-flight request, then no more work


def test_realtime_arrivals_and_single_gpu_server():
    g = FakeGPUs([100])
    srv = serving.MLEServer(0, slots=2, hbm_budget=100, make_context=FakeCtx, solve=g.solve,
                            footprint=g.footprint)
    rq = reqs([30, 30, 30, 30], spacing=0.02)
    res = run_bounded(srv, rq, realtime=True)
    assert all(r.status == 0 and r.device == 0 for r in res)
    for r, q in zip(res, rq):
        assert r.t_admit >= q.arrival - 1e-3 and r.latency > 0
    assert srv.hbm_budget == 100
    srv.close()


def test_a_gpu_that_cannot_start_is_left_out():
    budgets = [1000, 1000]
    g = FakeGPUs(budgets)

    def make(device):
        if device == 0:
            raise RuntimeError("out of memory")
        return FakeCtx(device)

    rt = serving.ReplicaRouter(devices=[0, 1], slots=2, hbm_budgets=budgets, make_context=make, solve=g.solve,
                               footprint=g.footprint)
    assert rt.failed == {0} and "out of memory" in rt.init_errors[0]
    res = run_bounded(rt, reqs([10] * 5))
    assert all(r.status == 0 and r.device == 1 for r in res)
    with pytest.raises(RuntimeError):
        serving.ReplicaRouter(devices=[0], slots=1, hbm_budgets=[10], make_context=make, solve=g.solve)
