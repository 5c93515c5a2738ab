"""The native request loop (lbx_server_*, include/lbx_server.h) on the CPU: the loop is driven by
a host-side fake engine through lbx_server_create_with_engine, so admission by footprint,
first-fit queueing, retirement, the adaptive chunk, cancellation, rejection and error
propagation are checked without a GPU.  The fake engine gives each request a footprint of its
cell count and makes it converge once it has taken `core[0] * 10` steps (checked at run ends),
and records every run it is asked for.
"""
from __future__ import annotations

import ctypes as C
import math
import threading
import time

import pytest

from openlb_b200 import lbx


class FakeEngine:
    def __init__(self, capacity: int, slots: int = 16, fail_after_runs: int | None = None):
        self.capacity = capacity
        self.slots = [None] * slots
        self.used = 0
        self.peak = 0
        self.runs: list[int] = []
        self.fail_after_runs = fail_after_runs
        self.admits = 0
        self.engine = lbx.ServerEngine(lbx.ENGINE_ADMIT(self._admit), lbx.ENGINE_RUN(self._run),
                                       lbx.ENGINE_STATUSES(self._statuses), lbx.ENGINE_RETIRE(self._retire),
                                       slots, 0)

    @staticmethod
    def cells(req) -> int:
        return int(req.core[0]) * int(req.core[1]) * int(req.core[2])

    def _admit(self, _ctx, req_p, slot_p):
        req = req_p.contents
        if req.core[0] <= 0:
            return -1  # invalid request: rejected
        n = self.cells(req)
        if n > self.capacity:
            return -5  # would never fit; the loop finds that out with an empty engine
        if self.used + n > self.capacity or None not in self.slots:
            return -5
        i = self.slots.index(None)
        self.slots[i] = {"cells": n, "steps": 0, "target": int(req.core[0]) * 10, "cap": int(req.max_steps),
                         "state": lbx.SLOT_RUNNING}
        self.used += n
        self.peak = max(self.peak, self.used)
        self.admits += 1
        slot_p[0] = i
        return 0

    def _run(self, _ctx, steps):
        self.runs.append(steps)
        if self.fail_after_runs is not None and len(self.runs) > self.fail_after_runs:
            return -3
        for s in self.slots:
            if s is None or s["state"] != lbx.SLOT_RUNNING:
                continue
            s["steps"] += steps
            if s["steps"] >= s["target"]:
                s["state"] = lbx.SLOT_CONVERGED
            elif s["steps"] >= s["cap"]:
                s["state"] = lbx.SLOT_MAX_STEPS
        time.sleep(0.0005)
        return 0

    def _statuses(self, _ctx, out, n):
        for i in range(n):
            s = self.slots[i] if i < len(self.slots) else None
            out[i].state = 0 if s is None else s["state"]
            out[i].steps = 0 if s is None else s["steps"]
            out[i].residual = 0.0 if s is None else (1e-7 if s["state"] == lbx.SLOT_CONVERGED else 1e-3)
        return 0

    def _retire(self, _ctx, slot):
        s = self.slots[slot]
        if s is None:
            return -1
        self.used -= s["cells"]
        self.slots[slot] = None
        return 0


def _req(edge: int, max_steps: int = 10 ** 6):
    return lbx.make_request((edge, edge, edge), 1.2, 0.05, 1e-6, max_steps)


def _serve(fake, reqs, realtime=False, min_chunk=10, max_chunk=50, cancel=None):
    with lbx.Server(fake.engine, min_chunk, max_chunk, realtime) as srv:
        srv.submit(reqs)
        srv.start()
        if cancel:
            cancel(srv)
        srv.close()
        assert srv.wait(timeout=30.0)
        return srv.records(), srv.stats()


def test_every_request_is_served_under_memory_pressure_with_first_fit():
    fake = FakeEngine(capacity=3 * 8 ** 3)
    edges = [8, 4, 8, 8, 4, 6, 8, 4, 5, 8]
    reqs = [(i, 0.001 * i, _req(e)) for i, e in enumerate(edges)]
    recs, stats = _serve(fake, reqs)
    assert sorted(r["id"] for r in recs) == list(range(len(edges)))
    assert all(r["state"] == lbx.SLOT_CONVERGED for r in recs)
    assert fake.peak <= fake.capacity and fake.used == 0
    by = {r["id"]: r for r in recs}
    for i, e in enumerate(edges):
        r = by[i]
        assert r["cells"] == e ** 3
        assert r["steps"] >= e * 10
        assert r["arrival"] <= r["admitted"] <= r["finished"]
    # first fit: the 4^3 request 4 arrived behind three 8^3 ones and the slab held three
    # 8^3 cavities, so it may not wait for all of them to finish
    assert by[4]["admitted"] < by[3]["finished"] or by[4]["admitted"] <= by[1]["finished"]
    assert stats["submitted"] == len(edges) and stats["finished"] == len(edges)
    assert stats["runs"] == len(fake.runs) and stats["steps"] == sum(fake.runs)


def test_chunk_is_short_while_requests_wait_and_long_otherwise():
    fake = FakeEngine(capacity=8 ** 3)
    # one 8^3 at a time: while one runs, the others wait for memory -> short runs
    reqs = [(i, 0.0, _req(8)) for i in range(3)]
    recs, stats = _serve(fake, reqs, min_chunk=10, max_chunk=40)
    assert len(recs) == 3
    assert set(fake.runs) <= {10, 40}
    # the last request runs alone with nothing waiting or due: long runs only
    n_last = math.ceil(80 / 40)
    assert fake.runs[-n_last:] == [40] * n_last
    assert 10 in fake.runs
    assert stats["short_runs"] + stats["long_runs"] == stats["runs"]


def test_oversized_and_invalid_requests_are_rejected_and_the_rest_served():
    fake = FakeEngine(capacity=10 ** 3)
    reqs = [(0, 0.0, _req(6)), (1, 0.0, _req(12)), (2, 0.0, _req(5)), (3, 0.0, _req(0))]
    recs, _ = _serve(fake, reqs)
    by = {r["id"]: r for r in recs}
    assert by[0]["state"] == by[2]["state"] == lbx.SLOT_CONVERGED
    assert by[1]["state"] == lbx.SERVER_REJECTED and math.isnan(by[1]["admitted"])
    assert by[3]["state"] == lbx.SERVER_REJECTED and by[3]["slot"] == -1


def test_cancel_waiting_and_running_requests():
    fake = FakeEngine(capacity=8 ** 3)
    reqs = [(0, 0.0, _req(8)), (1, 0.0, _req(8)), (2, 0.0, _req(8))]

    def cancel(srv):
        # wait until request 0 runs, then cancel it (running) and request 2 (waiting)
        for _ in range(2000):
            if srv.stats()["running"] >= 1:
                break
            time.sleep(0.001)
        srv.cancel(0)
        srv.cancel(2)
        with pytest.raises(lbx.LbxError):
            srv.cancel(99)

    recs, _ = _serve(fake, reqs, realtime=True, cancel=cancel)
    by = {r["id"]: r for r in recs}
    assert by[0]["state"] == lbx.SERVER_CANCELLED and by[0]["slot"] >= 0
    assert by[2]["state"] == lbx.SERVER_CANCELLED
    assert by[1]["state"] == lbx.SLOT_CONVERGED
    assert fake.used == 0


def test_engine_error_stops_the_loop_and_is_reported():
    fake = FakeEngine(capacity=8 ** 3, fail_after_runs=2)
    with lbx.Server(fake.engine, 10, 10, False) as srv:
        srv.submit([(0, 0.0, _req(8))])
        srv.start()
        srv.close()
        with pytest.raises(lbx.LbxError, match="engine run failed"):
            srv.wait(timeout=30.0)
    assert fake.used == 0  # the admitted slot was retired on the way out


def test_submissions_from_another_thread_while_the_loop_runs():
    fake = FakeEngine(capacity=4 * 6 ** 3)
    with lbx.Server(fake.engine, 10, 40, True) as srv:
        srv.start()

        def producer(base):
            for k in range(10):
                srv.submit([(base + k, -1.0, _req(4 + k % 3))])
                time.sleep(0.001)

        ths = [threading.Thread(target=producer, args=(100 * t,)) for t in range(3)]
        for t in ths:
            t.start()
        for t in ths:
            t.join()
        srv.close()
        with pytest.raises(lbx.LbxError):
            srv.submit([(999, -1.0, _req(4))])
        assert srv.wait(timeout=30.0)
        recs = srv.records()
    assert len(recs) == 30 and len({r["id"] for r in recs}) == 30
    assert all(r["state"] == lbx.SLOT_CONVERGED for r in recs)
    assert all(r["arrival"] <= r["admitted"] <= r["finished"] for r in recs)


def test_virtual_clock_jumps_idle_gaps():
    fake = FakeEngine(capacity=8 ** 3)
    reqs = [(0, 0.0, _req(4)), (1, 1000.0, _req(4))]
    t0 = time.perf_counter()
    recs, stats = _serve(fake, reqs)
    assert time.perf_counter() - t0 < 10.0
    by = {r["id"]: r for r in recs}
    assert by[1]["admitted"] >= 1000.0
    assert stats["clock"] >= 1000.0


def test_bad_configuration_is_refused():
    fake = FakeEngine(capacity=10)
    cfg = lbx.ServerConfig(0, 10, 0, 0)
    h = C.c_void_p()
    assert lbx.lib.lbx_server_create_with_engine(C.byref(fake.engine), None, C.byref(cfg), C.byref(h)) == -1
    cfg = lbx.ServerConfig(20, 10, 0, 0)
    assert lbx.lib.lbx_server_create_with_engine(C.byref(fake.engine), None, C.byref(cfg), C.byref(h)) == -1
