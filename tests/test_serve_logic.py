"""Host logic of the serving loop (pybrown_b200.serve) with a fake batch:
admission by memory footprint in arrival order, the concurrency cap, step
counts, latencies on the virtual clock, and the synthetic request stream.
No GPU."""
import math

import numpy as np
import pytest

from pybrown_b200.serve import Request, Server, make_stream, place_beads


class FakeBatch:
    def __init__(self):
        self.slots = {}
        self.next = 0
        self.steps = {}
        self.log = []  # membership at each step

    def footprint(self, n):
        return 1000 * n

    def add(self, positions, radii, box_length, **kw):
        s = self.next
        self.next += 1
        self.slots[s] = np.array(positions, float)
        self.steps[s] = 0
        return s

    def remove(self, s):
        del self.slots[s]

    def propagate(self, dt):
        self.log.append(sorted(self.slots))
        for s in self.slots:
            self.steps[s] += 1
            self.slots[s] = self.slots[s] + 1.0

    def positions(self, s):
        return self.slots[s]


def _req(rid, arrival, N, steps):
    return Request(rid, arrival, np.zeros((N, 3)), np.ones(N), 100.0, steps, seed=rid)


def test_every_request_runs_its_steps_and_completes():
    b = FakeBatch()
    reqs = [_req(0, 0.0, 10, 5), _req(1, 0.0015, 20, 3), _req(2, 0.01, 5, 7)]
    recs, summary = Server(b, memory_budget=10 ** 9).run(reqs, clock="virtual", tick=1e-3)
    assert [b.steps[s] for s in sorted(b.steps)] == [5, 3, 7]
    for r, rec in zip(reqs, recs):
        assert rec.completed > rec.arrival
        assert np.allclose(rec.positions, r.steps)  # the fake moves every bead by 1 per step
    assert summary["requests"] == 3
    assert summary["p99_ms"] >= summary["p50_ms"] > 0


def test_admission_respects_the_memory_budget_in_arrival_order():
    b = FakeBatch()
    # footprints 30k, 50k, 20k with a 60k budget: 0 runs, 1 waits (FIFO), 2 waits behind 1
    reqs = [_req(0, 0.0, 30, 4), _req(1, 0.0, 50, 2), _req(2, 0.0, 20, 2)]
    recs, summary = Server(b, memory_budget=60000).run(reqs, clock="virtual", tick=1e-3)
    assert summary["peak_bytes"] <= 60000
    # request 1 starts only after request 0 has finished
    assert recs[1].admitted >= recs[0].completed
    assert all(len(m) <= 2 for m in b.log)
    assert recs[2].admitted >= recs[1].admitted


def test_concurrency_cap_and_overlap():
    b = FakeBatch()
    reqs = [_req(k, 0.0, 5, 3 + k) for k in range(6)]
    _, summary = Server(b, memory_budget=10 ** 9, max_active=4).run(reqs, clock="virtual", tick=1e-3)
    assert summary["peak_active"] == 4
    assert max(len(m) for m in b.log) == 4
    # overlapping work: fewer batched steps than the sum of the step counts
    assert summary["batched_steps"] < sum(3 + k for k in range(6))


def test_latency_on_the_virtual_clock():
    b = FakeBatch()
    recs, _ = Server(b, memory_budget=10 ** 9).run([_req(0, 0.5, 4, 10)], clock="virtual", tick=2e-3)
    assert recs[0].admitted == pytest.approx(0.5)
    assert recs[0].latency == pytest.approx(10 * 2e-3)


def test_oversized_request_is_rejected():
    with pytest.raises(ValueError):
        Server(FakeBatch(), memory_budget=1000).run([_req(0, 0.0, 2, 1)], clock="virtual")


def test_stream_is_seeded_and_in_range():
    a = make_stream(3, rate=50, duration=0.5, n_max=64, steps_min=100, steps_max=200)
    b = make_stream(3, rate=50, duration=0.5, n_max=64, steps_min=100, steps_max=200)
    assert len(a) == len(b) > 5
    for x, y in zip(a, b):
        assert x.arrival == y.arrival and np.array_equal(x.positions, y.positions)
        assert 16 <= x.n_beads <= 64 and 100 <= x.steps <= 200
        assert np.all((x.radii >= 10) & (x.radii <= 40))
        assert 0 < x.arrival < 0.5
    arrivals = [x.arrival for x in a]
    assert arrivals == sorted(arrivals)


def test_placement_has_no_overlaps():
    rng = np.random.default_rng(0)
    radii = rng.uniform(10, 40, size=300)
    L = (np.sum(4 / 3 * np.pi * radii ** 3) / 0.05) ** (1 / 3)
    pos = place_beads(rng, radii, L)
    d = pos[:, None, :] - pos[None, :, :]
    d -= L * np.round(d / L)
    dist = np.sqrt((d ** 2).sum(-1))
    np.fill_diagonal(dist, math.inf)
    assert np.all(dist > radii[:, None] + radii[None, :])
    assert np.all(np.abs(pos) <= L / 2)


def test_fast_placement_has_no_overlaps_and_is_seeded():
    from pybrown_b200.serve import place_beads_fast
    radii = np.random.default_rng(1).uniform(10, 40, size=2048)
    L = (np.sum(4 / 3 * np.pi * radii ** 3) / 0.05) ** (1 / 3)
    pos = place_beads_fast(np.random.default_rng(2), radii, L)
    assert np.array_equal(pos, place_beads_fast(np.random.default_rng(2), radii, L))
    from scipy.spatial import cKDTree
    pairs = cKDTree(np.mod(pos + L / 2, L), boxsize=L).query_pairs(80.0, output_type="ndarray")
    d = pos[pairs[:, 0]] - pos[pairs[:, 1]]
    d -= L * np.round(d / L)
    assert np.all(np.sqrt((d ** 2).sum(1)) > radii[pairs[:, 0]] + radii[pairs[:, 1]])
    assert np.all(np.abs(pos) <= L / 2)


def test_lazy_stream_places_beads_on_first_use():
    a = make_stream(5, rate=50, duration=0.4, lazy=True)
    b = make_stream(5, rate=50, duration=0.4, lazy=True)
    assert all(r.positions is None for r in a)
    for x, y in zip(a, b):
        assert np.array_equal(x.materialize(), y.materialize())
        assert x.materialize().shape == (x.n_beads, 3)


def test_admission_window_and_drain_limit():
    """Admissions stop at stop_admission_at, the loop drain_limit later: the
    requests left are counted as backlog, latencies only over completed ones."""
    b = FakeBatch()
    # on the virtual clock a batched step is 1 ms; 1 runs from t=0 for 100 ms,
    # 2 arrives after the window, 3 waits behind the concurrency cap
    reqs = [_req(0, 0.0, 4, 5), _req(1, 0.0, 4, 100), _req(2, 0.05, 4, 5), _req(3, 0.001, 4, 3)]
    recs, summary = Server(b, memory_budget=10 ** 9, max_active=2).run(
        reqs, clock="virtual", tick=1e-3, stop_admission_at=0.02, drain_limit=0.03)
    assert summary["completed"] == 2  # 0 and 3
    assert summary["backlog_waiting"] == 1 and summary["backlog_running"] == 1
    assert not b.slots  # everything left the batch
    assert summary["p99_ms"] >= summary["p50_ms"] > 0
    assert summary["elapsed_s"] == pytest.approx(0.05, abs=2e-3)


def test_failed_factorisation_drops_only_that_request():
    class Fail(Exception):
        def __init__(self, slots):
            super().__init__("factorisation failed")
            self.slots = slots
            self.recheck = {s: 0 for s in slots}

    class FailingBatch(FakeBatch):
        def propagate(self, dt):
            super().propagate(dt)
            if len(self.log) == 3 and 1 in self.slots:
                raise Fail({1: 7})

    b = FailingBatch()
    reqs = [_req(0, 0.0, 4, 6), _req(1, 0.0, 4, 6), _req(2, 0.0, 4, 6)]
    recs, summary = Server(b, memory_budget=10 ** 9).run(reqs, clock="virtual", tick=1e-3)
    assert summary["failed"] == 1 and summary["completed"] == 2
    assert recs[1].failed == {"status": 7, "recheck": 0} and math.isnan(recs[1].completed)
    assert b.steps[0] == 6 and b.steps[2] == 6
    assert summary["failures"][0]["rid"] == 1


def test_smallest_work_policy_admits_the_cheapest_first():
    """With one request at a time, FIFO admits in arrival order and
    smallest_work in order of steps x (3N)^3 (ties by arrival)."""
    reqs = [_req(0, 0.0, 40, 4), _req(1, 0.0, 10, 6), _req(2, 0.0, 20, 2), _req(3, 0.0, 10, 6)]
    order = {}
    for policy in ("fifo", "smallest_work"):
        b = FakeBatch()
        server = Server(b, memory_budget=10 ** 9, max_active=1, policy=policy)
        recs, summary = server.run(reqs, clock="virtual", tick=1e-3)
        assert summary["completed"] == 4
        order[policy] = [r.rid for r in sorted(recs, key=lambda x: x.admitted)]
    assert order["fifo"] == [0, 1, 2, 3]
    # work: rid 2: 2 * 60^3 = 432000, rids 1 and 3: 6 * 30^3 = 162000, rid 0: 4 * 120^3
    assert order["smallest_work"] == [1, 3, 2, 0]


def test_unknown_policy_is_rejected():
    with pytest.raises(ValueError):
        Server(FakeBatch(), memory_budget=1, policy="random")
