"""The serving loop on the GPU: a request's result is the same alone and in a
mixed stream whose other requests arrive, run and leave around it, and the
memory budget limits what runs concurrently."""
import numpy as np
import pytest

from pybrown_b200.serve import Request, Server, place_beads

pytestmark = pytest.mark.gpu


def _request(rid, arrival, N, steps, seed):
    rng = np.random.default_rng(1000 + rid)
    radii = rng.uniform(10.0, 40.0, size=N)
    L = float((np.sum(4.0 / 3.0 * np.pi * radii ** 3) / 0.05) ** (1.0 / 3.0))
    return Request(rid, arrival, place_beads(rng, radii, L), radii, L, steps, seed)


def _serve(reqs, **kw):
    from pybrown_b200.batch import ReplicaBatch
    batch = ReplicaBatch(precision="mixed")
    try:
        recs, summary = Server(batch, memory_budget=kw.pop("memory_budget", 2 ** 34), **kw).run(
            reqs, clock="virtual", tick=1e-3)
    finally:
        batch.close()
    return {r.rid: r for r in recs}, summary


@pytest.mark.parametrize("policy", ["fifo", "smallest_work"])
def test_result_is_the_same_alone_and_in_the_mix(policy):
    """Under either admission policy (which only changes when a request runs
    and with whom)."""
    stream = [_request(0, 0.000, 60, 9, 11), _request(1, 0.002, 150, 4, 12), _request(2, 0.0035, 25, 12, 13),
              _request(3, 0.006, 90, 6, 14), _request(4, 0.0, 33, 2, 15)]
    mixed, summary = _serve(stream, policy=policy)
    assert summary["peak_active"] >= 3
    for r in stream:
        alone, _ = _serve([Request(r.rid, 0.0, r.positions, r.radii, r.box_length, r.steps, r.seed)])
        assert np.array_equal(alone[r.rid].positions, mixed[r.rid].positions), r.rid
        assert np.all(np.isfinite(mixed[r.rid].positions))
        assert not np.array_equal(mixed[r.rid].positions, r.positions)


def test_memory_budget_limits_concurrency():
    from pybrown_b200.batch import ReplicaBatch
    stream = [_request(k, 0.0, 64, 3, 20 + k) for k in range(5)]
    fp = ReplicaBatch(precision="mixed").footprint(64)
    recs, summary = _serve(stream, memory_budget=2 * fp + fp // 2)
    assert summary["peak_active"] == 2
    assert summary["peak_bytes"] <= 2 * fp + fp // 2
    assert all(np.isfinite(r.latency) for r in recs.values())
