"""Continuous-batching request loop: each request's result is the same alone and in the mix,
admission respects the device-memory budget, latencies are recorded."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("plain_above", [1 << 20, 14 ** 3])
def test_serving_results_same_alone_and_in_mix(plain_above):
    """All requests batched, and requests above 14^3 particles stepped as their own boxes."""
    import cosmictiger_b200 as ct
    from cosmictiger_b200 import serving

    ctx = ct.Context(order=7)
    reqs = serving.poisson_requests(5, rate=200.0, nmin=10, nmax=18, smin=1, smax=4, seed=3)
    states = {r.rid: serving.request_state(r) for r in reqs}
    # a budget that admits about two of these requests at a time
    budget = 2.2 * max(r.particles for r in reqs) * serving.BYTES_PER_PARTICLE
    srv = serving.Server(ctx, theta=0.55, hbm_budget=budget, plain_above=plain_above)
    done = srv.run(reqs, states)
    assert len(done) == len(reqs)
    assert srv.ticks < sum(r.steps for r in reqs)  # some ticks advanced several requests
    mixed = {r.rid: r.result for r in done}
    for r in reqs:
        assert r.latency is not None and r.latency >= 0
    alone = serving.poisson_requests(5, rate=200.0, nmin=10, nmax=18, smin=1, smax=4, seed=3)
    for r in alone:
        r.arrival = 0.0
        out = serving.run_sequential(ctx, [r], states)[0].result
        for f in ("x", "y", "z", "v", "rung"):
            assert np.array_equal(out[f], mixed[r.rid][f]), (r.rid, f)
    s = serving.summarize(done)
    assert s["p99_ms"] >= s["p50_ms"] > 0
    ctx.close()


def test_serving_two_lanes_results_same_alone_and_in_mix():
    """Two lanes (two contexts, two host threads, kernels of both on the device at once):
    every request's result is bit-identical to the request run alone."""
    import cosmictiger_b200 as ct
    from cosmictiger_b200 import serving

    lanes = [ct.Context(order=7), ct.Context(order=7)]
    reqs = serving.poisson_requests(8, rate=400.0, nmin=10, nmax=20, smin=1, smax=4, seed=7)
    states = {r.rid: serving.request_state(r) for r in reqs}
    srv = serving.Server(lanes, theta=0.55, hbm_budget=1e12, plain_above=14 ** 3)
    done = srv.run(reqs, states)
    assert len(done) == len(reqs)
    assert all(lane.ticks > 0 for lane in srv.lanes)
    mixed = {r.rid: r.result for r in done}
    alone = serving.poisson_requests(8, rate=400.0, nmin=10, nmax=20, smin=1, smax=4, seed=7)
    for r in alone:
        r.arrival = 0.0
        out = serving.run_sequential(lanes[0], [r], states)[0].result
        for f in ("x", "y", "z", "v", "rung"):
            assert np.array_equal(out[f], mixed[r.rid][f]), (r.rid, f)
    for c in lanes:
        c.close()
