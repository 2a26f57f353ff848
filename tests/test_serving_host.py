"""Host logic of the continuous-batching server, on a fake device context: every request
receives exactly its number of steps, its first step is flagged as the run's first call, and
admission keeps the resident particles within the memory budget."""
from cosmictiger_b200 import serving


class FakeBox:
    def __init__(self, n, log=None):
        self.n = n
        self.steps = 0
        self.closed = False
        self.log = log

    # a box stepped on its own (the server's plain path)
    def tree_create(self, *args):
        pass

    def kick(self, params):
        self.log.append((self.steps == 0) == bool(params.first_call))

    def drift(self, *args):
        self.steps += 1

    def upload(self, *state):
        self.steps = 0

    def download(self):
        return {"steps": self.steps}

    def close(self):
        self.closed = True


class FakeEnsemble:
    def __init__(self, counts, log, peak):
        self.slots = [0] * len(counts)
        self.first = None
        self.log = log
        self.ctx_peak = peak

    def set_box_params(self, h, gm):
        pass

    def reshape(self, counts):
        self.slots = [None] * len(counts)  # contents undefined until the next gather
        self.ctx_peak(counts)

    def gather(self, boxes):
        assert not any(b.closed for b in boxes)
        self.slots = [b.steps for b in boxes]

    def scatter(self, boxes):
        assert len(boxes) == len(self.slots)
        for b, s in zip(boxes, self.slots):
            b.steps = s

    def set_first_call(self, flags):
        self.first = list(flags)

    def tree_create(self, *args):
        pass

    def kick(self, params):
        for s, f in zip(self.slots, self.first):
            self.log.append((s == 0) == bool(f))

    def drift(self, *args):
        self.slots = [s + 1 for s in self.slots]

    def close(self):
        pass


class FakeContext:
    def __init__(self):
        self.log = []
        self.resident = 0
        self.peak = 0

    def box(self, n):
        return FakeBox(n, self.log)

    def note(self, counts):
        self.peak = max(self.peak, sum(counts))

    def ensemble(self, counts):
        self.note(counts)
        return FakeEnsemble(counts, self.log, self.note)

    def synchronize(self):
        pass

    def set_priority(self, p):
        self.priority = p


def test_server_steps_and_budget():
    reqs = serving.poisson_requests(40, rate=5000.0, nmin=8, nmax=20, smin=1, smax=9, seed=11)
    states = {r.rid: () for r in reqs}
    budget = 3.0 * max(r.particles for r in reqs) * serving.BYTES_PER_PARTICLE
    ctx = FakeContext()
    srv = serving.Server(ctx, hbm_budget=budget)
    done = srv.run(reqs, states)
    assert sorted(r.rid for r in done) == list(range(len(reqs)))
    for r in done:
        assert r.result["steps"] == r.steps, (r.rid, r.result, r.steps)
        assert r.done >= r.admitted >= r.arrival - 1e-9
    assert all(ctx.log) and len(ctx.log) == sum(r.steps for r in reqs)
    assert ctx.peak * serving.BYTES_PER_PARTICLE <= budget
    assert srv.ticks < sum(r.steps for r in reqs)


def test_server_plain_path_for_large_requests():
    """Requests above plain_above step as their own boxes in the same ticks as the batched
    ones: exact step counts and first-call flags for both kinds; the ensemble holds only the
    small ones."""
    reqs = serving.poisson_requests(40, rate=5000.0, nmin=8, nmax=20, smin=1, smax=9, seed=12)
    states = {r.rid: () for r in reqs}
    cut = 12 ** 3
    assert any(r.particles > cut for r in reqs) and any(r.particles <= cut for r in reqs)
    ctx = FakeContext()
    srv = serving.Server(ctx, hbm_budget=1e18, plain_above=cut)
    done = srv.run(reqs, states)
    assert sorted(r.rid for r in done) == list(range(len(reqs)))
    for r in done:
        assert r.result["steps"] == r.steps, (r.rid, r.result, r.steps)
    assert all(ctx.log) and len(ctx.log) == sum(r.steps for r in reqs)
    assert ctx.peak <= sum(r.particles for r in reqs if r.particles <= cut)


def test_server_lanes_share_the_work_and_keep_large_requests_in_order():
    """Two lanes (two contexts, two host threads): every request gets exactly its steps with
    the right first-call flags, both lanes step requests, no lane ever holds more than one
    large request, and large requests are admitted in arrival order."""
    reqs = serving.poisson_requests(60, rate=4000.0, nmin=8, nmax=20, smin=1, smax=9, seed=13)
    states = {r.rid: () for r in reqs}
    cut = 12 ** 3
    lanes = [FakeContext(), FakeContext()]
    srv = serving.Server(lanes, hbm_budget=1e18, plain_above=cut)
    big_live = {id(c): 0 for c in lanes}
    worst = {id(c): 0 for c in lanes}
    for c in lanes:
        orig = c.box

        def box(n, c=c, orig=orig):
            b = orig(n)
            if n > cut:
                big_live[id(c)] += 1
                worst[id(c)] = max(worst[id(c)], big_live[id(c)])
                close = b.close

                def closing(close=close, c=c):
                    big_live[id(c)] -= 1
                    close()
                b.close = closing
            return b
        c.box = box
    done = srv.run(reqs, states)
    assert sorted(r.rid for r in done) == list(range(len(reqs)))
    for r in done:
        assert r.result["steps"] == r.steps, (r.rid, r.result, r.steps)
    for c in lanes:
        assert all(c.log)
    assert sum(len(c.log) for c in lanes) == sum(r.steps for r in reqs)
    assert all(lane.ticks > 0 for lane in srv.lanes)
    assert max(worst.values()) == 1
    big = sorted((r for r in done if r.particles > cut), key=lambda r: r.arrival)
    assert [r.admitted for r in big] == sorted(r.admitted for r in big)


def test_server_lane_error_reaches_the_caller_and_closes_ensembles():
    """A step that raises in a lane's thread ends the run with that exception; every lane's
    ensemble is closed."""
    reqs = serving.poisson_requests(20, rate=4000.0, nmin=8, nmax=10, smin=2, smax=5, seed=14)
    states = {r.rid: () for r in reqs}
    lanes = [FakeContext(), FakeContext()]
    closed = []

    def failing(c):
        def ensemble(counts):
            e = FakeEnsemble(counts, c.log, c.note)

            def kick(params):
                raise RuntimeError("device step failed")
            e.kick = kick
            e.close = lambda: closed.append(1)
            return e
        return ensemble
    for c in lanes:
        c.ensemble = failing(c)
    srv = serving.Server(lanes, hbm_budget=1e18)
    try:
        srv.run(reqs, states)
        raise AssertionError("the lane's exception was not raised")
    except RuntimeError as e:
        assert "device step failed" in str(e)
    assert all(lane.ens is None for lane in srv.lanes)
    assert closed


def test_lane_with_the_oldest_request_gets_the_high_priority():
    """The lane holding the oldest active request (earliest arrival) asks for the high stream
    priority, every other lane for the default; a single lane never changes priority."""
    lanes = [FakeContext(), FakeContext(), FakeContext()]
    srv = serving.Server(lanes, hbm_budget=1e18)
    reqs = serving.poisson_requests(5, rate=10.0, nmin=8, nmax=10, seed=15)
    a, b, c = srv.lanes
    a.active = [[reqs[3], None, 1]]
    b.active = [[reqs[1], None, 1], [reqs[4], None, 1]]
    c.active = []
    assert srv._wanted_priority(b) == serving.Server.HIGH_PRIORITY
    assert srv._wanted_priority(a) == 0
    assert srv._wanted_priority(c) == 0
    b.active = [[reqs[4], None, 1]]
    assert srv._wanted_priority(a) == serving.Server.HIGH_PRIORITY
    one = serving.Server(FakeContext(), hbm_budget=1e18)
    one.lanes[0].active = [[reqs[0], None, 1]]
    assert one._wanted_priority(one.lanes[0]) == 0


def test_big_total_runs_large_requests_one_at_a_time_in_arrival_order():
    """big_total=1 over two lanes: never two large requests resident at once, large requests
    admitted in arrival order, every request stepped exactly its number of times."""
    import threading

    reqs = serving.poisson_requests(50, rate=4000.0, nmin=8, nmax=20, smin=1, smax=6, seed=16)
    states = {r.rid: () for r in reqs}
    cut = 12 ** 3
    lanes = [FakeContext(), FakeContext()]
    live = [0]
    worst = [0]
    lock = threading.Lock()
    for c in lanes:
        orig = c.box

        def box(n, orig=orig):
            b = orig(n)
            if n > cut:
                with lock:
                    live[0] += 1
                    worst[0] = max(worst[0], live[0])
                close = b.close

                def closing(close=close):
                    with lock:
                        live[0] -= 1
                    close()
                b.close = closing
            return b
        c.box = box
    srv = serving.Server(lanes, hbm_budget=1e18, plain_above=cut, big_total=1)
    done = srv.run(reqs, states)
    assert sorted(r.rid for r in done) == list(range(len(reqs)))
    for r in done:
        assert r.result["steps"] == r.steps
    assert worst[0] == 1
    big = sorted((r for r in done if r.particles > cut), key=lambda r: r.arrival)
    assert len(big) > 2
    assert [r.admitted for r in big] == sorted(r.admitted for r in big)
    assert srv.big_active == 0 and all(lane.big == 0 for lane in srv.lanes)
