"""Continuous-batching request loop for gravity-step requests.

A request asks for `steps` gravity steps (tree build + kick + drift, all particles active) of
its own periodic box of n^3 particles.  The server keeps every admitted request's particles
resident on the device between steps, admits waiting requests while the device-memory
budget allows, and advances the active requests in ticks: each tick of a lane gathers its
small boxes into one ensemble (one set of kernel launches for all of them, ct_ensemble_*),
steps its large boxes on their own, and retires requests whose steps are done.  Several lanes
(device contexts with their own streams, each driven by its own host thread) run their ticks
independently, so that one lane's uploads, host round trips and kernel tails overlap another
lane's kernels.  Requests that arrive while a tick runs join at a later tick.  Results do not
depend on the mix: boxes of an ensemble never interact, every kernel treats them
independently and contexts share no device state that a step writes, so a request's result
is bit-identical alone and batched with others.

The reference has no serving layer; this one admits requests by a device-memory budget,
keeps their state resident on the device between steps and reports p50/p99 latency.
"""
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import KickParams, ics

# device bytes per particle while resident and stepping: particle state (41), tree nodes and
# multipoles (~12), interaction lists and expansions (~40), P2P scratch (16), with headroom
BYTES_PER_PARTICLE = 160


@dataclass
class Request:
    rid: int
    n: int                    # particles per side
    steps: int
    arrival: float            # seconds from the start of the run
    seed: int = 0
    index: float = -2.0       # Zel'dovich spectral index
    rms: float = 0.25         # RMS displacement in mean spacings
    # filled by the server
    admitted: float = None
    done: float = None
    result: dict = field(default=None, repr=False)

    @property
    def particles(self):
        return self.n ** 3

    @property
    def latency(self):
        return None if self.done is None else self.done - self.arrival


def request_state(req):
    """Seeded initial particles of a request (host arrays)."""
    return ics.zeldovich_lattice(req.n, index=req.index, rms_spacing=req.rms, seed=req.seed)


class _Lane:
    """One device context driven by its own host thread: its active requests and its ensemble."""

    def __init__(self, ctx):
        self.ctx = ctx
        self.active = []      # [[request, box, remaining steps]]
        self.ens = None
        self.ens_members = None
        self.ens_boxes = []
        self.ens_dirty = False  # the ensemble holds state newer than its member boxes
        self.hmax = 0.0
        self.ticks = 0
        self.priority = 0     # CUDA stream priority of the lane's context (0 default)
        self.big = 0          # large requests admitted to this lane and not yet retired (under the server's lock)


class Server:
    """Continuous batching over one or more lanes.  A lane is a device context (its own CUDA
    stream) driven by its own host thread; the library releases the interpreter lock while it
    works, so the lanes' uploads, kernels and host round trips overlap on the device.  Within a
    lane, requests of at most `plain_above` particles advance together as one ensemble per
    tick and larger ones advance as their own boxes in the same tick (batching gains little for
    them and would cost a re-batch whenever membership changes).  A lane holds at most
    `big_per_lane` large requests at a time, so that large requests start in arrival order
    across the lanes (first come, first served, as many at once as there are lanes) while
    small ones join whichever lane takes them first; `big_total` caps the large requests active
    at once over all lanes (1: large requests run one at a time, first come first served, while
    the other lanes step small requests beside them).  With several lanes, the lane that holds the
    oldest active request runs its streams at the device's highest priority and the others at
    the default: the oldest request's kernels take the SMs first and the others fill what it
    leaves idle (host round trips, kernel tails), so that overlapping requests add throughput
    without stretching the request that started first.  Admission keeps the resident particles
    of all lanes within `hbm_budget` (a request is admitted regardless when nothing is
    resident)."""

    HIGH_PRIORITY = -100  # clamped by the library to the device's highest stream priority

    def __init__(self, ctx, theta=0.55, hbm_budget=150e9, t0=1.0 / 64, bucket=128, plain_above=1 << 20, big_per_lane=1, big_total=None):
        ctxs = list(ctx) if isinstance(ctx, (list, tuple)) else [ctx]
        if not ctxs:
            raise ValueError("a server needs at least one context")
        if big_per_lane < 1:
            raise ValueError("big_per_lane must be at least 1")
        if big_total is not None and big_total < 1:
            raise ValueError("big_total must be at least 1")
        self.lanes = [_Lane(c) for c in ctxs]
        self.ctx = ctxs[0]
        self.plain_above = plain_above
        self.big_per_lane = big_per_lane
        self.big_total = big_total  # large requests active at once over all lanes (None: lanes x big_per_lane)
        self.theta = theta
        self.budget = hbm_budget
        self.t0 = t0
        self.bucket = bucket
        self.waiting = []
        self.finished = []
        self.reserved = 0     # device bytes of the requests admitted and not yet retired
        self.big_active = 0   # large requests admitted and not yet retired, all lanes
        self.lock = threading.Lock()
        self.particle_steps = 0
        self.error = None

    @property
    def ticks(self):
        return sum(lane.ticks for lane in self.lanes)

    def _bytes(self, req):
        return req.particles * BYTES_PER_PARTICLE

    def _big(self, req):
        return req.particles > self.plain_above

    def _take(self, lane):
        """Under the lock: the waiting requests this lane admits now, in arrival order."""
        cap_all = self.big_total if self.big_total is not None else len(self.lanes) * self.big_per_lane
        take = []
        for req in list(self.waiting):
            if self._big(req) and (lane.big >= self.big_per_lane or self.big_active >= cap_all):
                continue
            if self.reserved + self._bytes(req) <= self.budget or self.reserved == 0:
                self.reserved += self._bytes(req)
                self.waiting.remove(req)
                take.append(req)
                if self._big(req):
                    lane.big += 1
                    self.big_active += 1
        return take

    def _wanted_priority(self, lane):
        """Under the lock: the stream priority this lane should run at."""
        if len(self.lanes) == 1 or not lane.active:
            return 0
        # snapshots: another lane's thread may be adding to or retiring from its list
        oldest = min((it[0].arrival, it[0].rid) for ln in self.lanes for it in list(ln.active))
        return self.HIGH_PRIORITY if any((it[0].arrival, it[0].rid) == oldest for it in list(lane.active)) else 0

    def _admit(self, lane, reqs, now, states):
        for req in reqs:
            box = lane.ctx.box(req.particles)
            box.upload(*states[req.rid])
            req.admitted = now
            lane.active.append([req, box, req.steps])

    def _ensemble(self, lane, batched):
        members = [r.rid for r, _, _ in batched]
        if members != lane.ens_members:
            counts = [r.particles for r, _, _ in batched]
            if lane.ens is None:
                lane.ens = lane.ctx.ensemble(counts)
            else:
                if lane.ens_dirty:
                    # members still running keep their advanced state across the re-batch
                    lane.ens.scatter(lane.ens_boxes)
                # one ensemble per lane for the whole run, re-batched in place (device arrays reused)
                lane.ens.reshape(counts)
            h = np.array([ics.softening(c, 0.02) for c in counts], np.float32)
            gm = np.array([1.0 / c for c in counts], np.float32)
            lane.ens.set_box_params(h, gm)
            lane.ens_boxes = [b for _, b, _ in batched]
            lane.ens.gather(lane.ens_boxes)
            lane.ens_dirty = False
            lane.ens_members = members
            lane.hmax = float(h.max())
        return lane.ens

    def _tick(self, lane, now_fn):
        """One step of every active request of the lane; retire the finished ones."""
        batched = [it for it in lane.active if not self._big(it[0])]
        if batched:
            ens = self._ensemble(lane, batched)
            # a request's first step is its run's first call (no ascending half kick)
            ens.set_first_call([int(rem == r.steps) for r, _, rem in batched])
            ens.tree_create(self.theta, lane.hmax, self.bucket)
            ens.kick(KickParams.make(theta=self.theta, h=lane.hmax, GM=1.0, eta=ics.eta_default(), t0=self.t0, first_call=False, save_force=False))
            ens.drift(0, 1.0, self.t0)
            lane.ens_dirty = True
        for req, box, rem in lane.active:
            if self._big(req):
                # the plain path, exactly as run_sequential steps a request
                h = ics.softening(req.particles, 0.02)
                box.tree_create(self.theta, h, self.bucket)
                box.kick(KickParams.make(theta=self.theta, h=h, GM=1.0 / req.particles, eta=ics.eta_default(), t0=self.t0, first_call=rem == req.steps,
                                         save_force=False))
                box.drift(0, 1.0, self.t0)
        lane.ticks += 1
        done = []
        stepped = 0
        for item in lane.active:
            item[2] -= 1
            stepped += item[0].particles
            if item[2] == 0:
                done.append(item)
        if done:
            # bring the batched boxes' state back, then retire the finished requests
            if any(not self._big(it[0]) for it in done):
                lane.ens.scatter(lane.ens_boxes)
                lane.ens_dirty = False
                lane.ens_members = None  # membership changes
            lane.ctx.synchronize()
            t = now_fn()
            for item in done:
                req, box, _ = item
                req.result = box.download()
                req.done = t
                box.close()
                lane.active.remove(item)
        with self.lock:
            self.particle_steps += stepped
            for req, _, _ in done:
                self.reserved -= self._bytes(req)
                if self._big(req):
                    lane.big -= 1
                    self.big_active -= 1
                self.finished.append(req)

    def run(self, requests, states, clock=time.perf_counter):
        """Serve an open-loop arrival sequence in real time; returns the finished requests."""
        pending = sorted(requests, key=lambda r: r.arrival)
        t_start = clock()
        now = lambda: clock() - t_start  # noqa: E731

        def lane_loop(lane):
            while self.error is None:
                t = now()
                with self.lock:
                    while pending and pending[0].arrival <= t:
                        self.waiting.append(pending.pop(0))
                    take = self._take(lane)
                    if not take and not lane.active and not pending and not self.waiting:
                        return
                    next_arrival = pending[0].arrival if pending else None
                self._admit(lane, take, t, states)
                if lane.active:
                    with self.lock:
                        want = self._wanted_priority(lane)
                    if want != lane.priority:
                        lane.ctx.set_priority(want)
                        lane.priority = want
                    self._tick(lane, now)
                else:
                    wait = 0.002 if next_arrival is None else next_arrival - now()
                    time.sleep(max(0.0, min(0.002, wait)))

        def guarded(lane):
            try:
                lane_loop(lane)
            except BaseException as e:  # noqa: BLE001 - handed to the caller after the join
                with self.lock:
                    if self.error is None:
                        self.error = e

        try:
            if len(self.lanes) == 1:
                guarded(self.lanes[0])
            else:
                threads = [threading.Thread(target=guarded, args=(lane,), daemon=True) for lane in self.lanes]
                for th in threads:
                    th.start()
                for th in threads:
                    th.join()
            if self.error is not None:
                raise self.error
        finally:
            # also when a step raises: the ensembles' device arrays go back to their contexts
            for lane in self.lanes:
                if lane.ens is not None:
                    lane.ens.close()
                    lane.ens = None
        return self.finished


def run_sequential(ctx, requests, states, theta=0.55, t0=1.0 / 64, clock=time.perf_counter):
    """The plain path, one request at a time in arrival order (FIFO, no batching)."""
    pending = sorted(requests, key=lambda r: r.arrival)
    t_start = clock()
    out = []
    for req in pending:
        while clock() - t_start < req.arrival:
            time.sleep(max(0.0, min(0.01, req.arrival - (clock() - t_start))))
        box = ctx.box(req.particles)
        box.upload(*states[req.rid])
        h = ics.softening(req.particles, 0.02)
        for s in range(req.steps):
            box.tree_create(theta, h, 128)
            box.kick(KickParams.make(theta=theta, h=h, GM=1.0 / req.particles, eta=ics.eta_default(), t0=t0, first_call=s == 0, save_force=False))
            box.drift(0, 1.0, t0)
        ctx.synchronize()
        req.result = box.download()
        req.done = clock() - t_start
        box.close()
        out.append(req)
    return out


def poisson_requests(count, rate, nmin, nmax, smin=1, smax=16, seed=5):
    """Open-loop Poisson arrivals: exponential gaps at `rate` per second; n log-uniform in
    [nmin, nmax]; steps uniform in [smin, smax]; Zel'dovich parameters as the ensemble
    generator (index uniform in [-2.5, -1], RMS uniform in 0.1-0.6 spacings)."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, count)) if rate > 0 else np.zeros(count)
    ns = np.rint(np.exp(rng.uniform(np.log(nmin), np.log(nmax), count))).astype(int)
    steps = rng.integers(smin, smax + 1, count)
    idx = rng.uniform(-2.5, -1.0, count)
    rms = rng.uniform(0.1, 0.6, count)
    return [Request(rid=i, n=int(ns[i]), steps=int(steps[i]), arrival=float(t[i]), seed=int(seed * 7919 + i), index=float(idx[i]), rms=float(rms[i]))
            for i in range(count)]


def summarize(reqs):
    lat = np.array([r.latency for r in reqs])
    ps = sum(r.particles * r.steps for r in reqs)
    span = max(r.done for r in reqs) - min(r.arrival for r in reqs)
    return {"requests": len(reqs), "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "particle_steps_s": ps / span if span > 0 else None, "makespan_s": span}
