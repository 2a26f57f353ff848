"""Continuous-batching request loop for gravity-step requests.

A request asks for `steps` gravity steps (tree build + kick + drift, all particles active) of
its own periodic box of n^3 particles.  The server keeps every admitted request's particles
resident on the device between steps, admits waiting requests while the device-memory
budget allows, and advances all active requests together: each tick gathers the active boxes
into one ensemble (one set of kernel launches for all of them, ct_ensemble_*), runs one step,
and retires requests whose steps are done.  Requests that arrive while a tick runs join at
the next tick.  Results do not depend on the mix: boxes of an ensemble never interact and
every kernel treats them independently, so a request's result is bit-identical alone and
batched with others.

The reference has no serving layer; this one admits requests by a device-memory budget,
keeps their state resident on the device between steps and reports p50/p99 latency.
"""
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


class Server:
    """Continuous batching.  Requests of at most `plain_above` particles advance together as one
    ensemble per tick; larger ones advance as their own boxes in the same tick (batching gains
    little for them and would cost a re-batch whenever membership changes)."""

    def __init__(self, ctx, theta=0.55, hbm_budget=150e9, t0=1.0 / 64, bucket=128, plain_above=1 << 20):
        self.ctx = ctx
        self.plain_above = plain_above
        self.theta = theta
        self.budget = hbm_budget
        self.t0 = t0
        self.bucket = bucket
        self.active = []      # [(request, box, remaining steps)]
        self.waiting = []
        self.finished = []
        self.ens = None
        self.ens_members = None
        self.ens_boxes = []
        self.ens_dirty = False  # the ensemble holds state newer than its member boxes
        self.ticks = 0
        self.particle_steps = 0

    def _bytes(self, req):
        return req.particles * BYTES_PER_PARTICLE

    def _in_use(self):
        return sum(self._bytes(r) for r, _, _ in self.active)

    def admit(self, now, states):
        """Admit waiting requests in arrival order while the budget allows."""
        keep = []
        for req in self.waiting:
            if self._in_use() + self._bytes(req) <= self.budget or not self.active:
                box = self.ctx.box(req.particles)
                box.upload(*states[req.rid])
                req.admitted = now
                self.active.append([req, box, req.steps])
            else:
                keep.append(req)
        self.waiting = keep

    def _batched(self, item):
        return item[0].particles <= self.plain_above

    def _ensemble(self, batched):
        members = [r.rid for r, _, _ in batched]
        if members != self.ens_members:
            counts = [r.particles for r, _, _ in batched]
            if self.ens is None:
                self.ens = self.ctx.ensemble(counts)
            else:
                if self.ens_dirty:
                    # members still running keep their advanced state across the re-batch
                    self.ens.scatter(self.ens_boxes)
                # one ensemble for the whole run, re-batched in place (device arrays reused)
                self.ens.reshape(counts)
            h = np.array([ics.softening(c, 0.02) for c in counts], np.float32)
            gm = np.array([1.0 / c for c in counts], np.float32)
            self.ens.set_box_params(h, gm)
            self.ens_boxes = [b for _, b, _ in batched]
            self.ens.gather(self.ens_boxes)
            self.ens_dirty = False
            self.ens_members = members
            self.hmax = float(h.max())
        return self.ens

    def tick(self, now_fn):
        """One step of every active request; retire the finished ones."""
        batched = [it for it in self.active if self._batched(it)]
        if batched:
            ens = self._ensemble(batched)
            # a request's first step is its run's first call (no ascending half kick)
            ens.set_first_call([int(rem == r.steps) for r, _, rem in batched])
            ens.tree_create(self.theta, self.hmax, self.bucket)
            ens.kick(KickParams.make(theta=self.theta, h=self.hmax, GM=1.0, eta=ics.eta_default(), t0=self.t0, first_call=False, save_force=False))
            ens.drift(0, 1.0, self.t0)
            self.ens_dirty = True
        for req, box, rem in self.active:
            if req.particles > self.plain_above:
                # the plain path, exactly as run_sequential steps a request
                h = ics.softening(req.particles, 0.02)
                box.tree_create(self.theta, h, self.bucket)
                box.kick(KickParams.make(theta=self.theta, h=h, GM=1.0 / req.particles, eta=ics.eta_default(), t0=self.t0, first_call=rem == req.steps,
                                         save_force=False))
                box.drift(0, 1.0, self.t0)
        self.ticks += 1
        done = []
        for item in self.active:
            item[2] -= 1
            self.particle_steps += item[0].particles
            if item[2] == 0:
                done.append(item)
        if done:
            # bring the batched boxes' state back, then retire the finished requests
            if any(self._batched(it) for it in done):
                self.ens.scatter(self.ens_boxes)
                self.ens_dirty = False
                self.ens_members = None  # membership changes
            self.ctx.synchronize()
            t = now_fn()
            for item in done:
                req, box, _ = item
                req.result = box.download()
                req.done = t
                box.close()
                self.active.remove(item)
                self.finished.append(req)

    def run(self, requests, states, clock=time.perf_counter):
        """Serve an open-loop arrival sequence in real time; returns the finished requests."""
        pending = sorted(requests, key=lambda r: r.arrival)
        t_start = clock()
        now = lambda: clock() - t_start  # noqa: E731
        try:
            while pending or self.waiting or self.active:
                t = now()
                while pending and pending[0].arrival <= t:
                    self.waiting.append(pending.pop(0))
                self.admit(t, states)
                if self.active:
                    self.tick(now)
                elif pending:
                    time.sleep(max(0.0, min(0.01, pending[0].arrival - now())))
        finally:
            # also when a step raises: the ensemble's device arrays go back to the context
            if self.ens is not None:
                self.ens.close()
                self.ens = None
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
