"""Autotuning of the kick's launch shape and leaf size for a workload.

The knobs (the reference fixes all of them at build time):
  * the leaf size -- the tree's bucket, the reference's `bucket_size` option passed to
    tree_create (src/tree.cpp:273); larger leaves move work from the multipole operators (M2L,
    P2L, M2P, tree depth) to direct particle pairs, and change the forces within the
    expansion's truncation error;
  * the P2P cell-list size -- source particles staged in shared memory per pass (the
    reference's KICK_PP_MAX, cosmictiger/kick.hpp:48): 64, 128 or 256;
  * warps per sink tile -- one warp, or a pair splitting the tile's sources: 1 or 2;
  * sink tile width -- sinks per tile for P2P and the leaf kick: 32, or 16 (each sink's
    sources and multipoles then spread over two or more lanes).
The last three change only the order of the per-sink sums (ct_ctx_set_tuning).

tune() times every (leaf size, launch shape) pair on a representative state and returns the
fastest whose forces stay within `max_force_rms` of the reference configuration's.

tune_bucket times every candidate on a representative state with the library's own device
timings of the phases (tree build, walk, M2L, L2L, P2P, leaf kick; the kick changes velocities
and rungs, so the state is uploaded again before every run) and returns the fastest candidate
whose forces stay within `max_force_rms` (relative RMS) of those at `reference_bucket`.
Particles are matched across runs by position: the tree build reorders them, differently for
different leaf sizes, and the kick does not move them.
"""
import numpy as np

from . import ics

PHASES = ("ms_tree", "ms_walk", "ms_m2l", "ms_l2l", "ms_leaf", "ms_leafkick")


def _by_position(out):
    order = np.lexsort((out["z"], out["y"], out["x"]))
    return np.stack([out["gx"][order], out["gy"][order], out["gz"][order]], axis=1).astype(np.float64)


def tune_bucket(ctx, state, theta=0.55, h=None, candidates=(64, 96, 128, 160, 192), reference_bucket=128, max_force_rms=None, repeats=2):
    """Returns {"best": bucket, "rows": [{"bucket", "ms", "force_rms"}...]}.  `state` is
    (x, y, z, vxyz, rung) host arrays of one box; `max_force_rms` None skips the force check."""
    from . import KickParams

    if repeats < 1:
        raise ValueError("repeats must be >= 1 (the first run of each candidate is not timed)")
    if not candidates:
        raise ValueError("no candidate leaf sizes")
    x, y, z, v, r = state
    n = len(x)
    h = ics.softening(n, 0.02) if h is None else h
    check = max_force_rms is not None
    order = list(candidates)
    if check:
        order = [reference_bucket] + [b for b in order if b != reference_bucket]
    box = ctx.box(n)
    rows = []
    ref = None
    try:
        for bucket in order:
            times = []
            g = None
            for rep in range(repeats + 1):
                box.upload(x, y, z, v, r)
                box.tree_create(theta, h, bucket)
                box.kick(KickParams.make(theta=theta, h=h, GM=1.0 / n, eta=ics.eta_default(), t0=1.0 / 64, first_call=True, save_force=check))
                c = box.counters()
                if rep > 0:  # the first run grows buffers and is not timed
                    times.append(sum(c[p] for p in PHASES))
                if check and rep == repeats:
                    g = _by_position(box.download(forces=True))
            row = {"bucket": bucket, "ms": float(min(times)), "force_rms": None}
            if check:
                if ref is None:
                    ref = g
                row["force_rms"] = float(np.sqrt(np.sum((g - ref) ** 2) / np.sum(ref ** 2)))
            rows.append(row)
    finally:
        box.close()
    ok = [row for row in rows if not check or row["force_rms"] <= max_force_rms]
    best = min(ok, key=lambda row: row["ms"])["bucket"]
    return {"best": best, "rows": sorted(rows, key=lambda row: row["bucket"])}


SHAPES = tuple((s, w, t) for s in (64, 128, 256) for w in (1, 2) for t in (32, 16))


def tune(ctx, state, theta=0.55, h=None, buckets=(128,), shapes=SHAPES, reference=(128, (128, 1, 32)), max_force_rms=1e-5, repeats=2,
         box_factory=None, forces=True):
    """Joint search over leaf sizes and launch shapes (p2p_stage, warps_per_tile, tile_width).
    Every candidate runs repeats + 1 times (the first untimed) on the state uploaded again each
    time; the time is the library's device time of the kick's phases (tree build included).
    Forces are compared with the reference candidate's (particles matched by position);
    max_force_rms None keeps every candidate.  box_factory() (default ctx.box(n)) makes the box
    the candidates run on, e.g. an ensemble with its per-box parameters set.  forces=False times
    the candidates only (no force download or comparison, force_rms None; max_force_rms must be
    None): for launch shapes alone, which change the forces only by rounding.  Leaves the context
    at the chosen shape; returns {"best": {...}, "reference": {...}, "rows": [...]}."""
    from . import KickParams

    if repeats < 1:
        raise ValueError("repeats must be >= 1 (the first run of each candidate is not timed)")
    if not forces and max_force_rms is not None:
        raise ValueError("a force bound needs the forces (forces=True)")
    x, y, z, v, r = state
    n = len(x)
    h = ics.softening(n, 0.02) if h is None else h
    cands = [(b, sh) for b in buckets for sh in shapes]
    if reference in cands:
        cands.remove(reference)
    cands = [reference] + cands
    box = box_factory() if box_factory else ctx.box(n)
    rows = []
    ref = None
    # the tree order depends on the leaf size only: particles are matched by position once per
    # leaf size (a sort of all particles), and the launch shapes of one leaf size compare in
    # tree order
    order_of = {}
    try:
        for bucket, shape in cands:
            ctx.set_tuning(*shape)
            times = []
            g = None
            for rep in range(repeats + 1):
                box.upload(x, y, z, v, r)
                box.tree_create(theta, h, bucket)
                box.kick(KickParams.make(theta=theta, h=h, GM=1.0 / n, eta=ics.eta_default(), t0=1.0 / 64, first_call=True, save_force=forces))
                c = box.counters()
                if rep > 0:
                    times.append(sum(c[p] for p in PHASES))
                if forces and rep == repeats:
                    out = box.download(forces=True)
                    if bucket not in order_of:
                        order_of[bucket] = (out["x"].copy(), np.lexsort((out["z"], out["y"], out["x"])))
                    tree_x, order = order_of[bucket]
                    if not np.array_equal(out["x"], tree_x):
                        raise RuntimeError("the tree order changed between launch shapes of one leaf size")
                    g = np.stack([out["gx"][order], out["gy"][order], out["gz"][order]], axis=1).astype(np.float64)
                    del out
            if forces and ref is None:
                ref = g
            rows.append({"bucket": bucket, "p2p_stage": shape[0], "warps_per_tile": shape[1], "tile_width": shape[2], "ms": float(min(times)),
                         "force_rms": float(np.sqrt(np.sum((g - ref) ** 2) / np.sum(ref ** 2))) if forces else None})
    finally:
        box.close()
    ok = [row for row in rows if max_force_rms is None or row["force_rms"] <= max_force_rms]
    best = min(ok, key=lambda row: row["ms"])
    ctx.set_tuning(best["p2p_stage"], best["warps_per_tile"], best["tile_width"])
    return {"best": best, "reference": rows[0], "rows": rows}
