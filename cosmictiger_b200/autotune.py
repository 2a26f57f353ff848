"""Leaf-size tuning for a workload.

The kick kernels' sink tile (32 sinks per warp, 16 or fewer in the small-tile launch) and the
warps per tile are fixed when the library is built; the leaf size -- the tree's bucket, the
reference's `bucket_size` option passed to tree_create (src/tree.cpp:273) -- is the run-time
knob.  Larger leaves move work from the multipole operators (M2L, P2L, M2P, tree depth) to
direct particle pairs; the best size depends on the clustering and on theta.

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
