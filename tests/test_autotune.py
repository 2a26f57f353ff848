"""Leaf-size tuning (cosmictiger_b200/autotune.py) on a fake device: the fastest candidate is
chosen, candidates whose forces leave the tolerance are excluded, particles are matched by
position although every run returns them in another order, and the state is uploaded before
every run."""
import numpy as np
import pytest

from cosmictiger_b200 import autotune

TIME = {64: 9.0, 96: 6.0, 128: 7.0, 160: 5.0, 192: 8.0}   # device ms per phase sum
ERR = {64: 1e-4, 96: 2e-4, 128: 0.0, 160: 5e-3, 192: 1e-3}  # relative force change


class FakeBox:
    def __init__(self, ctx, n):
        self.ctx = ctx
        self.n = n
        self.bucket = None
        self.uploads = 0
        self.kicks_since_upload = 0

    def upload(self, x, y, z, v, r):
        self.state = (x, y, z)
        self.uploads += 1
        self.kicks_since_upload = 0

    def tree_create(self, theta, h, bucket):
        self.bucket = bucket

    def kick(self, params):
        assert self.kicks_since_upload == 0, "a kick on a state that was not uploaded again"
        self.kicks_since_upload += 1
        self.save = bool(params.save_force)

    def counters(self):
        t = TIME[self.bucket] / len(autotune.PHASES)
        return {p: t for p in autotune.PHASES}

    def download(self, forces=False):
        assert forces and self.save
        x, y, z = self.state
        g = self.ctx.g * (1.0 + ERR[self.bucket])
        perm = self.ctx.rng.permutation(self.n)  # the tree build reorders particles
        return {"x": x[perm], "y": y[perm], "z": z[perm], "gx": g[perm, 0], "gy": g[perm, 1], "gz": g[perm, 2]}

    def close(self):
        self.ctx.closed += 1


class FakeContext:
    def __init__(self, n):
        self.rng = np.random.default_rng(1)
        self.g = self.rng.standard_normal((n, 3))
        self.closed = 0
        self.boxes = []

    def box(self, n):
        b = FakeBox(self, n)
        self.boxes.append(b)
        return b


def _state(n):
    rng = np.random.default_rng(2)
    x, y, z = (rng.choice(2 ** 32, n, replace=False).astype(np.uint32) for _ in range(3))
    return x, y, z, np.zeros((n, 3), np.float32), np.zeros(n, np.int8)


def test_fastest_without_force_check():
    ctx = FakeContext(500)
    res = autotune.tune_bucket(ctx, _state(500), repeats=2)
    assert res["best"] == 160
    assert [r["bucket"] for r in res["rows"]] == sorted(TIME)
    assert all(r["ms"] == TIME[r["bucket"]] for r in res["rows"])
    assert ctx.closed == 1 and ctx.boxes[0].uploads == 3 * len(TIME)


def test_force_tolerance_excludes_candidates():
    ctx = FakeContext(500)
    res = autotune.tune_bucket(ctx, _state(500), max_force_rms=1.5e-3, repeats=1)
    errs = {r["bucket"]: r["force_rms"] for r in res["rows"]}
    for b, e in ERR.items():
        assert abs(errs[b] - e) < 1e-9, (b, errs[b])
    assert res["best"] == 96  # 160 is faster but changes the forces by 5e-3


def test_rejects_untimed_settings():
    """Every candidate's first run only grows buffers, so at least one more is needed; an empty
    candidate list has nothing to choose.  Both are refused before any device work."""
    ctx = FakeContext(500)
    with pytest.raises(ValueError):
        autotune.tune_bucket(ctx, _state(500), repeats=0)
    with pytest.raises(ValueError):
        autotune.tune_bucket(ctx, _state(500), candidates=())
    assert not ctx.boxes


SHAPE_TIME = {(64, 1, 32): 9.0, (128, 1, 32): 8.0, (256, 1, 32): 7.5, (128, 2, 32): 6.0, (128, 1, 16): 5.0, (256, 2, 16): 7.0}
SHAPE_ERR = {(128, 1, 16): 3e-5}  # a shape whose forces leave the tolerance (it must not win)


class ShapeCtx:
    def __init__(self):
        self.shape = (128, 1, 32)
        self.set_calls = []

    def set_tuning(self, p2p_stage=128, warps_per_tile=1, tile_width=32):
        self.shape = (p2p_stage, warps_per_tile, tile_width)
        self.set_calls.append(self.shape)

    def box(self, n):
        return ShapeBox(self, n)


class ShapeBox(FakeBox):
    def counters(self):
        t = SHAPE_TIME[self.ctx.shape] * TIME[self.bucket] / 7.0 / len(autotune.PHASES)
        return {p: t for p in autotune.PHASES}

    def download(self, forces=False):
        # the tree order depends on the leaf size (the bucket), not on the launch shape
        assert forces and self.save
        rng = np.random.default_rng(self.bucket)
        perm = rng.permutation(self.n)
        x, y, z = (a[perm] for a in self.state)
        g = (x.astype(np.float64) + 2.0 * y + 3.0 * z) * (1.0 + SHAPE_ERR.get(self.ctx.shape, 0.0) + ERR[self.bucket])
        return {"x": x, "y": y, "z": z, "gx": g, "gy": g, "gz": g}

    def close(self):
        pass


def test_tune_picks_the_fastest_shape_within_the_force_tolerance():
    ctx = ShapeCtx()
    n = 500
    rng = np.random.default_rng(3)
    state = [rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32) for _ in range(3)] + [np.zeros((n, 3), np.float32), np.zeros(n, np.int8)]
    res = autotune.tune(ctx, state, h=1e-3, shapes=list(SHAPE_TIME), max_force_rms=1e-5)
    # the reference runs first and the winner is left set on the context
    assert ctx.set_calls[0] == (128, 1, 32)
    assert res["reference"]["p2p_stage"] == 128 and res["reference"]["force_rms"] == 0.0
    best = (res["best"]["p2p_stage"], res["best"]["warps_per_tile"], res["best"]["tile_width"])
    assert best == (128, 2, 32), best  # (128, 1, 16) is faster but its forces moved 3e-5
    assert ctx.shape == best
    assert len(res["rows"]) == len(SHAPE_TIME)
    # joint search with leaf sizes, no force limit: the fastest pair overall
    ctx2 = ShapeCtx()
    res2 = autotune.tune(ctx2, state, h=1e-3, buckets=(96, 128, 160), shapes=list(SHAPE_TIME), max_force_rms=None)
    assert (res2["best"]["bucket"], res2["best"]["p2p_stage"], res2["best"]["warps_per_tile"], res2["best"]["tile_width"]) == (160, 128, 1, 16)
    assert len(res2["rows"]) == 3 * len(SHAPE_TIME)


def test_tune_timing_only_downloads_nothing():
    """forces=False times the launch shapes without saving or downloading forces (the box's
    download raises if it is reached), still picks the fastest and leaves it set; a force bound
    without the forces is refused before any device work."""
    class NoDownload(ShapeBox):
        def download(self, forces=False):
            raise AssertionError("timing-only tuning downloaded the state")

    class Ctx(ShapeCtx):
        def box(self, n):
            return NoDownload(self, n)

    n = 300
    rng = np.random.default_rng(4)
    state = [rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32) for _ in range(3)] + [np.zeros((n, 3), np.float32), np.zeros(n, np.int8)]
    ctx = Ctx()
    res = autotune.tune(ctx, state, h=1e-3, shapes=list(SHAPE_TIME), max_force_rms=None, repeats=1, forces=False)
    best = (res["best"]["p2p_stage"], res["best"]["warps_per_tile"], res["best"]["tile_width"])
    assert best == (128, 1, 16) and ctx.shape == best
    assert all(r["force_rms"] is None for r in res["rows"])
    ctx2 = Ctx()
    with pytest.raises(ValueError):
        autotune.tune(ctx2, state, h=1e-3, max_force_rms=1e-5, forces=False)
    assert not ctx2.set_calls
