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
