"""The kick's launch shapes (ct_ctx_set_tuning: P2P cell-list size, warps per sink tile, sink
tile width) give the same forces to float rounding -- only the order of each sink's sums
differs -- and each shape is deterministic; out-of-range shapes are refused."""
import ctypes

import numpy as np
import pytest

from cosmictiger_b200 import autotune, ics

pytestmark = pytest.mark.gpu


def test_every_launch_shape_matches_the_default():
    import cosmictiger_b200 as ct

    x, y, z, v, r = ics.clustered_box(32, nspheres=40, seed=12)
    N = len(x)
    theta = 0.55
    h = ics.softening(N, 0.02)
    ctx = ct.Context(order=7)
    box = ctx.box(N)

    def run():
        box.upload(x, y, z, v, r)
        box.tree_create(theta, h, 128)
        kr = box.kick(ct.KickParams.make(theta=theta, h=h, GM=1.0 / N, eta=ics.eta_default(), t0=1.0 / 64, first_call=True))
        o = box.download(forces=True)
        return kr, o, np.stack([o["gx"], o["gy"], o["gz"]], 1).astype(np.float64)

    assert ctx.tuning() == {"p2p_stage": 128, "warps_per_tile": 1, "tile_width": 32}
    kr0, o0, g0 = run()
    for shape in autotune.SHAPES:
        ctx.set_tuning(*shape)
        kr, o, g = run()
        _, o2, _ = run()
        for f in ("gx", "gy", "gz", "pot", "v", "rung"):
            assert np.array_equal(o[f], o2[f]), (shape, f)  # deterministic
        assert np.array_equal(o["x"], o0["x"])  # same tree order
        err = float(np.sqrt(np.sum((g - g0) ** 2) / np.sum(g0 ** 2)))
        assert err < 1e-6, (shape, err)
        assert kr.max_rung == kr0.max_rung
        assert np.mean(o["rung"] != o0["rung"]) < 1e-3
    with pytest.raises(ct.GravityError):
        ctx.set_tuning(96, 1, 32)
    with pytest.raises(ct.GravityError):
        ctx.set_tuning(128, 3, 32)
    with pytest.raises(ct.GravityError):
        ctx.set_tuning(128, 1, 24)
    box.close()
    ctx.close()
