"""CUDA path vs the CPU oracle on the same seeded inputs (through the C ABI).

Integer work (tree keys, particle order, node ranges, fixed-point drift, rung partition) must
be bit-exact; node geometry (centres, radii, boxes) too, since it decides the opening tests;
kick forces and potentials within 1e-5 relative RMS.
"""
import numpy as np
import pytest

from cosmictiger_b200 import ics

pytestmark = pytest.mark.gpu

KICK_RMS_TOL = 1e-5


@pytest.fixture(scope="module")
def ctx():
    import cosmictiger_b200 as ct

    c = ct.Context(order=7)
    yield c
    c.close()


def lattice(n, seed=1, index=-2.0, rms=0.25):
    return ics.zeldovich_lattice(n, index=index, rms_spacing=rms, seed=seed)


def kick_params(theta, h, N, **kw):
    import cosmictiger_b200 as ct

    return ct.KickParams.make(theta=theta, h=h, GM=1.0 / N, eta=ics.eta_default(), **kw)


def oracle_kick_params(theta, h, N, **kw):
    from tests import oracle_lib

    d = dict(sign=1.0, min_rung=0, a=1.0, t0=1.0, theta=theta, h=h, eta=ics.eta_default(), GM=1.0 / N, max_dt=1e30, save_force=1, first_call=1,
             ascending=1, descending=1, top=1, do_phi=1)
    d.update({k: int(v) if isinstance(v, bool) else v for k, v in kw.items()})
    return oracle_lib.KickParams(**d)


def rel_rms(a, b):
    return float(np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)))


def test_drift_bitexact(ctx, oracle):
    rng = np.random.default_rng(7)
    N = 50000
    x, y, z = (rng.integers(0, 2 ** 32, N, dtype=np.uint64).astype(np.uint32) for _ in range(3))
    v = (rng.standard_normal((N, 3)) * 0.3).astype(np.float32)
    r = rng.integers(0, 3, N).astype(np.int8)
    for drag in (0.0, 0.25):
        box = ctx.box(N)
        box.upload(x, y, z, v, r)
        box.drift(1, 0.7, 0.013, drag)
        out = box.download()
        ox, oy, oz, ov = x.copy(), y.copy(), z.copy(), v.copy()
        oracle.drift(ox, oy, oz, ov, r, 1, 0.7, 0.013, drag)
        assert np.array_equal(out["x"], ox) and np.array_equal(out["y"], oy) and np.array_equal(out["z"], oz)
        assert np.array_equal(out["v"], ov)
        box.close()


def test_sort_by_rung_bitexact(ctx, oracle):
    rng = np.random.default_rng(8)
    N = 30001
    x, y, z = (rng.integers(0, 2 ** 32, N, dtype=np.uint64).astype(np.uint32) for _ in range(3))
    v = rng.standard_normal((N, 3)).astype(np.float32)
    r = rng.integers(0, 4, N).astype(np.int8)
    box = ctx.box(N)
    box.upload(x, y, z, v, r)
    ox, oy, oz, ov, orr = x.copy(), y.copy(), z.copy(), v.copy(), r.copy()
    begin = 0
    for minrung in (1, 2, 3):
        rb = box.sort_by_rung(minrung)
        begin = oracle.sort_by_rung(ox, oy, oz, ov, orr, minrung, begin)
        assert rb == begin
    out = box.download()
    for k, ref in (("x", ox), ("y", oy), ("z", oz), ("v", ov), ("rung", orr)):
        assert np.array_equal(out[k], ref), k
    box.close()


@pytest.mark.parametrize("n,theta,bucket,seed", [(16, 0.7, 128, 1), (32, 0.55, 128, 2), (24, 0.7, 64, 3)])
def test_tree_bitexact(ctx, oracle, n, theta, bucket, seed):
    x, y, z, v, r = lattice(n, seed=seed)
    N = len(x)
    h = ics.softening(N, 0.02)
    box = ctx.box(N)
    box.upload(x, y, z, v, r)
    box.tree_create(theta, h, bucket)
    nodes = box.tree()
    out = box.download()
    ox, oy, oz, ov, orr = x.copy(), y.copy(), z.copy(), v.copy(), r.copy()
    onodes = oracle.tree_build(ox, oy, oz, ov, orr, theta, h, bucket)
    # particle order
    assert np.array_equal(out["x"], ox) and np.array_equal(out["y"], oy) and np.array_equal(out["z"], oz)
    assert np.array_equal(out["v"], ov) and np.array_equal(out["rung"], orr)
    # nodes by heap key
    assert len(nodes) == len(onodes)
    a = nodes[np.argsort(nodes["key"])]
    b = onodes[np.argsort(onodes["key"])]
    assert np.array_equal(a["key"], b["key"])
    for f in ("part_begin", "part_end", "leaf", "depth", "pos", "box_begin", "box_end"):
        assert np.array_equal(a[f], b[f]), f
    assert np.array_equal(a["radius"].view(np.uint32), b["radius"].view(np.uint32)), "radius"
    # multipoles: the P2M sums run in a different order (double accumulation, float result)
    m_a, m_b = a["multi"], b["multi"]
    assert np.max(np.abs(m_a - m_b) / (np.abs(m_b) + 1e-6 * np.abs(m_b[:, :1]) + 1e-30)) < 1e-5
    box.close()


@pytest.mark.parametrize("n,theta,seed", [(16, 0.7, 1), (24, 0.55, 4)])
def test_kick_parity(ctx, oracle, n, theta, seed):
    x, y, z, v, r = lattice(n, seed=seed)
    N = len(x)
    h = ics.softening(N, 0.02)
    box = ctx.box(N)
    box.upload(x, y, z, v, r)
    box.tree_create(theta, h, 128)
    kr = box.kick(kick_params(theta, h, N))
    out = box.download(forces=True)
    ox, oy, oz, ov, orr = x.copy(), y.copy(), z.copy(), v.copy(), r.copy()
    onodes = oracle.tree_build(ox, oy, oz, ov, orr, theta, h, 128)
    (gx, gy, gz, pot), orc, _ = oracle.kick(oracle_kick_params(theta, h, N), onodes, ox, oy, oz, ov, orr)
    g_gpu = np.stack([out["gx"], out["gy"], out["gz"]], 1).astype(np.float64)
    g_or = np.stack([gx, gy, gz], 1).astype(np.float64)
    err = rel_rms(g_gpu, g_or)
    perr = rel_rms(out["pot"].astype(np.float64), pot.astype(np.float64))
    assert err < KICK_RMS_TOL, err
    assert perr < KICK_RMS_TOL, perr
    # velocities after the kick and rungs
    assert rel_rms(out["v"].astype(np.float64), ov.astype(np.float64)) < KICK_RMS_TOL
    assert np.mean(out["rung"] != orr) < 1e-3
    assert kr.max_rung == orc.max_rung
    assert abs(kr.pot - orc.pot) <= 1e-5 * abs(orc.pot)
    assert abs(kr.kin - orc.kin) <= 1e-5 * abs(orc.kin)
    box.close()


def test_direct_ewald_matches_oracle(ctx, oracle):
    x, y, z, v, r = lattice(12, seed=5)
    N = len(x)
    h = ics.softening(N, 0.02)
    box = ctx.box(N)
    box.upload(x, y, z, v, r)
    sel = np.arange(0, N, 37)
    g = box.direct_ewald(x[sel], y[sel], z[sel], h)
    o = oracle.direct_ewald(x, y, z, x[sel], y[sel], z[sel], h)
    for a, b in zip(g, o):
        assert np.max(np.abs(a - b)) <= 1e-9 * np.max(np.abs(b))
    box.close()


def test_force_accuracy_vs_direct_ewald(ctx):
    """Tree forces vs the FP64 direct Ewald sum at small theta (the reference's force_test
    protocol, src/test.cpp:335-400)."""
    x, y, z, v, r = lattice(16, seed=9)
    N = len(x)
    h = ics.softening(N, 0.02)
    box = ctx.box(N)
    box.upload(x, y, z, v, r)
    box.tree_create(0.3, h, 128)
    box.kick(kick_params(0.3, h, N))
    out = box.download(forces=True)
    sel = np.arange(0, N, 16)
    dg = box.direct_ewald(out["x"][sel], out["y"][sel], out["z"][sel], h)
    g_t = np.stack([out["gx"][sel], out["gy"][sel], out["gz"][sel]], 1).astype(np.float64)
    g_d = np.stack(dg[:3], 1) / N
    err = np.linalg.norm(g_t - g_d, axis=1) / np.linalg.norm(g_d, axis=1)
    assert np.sqrt(np.mean(err ** 2)) < 3e-3
    box.close()
