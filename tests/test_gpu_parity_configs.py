"""CUDA path vs the CPU oracle at the benchmark configurations' own sizes (through the C ABI).

* lattice 64^3 (Zel'dovich k^-2 lattice, 0.25 mean-spacing RMS, theta 0.7, softening 1/50 of
  the mean spacing, Ewald, one all-particles step): tree bit-exact (particle order, keys,
  particle ranges, leaf flags, depths, centres, radius bits, boxes), every particle's force,
  potential and velocity within the kick tolerance, rungs identical, drift bit-exact;
* clustered 256^3 (70% Zel'dovich k^-1.5 lattice, 30% in 20,000 Plummer spheres, theta 0.55):
  tree bit-exact over all 16.8M particles, the kick on >= 10^4 sinks (the oracle walks a seeded
  sample of its work items) within the tolerance, rungs identical;
* clustered 64^3, ten hierarchical steps (the rung ladder of kick_step_hierarchical, 4+ rungs):
  the ladder run kick by kick through the C ABI with the oracle in lock step -- every rung
  sort, tree build and drift bit-exact, every kick within the tolerance with identical rungs --
  and the same ladder as one ct_step_hierarchical call per step bit-identical to it.

Rungs.  The rung rule (kick.cu:133-140) compares log2(t0 / dt), dt = eta sqrt(a h / |g|), with
the kick's min_rung.  Forces that agree to 1e-7 can still fall on the two sides of that
boundary when a particle sits on it, so a rung may differ only where the two kicks' own forces
put log2(t0 / dt) on different sides of the boundary or within 1e-5 of it; every other rung
must be identical.  The tests count those particles and require them to be rare.
"""
import numpy as np
import pytest

from cosmictiger_b200 import ics

pytestmark = pytest.mark.gpu

KICK_RMS_TOL = 1e-5
RUNG_EDGE = 1e-5  # |log2(t0/dt) - boundary| below which float rounding may decide a rung
POT_SCALE_TOL = 1e-6
MEAN_INV_R_UNIT_CELL = 2.3800772
CLUSTERED_N = 256  # the clustered workload: CLUSTERED_N^3 particles


@pytest.fixture(scope="module")
def ctx():
    import cosmictiger_b200 as ct

    c = ct.Context(order=7)
    yield c
    c.close()


def rel_rms(a, b):
    return float(np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)))


def oracle_params(**kw):
    from tests import oracle_lib

    d = dict(sign=1.0, min_rung=0, a=1.0, t0=1.0, theta=0.7, h=1e-3, eta=ics.eta_default(), GM=1.0, max_dt=1e30, save_force=1, first_call=1,
             ascending=1, descending=1, top=1, do_phi=1)
    d.update({k: int(v) if isinstance(v, bool) else v for k, v in kw.items()})
    return oracle_lib.KickParams(**d)


def compare_trees(gpu_nodes, or_nodes):
    assert len(gpu_nodes) == len(or_nodes)
    a = gpu_nodes[np.argsort(gpu_nodes["key"], kind="stable")]
    b = or_nodes[np.argsort(or_nodes["key"], kind="stable")]
    assert np.array_equal(a["key"], b["key"])
    for f in ("part_begin", "part_end", "leaf", "depth", "pos", "box_begin", "box_end"):
        assert np.array_equal(a[f], b[f]), f
    assert np.array_equal(a["radius"].view(np.uint32), b["radius"].view(np.uint32)), "radius"


def rung_edge_distance(g, kp):
    """log2(t0 / dt) minus the rung boundary (the kick's min_rung), from forces g (N, 3).  The
    rule clamps dt to t0 and max_dt, which only moves log2(t0 / dt) further from a boundary at
    min_rung >= 0, so the unclamped dt = eta sqrt(a h / |g|) decides the side."""
    gm = np.sqrt(np.sum(np.asarray(g, np.float64) ** 2, axis=1))
    dt = kp.eta * np.sqrt(kp.a * kp.h / np.maximum(gm, 1e-300))
    return np.log2(kp.t0 / dt) - kp.min_rung


def check_rungs(r_gpu, r_or, g_gpu, g_or, kp, r_before):
    """Rungs identical except where the two force sets straddle the rung boundary (or sit within
    RUNG_EDGE of it) and the previous rung does not decide the result.  Returns the number of
    such boundary particles and of differing rungs."""
    e_g = rung_edge_distance(g_gpu, kp)
    e_o = rung_edge_distance(g_or, kp)
    # rung = max(min_rung + [ceil(log2(t0/dt)) > min_rung], rung - 1): only the comparison
    # log2(t0/dt) > min_rung can flip, and only while rung - 1 <= min_rung
    open_ = (np.asarray(r_before, np.int64) - 1) <= kp.min_rung
    edge = open_ & ((np.sign(e_g) != np.sign(e_o)) | (np.abs(e_g) < RUNG_EDGE) | (np.abs(e_o) < RUNG_EDGE))
    diff = r_gpu != r_or
    assert not np.any(diff & ~edge), "rungs differ away from the rung boundary at %s" % np.nonzero(diff & ~edge)[0][:10]
    return int(edge.sum()), int(diff.sum())


# ------------------------------------------------------------------ lattice 64^3
def test_lattice64_step_parity(ctx, oracle):
    import cosmictiger_b200 as ct

    x, y, z, v, r = ics.zeldovich_lattice(64, index=-2.0, rms_spacing=0.25, seed=3)
    N = len(x)
    theta = 0.7
    h = ics.softening(N, 0.02)
    box = ctx.box(N)
    box.upload(x, y, z, v, r)
    box.tree_create(theta, h, 128)
    nodes = box.tree()
    t_ord = box.download()
    ox, oy, oz, ov, orr = x.copy(), y.copy(), z.copy(), v.copy(), r.copy()
    onodes = oracle.tree_build(ox, oy, oz, ov, orr, theta, h, 128)
    for k, ref in (("x", ox), ("y", oy), ("z", oz), ("v", ov), ("rung", orr)):
        assert np.array_equal(t_ord[k], ref), k
    compare_trees(nodes, onodes)
    # one all-particles step at a single rung: first call, top, ascending and descending
    kr = box.kick(ct.KickParams.make(theta=theta, h=h, GM=1.0 / N, eta=ics.eta_default(), t0=1.0, first_call=True))
    out = box.download(forces=True)
    okp = oracle_params(theta=theta, h=h, GM=1.0 / N, t0=1.0)
    ov2 = ov.copy()
    (gx, gy, gz, pot), orc, _ = oracle.kick(okp, onodes, ox, oy, oz, ov2, orr)
    g_gpu = np.stack([out["gx"], out["gy"], out["gz"]], 1).astype(np.float64)
    g_or = np.stack([gx, gy, gz], 1).astype(np.float64)
    ferr = rel_rms(g_gpu, g_or)
    verr = rel_rms(out["v"].astype(np.float64), ov2.astype(np.float64))
    dphi = out["pot"].astype(np.float64) - pot.astype(np.float64)
    pscale = float(np.sqrt(np.mean(dphi ** 2))) / MEAN_INV_R_UNIT_CELL
    nedge, ndiff = check_rungs(out["rung"], orr, g_gpu, g_or, okp, t_ord["rung"])
    print("lattice 64^3: force rel rms %.3g, velocity %.3g, potential/scale %.3g, rungs %s, boundary %d, differing %d"
          % (ferr, verr, pscale, np.bincount(out["rung"]), nedge, ndiff))
    assert ferr < KICK_RMS_TOL and verr < KICK_RMS_TOL
    assert pscale < POT_SCALE_TOL
    assert ndiff <= max(2, N // 10000)
    assert kr.max_rung == orc.max_rung
    assert abs(kr.kin - orc.kin) <= 1e-5 * abs(orc.kin)
    # the drift of the kicked particles, bit for bit
    box.drift(0, 1.0, 1.0 / 64)
    d = box.download()
    dx, dy, dz, dv = out["x"].copy(), out["y"].copy(), out["z"].copy(), out["v"].copy()
    oracle.drift(dx, dy, dz, dv, out["rung"], 0, 1.0, 1.0 / 64)
    for k, ref in (("x", dx), ("y", dy), ("z", dz), ("v", dv)):
        assert np.array_equal(d[k], ref), k
    # t0 = 1 puts every particle on rung 1; a t0 at the median timestep splits them in half,
    # so that the rung decision is compared on both sides of its boundary
    dts = ics.eta_default() * np.sqrt(h / np.linalg.norm(g_or, axis=1))
    t0 = float(np.median(dts))
    box.upload(ox, oy, oz, ov, np.zeros(N, np.int8))
    box.tree_create(theta, h, 128)
    box.kick(ct.KickParams.make(theta=theta, h=h, GM=1.0 / N, eta=ics.eta_default(), t0=t0, first_call=True))
    out = box.download(forces=True)
    okp = oracle_params(theta=theta, h=h, GM=1.0 / N, t0=t0)
    ov3, or3 = ov.copy(), np.zeros(N, np.int8)
    (gx, gy, gz, pot), orc, _ = oracle.kick(okp, onodes, ox, oy, oz, ov3, or3)
    g_gpu = np.stack([out["gx"], out["gy"], out["gz"]], 1).astype(np.float64)
    g_or = np.stack([gx, gy, gz], 1).astype(np.float64)
    nedge, ndiff = check_rungs(out["rung"], or3, g_gpu, g_or, okp, np.zeros(N, np.int8))
    print("lattice 64^3 at the median timestep: rungs %s, boundary %d, differing %d" % (np.bincount(out["rung"]), nedge, ndiff))
    assert min(np.bincount(out["rung"], minlength=2)[:2]) > N // 4
    assert ndiff <= max(2, N // 10000)
    assert rel_rms(out["v"].astype(np.float64), ov3.astype(np.float64)) < KICK_RMS_TOL
    box.close()


# ------------------------------------------------------------------ clustered 256^3
def test_clustered256_tree_and_sampled_kick_parity(ctx, oracle):
    import cosmictiger_b200 as ct

    n = CLUSTERED_N
    x, y, z, v, r = ics.clustered_box(n, nspheres=max(1, int(round(20000 * (n / 256) ** 3))), seed=3)
    N = len(x)
    theta = 0.55
    h = ics.softening(N, 0.02)
    box = ctx.box(N)
    box.upload(x, y, z, v, r)
    box.tree_create(theta, h, 128)
    nodes = box.tree()
    t_ord = box.download()
    ox, oy, oz, ov, orr = x, y, z, v, r  # the oracle reorders in place (the inputs are not needed again)
    onodes = oracle.tree_build(ox, oy, oz, ov, orr, theta, h, 128)
    for k, ref in (("x", ox), ("y", oy), ("z", oz), ("v", ov), ("rung", orr)):
        assert np.array_equal(t_ord[k], ref), k
    compare_trees(nodes, onodes)
    del nodes, t_ord
    # rungs by |a| as the benchmark sets them: t0 such that 1% of the particles want dt < t0/8
    kr0 = box.kick(ct.KickParams.make(theta=theta, h=h, GM=1.0 / N, eta=ics.eta_default(), t0=1.0, save_force=True, ascending=False, descending=False))
    del kr0
    f0 = box.download(forces=True)
    gm = np.sqrt(f0["gx"].astype(np.float64) ** 2 + f0["gy"] ** 2 + f0["gz"] ** 2)
    t0 = float(8.0 * np.percentile(ics.eta_default() * np.sqrt(h / gm), 1))
    del f0, gm
    box.upload(ox, oy, oz, ov, orr)
    box.tree_create(theta, h, 128)
    kr = box.kick(ct.KickParams.make(theta=theta, h=h, GM=1.0 / N, eta=ics.eta_default(), t0=t0, first_call=True))
    out = box.download(forces=True)
    box.close()
    # the tree of already partitioned particles keeps their order
    assert np.array_equal(out["x"], ox) and np.array_equal(out["y"], oy) and np.array_equal(out["z"], oz)
    okp = oracle_params(theta=theta, h=h, GM=1.0 / N, t0=t0)
    ovk, ork = ov.copy(), orr.copy()
    plan = oracle.plan(okp, onodes, ox, oy, oz, max_parts=2048)
    rng = np.random.default_rng(2024)
    sel = np.zeros(plan.nitems, bool)
    order = rng.permutation(plan.nitems)
    tot = 0
    for i in order:  # seeded items until at least 2 x 10^4 sinks
        sel[i] = True
        tot += plan.nparts[i]
        if tot >= 20000:
            break
    (gx, gy, gz, pot), _, _, _ = plan.run(ovk, ork, select=sel)
    plan.close()
    idx = plan.particles(sel)
    assert len(idx) >= 10000
    g_gpu = np.stack([out["gx"][idx], out["gy"][idx], out["gz"][idx]], 1).astype(np.float64)
    g_or = np.stack([gx[idx], gy[idx], gz[idx]], 1).astype(np.float64)
    ferr = rel_rms(g_gpu, g_or)
    perr = rel_rms(out["pot"][idx].astype(np.float64), pot[idx].astype(np.float64))
    # potentials of the lattice particles are small residuals of the direct and Ewald sums
    # (each about MEAN_INV_R_UNIT_CELL), so they are compared against that scale
    pscale = float(np.sqrt(np.mean((out["pot"][idx].astype(np.float64) - pot[idx]) ** 2))) / MEAN_INV_R_UNIT_CELL
    verr = rel_rms(out["v"][idx].astype(np.float64), ovk[idx].astype(np.float64))
    nedge, ndiff = check_rungs(out["rung"][idx], ork[idx], g_gpu, g_or, okp, orr[idx])
    print("clustered 256^3: %d sinks in %d work items; force rel rms %.3g, potential %.3g (/scale %.3g), velocity %.3g; rungs %s, boundary %d, differing %d"
          % (len(idx), sel.sum(), ferr, perr, pscale, verr, np.bincount(out["rung"][idx]), nedge, ndiff))
    assert ferr < KICK_RMS_TOL and verr < KICK_RMS_TOL
    assert pscale < POT_SCALE_TOL
    assert ndiff <= max(2, len(idx) // 10000)
    assert kr.max_rung >= int(ork[idx].max())


# ------------------------------------------------------------------ hierarchical ladder
def ladder_step(box, sp, on_sort=None, on_tree=None, on_kick=None, on_drift=None):
    """One step of the rung ladder of ct_step_hierarchical (kick_step_hierarchical,
    driver.cpp:382-593) through the single-call entry points, kicks with save_force so that
    every kick's forces can be compared.  The callbacks see the state around each operation."""
    import cosmictiger_b200 as ct

    minrung = sp["minrung"]
    max_rung = max(sp["max_rung"], minrung)
    levels = list(range(max_rung, minrung, -1)) + [minrung]
    ascending, clip_top = True, False
    top_kr = None
    li = 0
    while li < len(levels):
        level = levels[li]
        top = level == minrung
        if top:
            ascending = False
        if not ascending and not top:
            rb, stack = box.rung_state()
            box.set_rung_state(rb, stack + [rb])  # particles_push_rungs
        if not ascending:
            pre = on_sort and on_sort(None, level)
            rb = box.sort_by_rung(level)
            if on_sort:
                on_sort(pre, level, rb)
        if top and minrung == sp["minrung0"]:
            counts = box.rung_counts().astype(np.int64)
            if np.nonzero(counts)[0].max() > sp["minrung0"]:
                fast = counts[sp["minrung0"] + 1:].sum()
                slow = counts[sp["minrung0"]]
                if 3 * fast > slow:
                    clip_top = not sp["nocrop"]
        pre = on_tree and on_tree(None, level)
        box.tree_create(sp["theta"], sp["hsoft"], sp["bucket"], min_rung=level)
        if on_tree:
            on_tree(pre, level)
        kp = ct.KickParams.make(theta=sp["theta"], h=sp["hsoft"], GM=sp["GM"], eta=sp["eta"], min_rung=level, a=sp["a"], t0=sp["t0"],
                                max_dt=sp["max_dt"], save_force=True, first_call=sp["tau"] == 0.0, ascending=ascending or top,
                                descending=False if (clip_top and top) else ((not ascending) or top),
                                top=True if (clip_top and level == sp["minrung0"] + 1) else top, do_phi=bool(sp["do_phi"] and top))
        pre = on_kick and on_kick(None, kp)
        kr = box.kick(kp)
        if on_kick:
            on_kick(pre, kp, kr)
        if clip_top and top:
            d = box.download()
            rb, stack = box.rung_state()
            box.upload(d["x"], d["y"], d["z"], d["v"], np.maximum(d["rung"], sp["minrung0"] + 1).astype(np.int8))
            box.set_rung_state(rb, stack)
        if top:
            top_kr = kr
        if clip_top and top:
            levels.append(sp["minrung0"] + 1)
        elif (not ascending) or top:
            max_rung = kr.max_rung
            if max_rung > level:
                levels.append(level + 1)
        if ((not ascending) or top) and not (clip_top and top):
            pre = on_drift and on_drift(None, level)
            box.drift(level, sp["a"], (1.0 / (1 << level)) * sp["t0"], sp["drag"])
            if on_drift:
                on_drift(pre, level)
        if ascending and not top:
            rb, stack = box.rung_state()
            box.set_rung_state(stack[-1], stack[:-1])  # particles_pop_rungs
        li += 1
    if clip_top:
        minrung += 1
    return top_kr, minrung, max_rung


def test_hierarchical_ladder_lockstep_64(ctx, oracle):
    """Ten hierarchical steps of a clustered 64^3 box: every operation of the ladder against
    the oracle on the same state (the device state is the master; the oracle restarts from it
    before each operation), and ct_step_hierarchical on a second box bit-identical to the
    ladder run operation by operation."""
    import cosmictiger_b200 as ct

    n = 64
    x, y, z, v, r = ics.clustered_box(n, nspheres=int(round(20000 * (n / 256) ** 3)), seed=5)
    N = len(x)
    theta = 0.55
    h = ics.softening(N, 0.02)
    eta = ics.eta_default()
    box = ctx.box(N)
    box.upload(x, y, z, v, r)
    box.tree_create(theta, h, 128)
    box.kick(ct.KickParams.make(theta=theta, h=h, GM=1.0 / N, eta=eta, t0=1.0, save_force=True, ascending=False, descending=False))
    f = box.download(forces=True)
    gm = np.sqrt(f["gx"].astype(np.float64) ** 2 + f["gy"] ** 2 + f["gz"] ** 2)
    t0 = float(8.0 * np.percentile(eta * np.sqrt(h / gm), 1))
    box.upload(x, y, z, v, r)
    box.sort_by_rung(0)
    twin = ctx.box(N)
    twin.upload(x, y, z, v, r)
    twin.sort_by_rung(0)
    sp = dict(minrung=0, minrung0=0, max_rung=0, a=1.0, tau=0.0, t0=t0, theta=theta, hsoft=h, bucket=128, eta=eta, GM=1.0 / N, max_dt=1e30,
              do_phi=1, nocrop=0, drag=0.0, sign=1.0)
    stats = {"kicks": 0, "trees": 0, "sorts": 0, "drifts": 0, "edge": 0, "diff": 0, "active": 0, "ferr": 0.0, "verr": 0.0}

    def state():
        d = box.download()
        rb, stack = box.rung_state()
        d["rung_begin"] = rb
        return d

    def on_sort(pre, level, rb=None):
        if pre is None:
            return state()
        ox, oy, oz, ov, orr = (pre[k].copy() for k in ("x", "y", "z", "v", "rung"))
        ob = oracle.sort_by_rung(ox, oy, oz, ov, orr, level, pre["rung_begin"]) if level > 0 else 0
        post = box.download()
        assert rb == ob, (level, rb, ob)
        for k, ref in (("x", ox), ("y", oy), ("z", oz), ("v", ov), ("rung", orr)):
            assert np.array_equal(post[k], ref), ("sort", level, k)
        stats["sorts"] += 1

    def on_tree(pre, level):
        if pre is None:
            return state()
        b = pre["rung_begin"]
        ox, oy, oz, ov, orr = (pre[k].copy() for k in ("x", "y", "z", "v", "rung"))
        onodes = oracle.tree_build(ox, oy, oz, ov, orr, theta, h, 128, begin=b)
        post = box.download()
        for k, ref in (("x", ox), ("y", oy), ("z", oz), ("v", ov), ("rung", orr)):
            assert np.array_equal(post[k], ref), ("tree", level, k)
        compare_trees(box.tree(), onodes)
        stats["trees"] += 1
        stats["onodes"] = onodes

    def on_kick(pre, kp, kr=None):
        if pre is None:
            return state()
        b = pre["rung_begin"]
        okp = oracle_params(sign=kp.sign, min_rung=kp.min_rung, a=kp.a, t0=kp.t0, theta=kp.theta, h=kp.h, eta=kp.eta, GM=kp.GM, max_dt=kp.max_dt,
                            save_force=1, first_call=kp.first_call, ascending=kp.ascending, descending=kp.descending, top=kp.top, do_phi=kp.do_phi)
        ox, oy, oz, ov, orr = (pre[k].copy() for k in ("x", "y", "z", "v", "rung"))
        (gx, gy, gz, pot), orc, _ = oracle.kick(okp, stats["onodes"], ox, oy, oz, ov, orr)
        post = box.download(forces=True)
        s = slice(b, N)
        g_gpu = np.stack([post["gx"][s], post["gy"][s], post["gz"][s]], 1).astype(np.float64)
        g_or = np.stack([gx[s], gy[s], gz[s]], 1).astype(np.float64)
        ferr = rel_rms(g_gpu, g_or)
        verr = rel_rms(post["v"][s].astype(np.float64), ov[s].astype(np.float64))
        assert ferr < KICK_RMS_TOL, ferr
        assert verr < KICK_RMS_TOL, verr
        # inactive particles untouched
        assert np.array_equal(post["v"][:b], pre["v"][:b]) and np.array_equal(post["rung"][:b], pre["rung"][:b])
        if kp.descending:
            ne, nd = check_rungs(post["rung"][s], orr[s], g_gpu, g_or, okp, pre["rung"][s])
            stats["edge"] += ne
            stats["diff"] += nd
            if nd == 0:
                assert kr.max_rung == orc.max_rung
        else:
            assert np.array_equal(post["rung"], pre["rung"])
        stats["kicks"] += 1
        stats["active"] += N - b
        stats["ferr"] = max(stats["ferr"], ferr)
        stats["verr"] = max(stats["verr"], verr)

    def on_drift(pre, level):
        if pre is None:
            return state()
        ox, oy, oz, ov = (pre[k].copy() for k in ("x", "y", "z", "v"))
        oracle.drift(ox, oy, oz, ov, pre["rung"], level, sp["a"], (1.0 / (1 << level)) * sp["t0"], sp["drag"])
        post = box.download()
        for k, ref in (("x", ox), ("y", oy), ("z", oz), ("v", ov)):
            assert np.array_equal(post[k], ref), ("drift", level, k)
        stats["drifts"] += 1

    ladders = []
    max_seen = 0
    for step in range(10):
        p = dict(sp)
        _, minrung, max_rung = ladder_step(box, p, on_sort, on_tree, on_kick, on_drift)
        tp = ct.StepParams(**sp)
        res = twin.step_hierarchical(tp)
        assert (res.minrung, res.max_rung) == (minrung, max_rung), (step, res.minrung, res.max_rung, minrung, max_rung)
        a, b2 = box.download(), twin.download()
        for k in ("x", "y", "z", "v", "rung"):
            assert np.array_equal(a[k], b2[k]), ("ct_step_hierarchical vs the ladder", step, k)
        assert box.rung_state() == twin.rung_state()
        ladders.append((minrung, max_rung))
        max_seen = max(max_seen, max_rung)
        sp.update(minrung=minrung, max_rung=max_rung, tau=sp["tau"] + t0)
    print("hierarchical 64^3, 10 steps: ladders %s; %d kicks (%.3g active kicks), %d trees, %d sorts, %d drifts bit-exact; worst force rel rms %.3g, "
          "velocity %.3g; rungs on the boundary %d, differing %d" % (ladders, stats["kicks"], stats["active"], stats["trees"], stats["sorts"],
                                                                    stats["drifts"], stats["ferr"], stats["verr"], stats["edge"], stats["diff"]))
    assert max_seen >= 3
    assert stats["diff"] <= max(2, stats["active"] // 100000)
    box.close()
    twin.close()
