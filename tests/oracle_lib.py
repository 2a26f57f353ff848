"""ctypes bindings of the CPU oracle (oracle/libct_oracle.so): test infrastructure only.

Imported by the tests, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg, always
as the checker of the CUDA path, never as the thing measured or shipped.
"""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
LIB = os.path.join(ORACLE_DIR, "libct_oracle.so")

NODE_DTYPE = np.dtype(
    [
        ("key", np.uint64),
        ("part_begin", np.int32),
        ("part_end", np.int32),
        ("child_left", np.int32),
        ("child_right", np.int32),
        ("pos", np.uint32, 3),
        ("radius", np.float32),
        ("box_begin", np.int32, 3),
        ("box_end", np.int32, 3),
        ("leaf", np.int32),
        ("depth", np.int32),
        ("multi", np.float32, 37),
    ],
    align=True,
)


# one lightcone crossing (ct_or_lc_entry / ct_lc_entry, the reference's lc_entry)
LC_ENTRY = np.dtype([("x", "<i4"), ("y", "<i4"), ("z", "<i4"), ("vx", "<f4"), ("vy", "<f4"), ("vz", "<f4"), ("pix", "<i4")])


class KickParams(ctypes.Structure):
    _fields_ = [
        ("sign", ctypes.c_float),
        ("min_rung", ctypes.c_int),
        ("a", ctypes.c_float),
        ("t0", ctypes.c_float),
        ("theta", ctypes.c_float),
        ("h", ctypes.c_float),
        ("eta", ctypes.c_float),
        ("GM", ctypes.c_float),
        ("max_dt", ctypes.c_float),
        ("save_force", ctypes.c_int),
        ("first_call", ctypes.c_int),
        ("ascending", ctypes.c_int),
        ("descending", ctypes.c_int),
        ("top", ctypes.c_int),
        ("do_phi", ctypes.c_int),
    ]


class KickReturn(ctypes.Structure):
    _fields_ = [
        ("max_rung", ctypes.c_int),
        ("pot", ctypes.c_double),
        ("kin", ctypes.c_double),
        ("dkin", ctypes.c_double),
        ("xmom", ctypes.c_double),
        ("ymom", ctypes.c_double),
        ("zmom", ctypes.c_double),
        ("nmom", ctypes.c_double),
    ]


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(ORACLE_DIR, f) for f in ("ct_oracle.cpp", "ct_oracle.h")]
    csrc = os.path.join(ROOT, "cosmictiger_b200", "csrc")
    deps += [os.path.join(csrc, f) for f in ("fmm_p7.h", "fmm_p5.h", "fmm_common.h")]
    return any(os.path.exists(d) and os.path.getmtime(d) > t for d in deps)


class Oracle:
    def __init__(self, path):
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.ct_or_tree_build.restype = ctypes.c_int
        L.ct_or_kick.restype = ctypes.c_int
        L.ct_or_sort_by_rung.restype = ctypes.c_int
        for name in ("ct_or_greens", "ct_or_ewald_greens", "ct_or_ewald_greens_d"):
            getattr(L, name).restype = ctypes.c_int

    # ---- operators
    def op(self, name, order, *arrays, flag=None):
        args = [ctypes.c_int(order)] + [_p(a) for a in arrays]
        if flag is not None:
            args.append(ctypes.c_int(flag))
        return getattr(self.lib, "ct_or_" + name)(*args)

    # ---- tree
    def tree_build(self, x, y, z, v, rung, theta, hsoft, bucket=128, order=7, begin=0, nthreads=0):
        """Tree over particles [begin, n), reordering them in place; nthreads <= 0 uses every
        core (the result does not depend on it)."""
        n = len(x)
        max_nodes = max(64, 8 * (n - begin) // max(bucket // 4, 1) + 1024)
        while True:
            nodes = np.zeros(max_nodes, NODE_DTYPE)
            cnt = self.lib.ct_or_tree_build(
                ctypes.c_int(order), ctypes.c_int(n), ctypes.c_int(begin), _p(x), _p(y), _p(z), _p(v), _p(rung),
                ctypes.c_double(theta), ctypes.c_double(hsoft), ctypes.c_int(bucket), _p(nodes), ctypes.c_int(max_nodes), ctypes.c_int(nthreads))
            if cnt >= 0:
                return nodes[:cnt]
            if cnt == -2:
                raise RuntimeError("oracle tree build: maximum depth exceeded")
            max_nodes *= 2
            if max_nodes > 1 << 28:
                raise RuntimeError("oracle tree build failed")

    def kick(self, params, nodes, x, y, z, v, rung, order=7, nthreads=0, save_force=True):
        n = len(x)
        gx = np.zeros(n, np.float32) if save_force else None
        gy = np.zeros(n, np.float32) if save_force else None
        gz = np.zeros(n, np.float32) if save_force else None
        pot = np.zeros(n, np.float32) if save_force else None
        rc = KickReturn()
        flops = ctypes.c_double(0)
        err = self.lib.ct_or_kick(ctypes.c_int(order), ctypes.byref(params), ctypes.c_int(len(nodes)), _p(nodes), _p(x), _p(y), _p(z), _p(v),
                                  _p(rung), _p(gx), _p(gy), _p(gz), _p(pot), ctypes.byref(rc), ctypes.c_int(nthreads), ctypes.byref(flops))
        if err:
            raise RuntimeError("oracle kick error %d" % err)
        return (gx, gy, gz, pot), rc, flops.value

    def plan(self, params, nodes, x, y, z, order=7, max_parts=0, nthreads=0):
        """The kick split into work items (see KickPlan)."""
        return KickPlan(self, params, nodes, x, y, z, order, max_parts, nthreads)

    def drift(self, x, y, z, v, rung, which_rung, a, dt, drag=0.0):
        self.lib.ct_or_drift(ctypes.c_int(len(x)), _p(x), _p(y), _p(z), _p(v), _p(rung), ctypes.c_int(which_rung), ctypes.c_float(a),
                             ctypes.c_float(dt), ctypes.c_double(drag))

    def healpix_nest(self, nside, x, y, z):
        f = self.lib.ct_or_healpix_nest
        f.restype = ctypes.c_int
        return f(ctypes.c_int(nside), ctypes.c_double(x), ctypes.c_double(y), ctypes.c_double(z))

    def drift_lc(self, x, y, z, v, rung, which_rung, a, dt, tau0, tau1, tau_max, nside, drag=0.0, max_out=None):
        """Drift with the lightcone capture (in place); returns the entries (LC_ENTRY rows)."""
        f = self.lib.ct_or_drift_lc
        f.restype = ctypes.c_int64
        cap = max_out if max_out is not None else 8 * len(x)
        out = np.zeros(max(cap, 1), LC_ENTRY)
        cnt = f(ctypes.c_int(len(x)), _p(x), _p(y), _p(z), _p(v), _p(rung), ctypes.c_int(which_rung), ctypes.c_float(a), ctypes.c_float(dt),
                ctypes.c_double(drag), ctypes.c_float(tau0), ctypes.c_float(tau1), ctypes.c_float(tau_max), ctypes.c_int(nside), _p(out),
                ctypes.c_int64(cap))
        if cnt > cap:
            raise RuntimeError("oracle lightcone: %d entries, room for %d" % (cnt, cap))
        return out[:cnt]

    def sort_by_rung(self, x, y, z, v, rung, minrung, begin=0):
        return self.lib.ct_or_sort_by_rung(ctypes.c_int(len(x)), ctypes.c_int(begin), ctypes.c_int(minrung), _p(x), _p(y), _p(z), _p(v), _p(rung))

    def direct_ewald(self, x, y, z, sx, sy, sz, h, nthreads=0):
        ns = len(sx)
        out = [np.zeros(ns) for _ in range(4)]
        self.lib.ct_or_direct_ewald(ctypes.c_int(len(x)), _p(x), _p(y), _p(z), ctypes.c_int(ns), _p(sx), _p(sy), _p(sz), ctypes.c_double(h),
                                    *[_p(a) for a in out], ctypes.c_int(nthreads))
        return out


class KickPlan:
    """The top of the kick walk run once (all threads, level by level) and the subtrees below
    it kept as work items, ordered by first particle (ct_or_kick_plan_*).  `run` walks all items
    or a selection, kicking only the selected items' particles."""

    def __init__(self, O, params, nodes, x, y, z, order, max_parts, nthreads):
        L = O.lib
        L.ct_or_kick_plan_create.restype = ctypes.c_void_p
        self.O, self.params, self.nodes, self.x, self.y, self.z = O, params, nodes, x, y, z
        self.nthreads = nthreads
        n = ctypes.c_int64(0)
        ts = ctypes.c_double(0)
        self.h = L.ct_or_kick_plan_create(ctypes.c_int(order), ctypes.byref(params), ctypes.c_int(len(nodes)), _p(nodes), _p(x), _p(y), _p(z),
                                          ctypes.c_int(max_parts), ctypes.c_int(nthreads), ctypes.byref(n), ctypes.byref(ts))
        if not self.h:
            raise RuntimeError("oracle kick plan failed")
        self.nitems = n.value
        self.top_seconds = ts.value
        self.self = np.zeros(self.nitems, np.int32)
        self.nparts = np.zeros(self.nitems, np.int32)
        self.near_parts = np.zeros(self.nitems, np.int64)
        self.ewald_checks = np.zeros(self.nitems, np.int32)
        L.ct_or_kick_plan_items(ctypes.c_void_p(self.h), _p(self.self), _p(self.nparts), _p(self.near_parts), _p(self.ewald_checks))
        self.part_begin = nodes["part_begin"][self.self]

    def run(self, v, rung, select=None, save_force=True):
        """Walk the selected items (a boolean mask over items; None: all).  Returns
        ((gx, gy, gz, pot), kick return, flops, per-item seconds); unselected particles keep
        zero forces."""
        n = len(self.x)
        g = [np.zeros(n, np.float32) for _ in range(4)] if save_force else [None] * 4
        sel = None if select is None else np.ascontiguousarray(select, dtype=np.int8)
        secs = np.zeros(self.nitems)
        rc = KickReturn()
        flops = ctypes.c_double(0)
        err = self.O.lib.ct_or_kick_plan_run(ctypes.c_void_p(self.h), _p(v), _p(rung), *[_p(a) for a in g], _p(sel), ctypes.c_int(self.nthreads),
                                             _p(secs), ctypes.byref(rc), ctypes.byref(flops))
        if err:
            raise RuntimeError("oracle kick error %d" % err)
        return tuple(g), rc, flops.value, secs

    def export(self, nexp=50):
        """The items as the reference's kick_workitem fields: dict of self (int32), L (nitems,
        nexp) float32, pos (nitems, 3) uint32, and the direct / Ewald check lists in CSR form
        (doff, dlist, eoff, elist)."""
        L_ = self.O.lib
        nd, ne = ctypes.c_int64(0), ctypes.c_int64(0)
        L_.ct_or_kick_plan_list_sizes(ctypes.c_void_p(self.h), ctypes.byref(nd), ctypes.byref(ne))
        out = {"self": np.zeros(self.nitems, np.int32), "L": np.zeros((self.nitems, nexp), np.float32), "pos": np.zeros((self.nitems, 3), np.uint32),
               "doff": np.zeros(self.nitems + 1, np.int64), "dlist": np.zeros(max(nd.value, 1), np.int32),
               "eoff": np.zeros(self.nitems + 1, np.int64), "elist": np.zeros(max(ne.value, 1), np.int32)}
        L_.ct_or_kick_plan_export(ctypes.c_void_p(self.h), _p(out["self"]), _p(out["L"]), ctypes.c_int(nexp), _p(out["pos"]), _p(out["doff"]),
                                  _p(out["dlist"]), _p(out["eoff"]), _p(out["elist"]))
        return out

    def particles(self, select):
        """Indices of the particles of the selected items."""
        idx = np.nonzero(select)[0]
        return np.concatenate([np.arange(self.part_begin[i], self.part_begin[i] + self.nparts[i]) for i in idx]) if len(idx) else np.zeros(0, np.int64)

    def close(self):
        if self.h:
            self.O.lib.ct_or_kick_plan_destroy(ctypes.c_void_p(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_cached = None


def load(build=True):
    global _cached
    if _cached is not None:
        return _cached
    if build and _stale():
        subprocess.check_call(["make", "-s", "-C", ORACLE_DIR, "libct_oracle.so"])
    _cached = Oracle(LIB)
    return _cached


def step_hierarchical(O, st, sp, order=7, nthreads=0):
    """The oracle's hierarchical step (src/driver.cpp:382-593) over particle state `st`
    (dict with x, y, z, v, rung, rung_begin, stack) and step parameters `sp` (dict with the
    fields of ct_step_params).  Mirrors ct_step_hierarchical; returns (top kick return,
    minrung, max_rung)."""
    minrung = sp["minrung"]
    max_rung = max(sp["max_rung"], minrung)
    levels = list(range(max_rung, minrung, -1)) + [minrung]
    ascending, clip_top = True, False
    x, y, z, v, r = st["x"], st["y"], st["z"], st["v"], st["rung"]
    top_kr = None
    li = 0
    while li < len(levels):
        level = levels[li]
        top = level == minrung
        if top:
            ascending = False
        if not ascending and not top:
            st["stack"].append(st["rung_begin"])
        if not ascending:
            st["rung_begin"] = O.sort_by_rung(x, y, z, v, r, level, st["rung_begin"]) if level > 0 else 0
        if top and minrung == sp["minrung0"]:
            counts = np.bincount(np.clip(r, 0, 15), minlength=16)
            if np.nonzero(counts)[0].max() > sp["minrung0"]:
                fast = counts[sp["minrung0"] + 1:].sum()
                slow = counts[sp["minrung0"]]
                if 3 * fast > slow:
                    clip_top = not sp["nocrop"]
        nodes = O.tree_build(x, y, z, v, r, sp["theta"], sp["hsoft"], sp["bucket"], order=order, begin=st["rung_begin"])
        kp = KickParams(sign=sp["sign"], min_rung=level, a=sp["a"], t0=sp["t0"], theta=sp["theta"], h=sp["hsoft"], eta=sp["eta"], GM=sp["GM"],
                        max_dt=sp["max_dt"], save_force=0, first_call=int(sp["tau"] == 0.0), ascending=int(ascending or top),
                        descending=int(False if (clip_top and top) else ((not ascending) or top)),
                        top=int(True if (clip_top and level == sp["minrung0"] + 1) else top), do_phi=int(sp["do_phi"] and top))
        _, kr, _ = O.kick(kp, nodes, x, y, z, v, r, order=order, nthreads=nthreads, save_force=False)
        if clip_top and top:
            np.maximum(r, sp["minrung0"] + 1, out=r)
        if top:
            top_kr = kr
        if clip_top and top:
            levels.append(sp["minrung0"] + 1)
        elif (not ascending) or top:
            max_rung = kr.max_rung
            if max_rung > level:
                levels.append(level + 1)
        if ((not ascending) or top) and not (clip_top and top):
            O.drift(x, y, z, v, r, level, sp["a"], (1.0 / (1 << level)) * sp["t0"], sp["drag"])
        if ascending and not top:
            st["rung_begin"] = st["stack"].pop()
        li += 1
    if clip_top:
        minrung += 1
    return top_kr, minrung, max_rung


def pps_select(proxy, frac, rng, min_items=0):
    """Poisson sampling with inclusion probabilities pi_i = min(1, k proxy_i), k chosen so that
    the sample is expected to cover `frac` of the total proxy and to hold at least `min_items`
    items (so that a timed sample keeps every thread busy, as the full walk does): returns
    (mask, pi)."""
    proxy = np.maximum(np.asarray(proxy, np.float64), 1.0)
    tot = proxy.sum()
    if frac >= 1.0 or min_items >= len(proxy):
        return np.ones(len(proxy), bool), np.ones(len(proxy))
    lo, hi = 0.0, 1.0 / proxy.min()
    for _ in range(60):
        k = 0.5 * (lo + hi)
        p = np.minimum(1.0, k * proxy)
        if np.sum(p * proxy) / tot < frac or np.sum(p) < min_items:
            lo = k
        else:
            hi = k
    pi = np.minimum(1.0, hi * proxy)
    mask = rng.random(len(proxy)) < pi
    return mask, pi


def item_proxy(plan):
    """Cost proxy of each work item: particle pairs with the particles of its direct check list
    (the near field that becomes P2P, P2L and M2P work) plus its Ewald checks."""
    return plan.nparts.astype(np.float64) * (plan.near_parts.astype(np.float64) + 64.0) + 4000.0 * plan.ewald_checks


def walk_makespan(proxy, mask, pi, secs, nthreads):
    """Estimated wall time of walking all items on nthreads threads that take items in order
    from a shared counter (the oracle's parallel_for): the sampled items' measured times, the
    others' predicted from their cost proxy (ratio estimator), the greedy schedule simulated,
    and scaled so that the items' total equals the unbiased Horvitz-Thompson total."""
    import heapq

    proxy = np.maximum(np.asarray(proxy, np.float64), 1.0)
    total = float(np.sum(secs[mask] / pi[mask]))
    if total <= 0.0:
        return 0.0
    rest = proxy[~mask].sum()
    beta = (total - secs[mask].sum()) / rest if rest > 0 else 0.0
    t = np.where(mask, secs, max(beta, 0.0) * proxy)
    busy = [0.0] * nthreads
    for ti in t:
        heapq.heappush(busy, heapq.heappop(busy) + ti)
    span = max(busy)
    return span * total / max(float(t.sum()), 1e-300)


def estimate_step_hierarchical(O, st, sp, frac, seed, order=7, nthreads=0, max_parts=None):
    """One hierarchical step of the oracle (the ladder of step_hierarchical above, on state `st`)
    with every kick timed on a sample: the tree build over the active particles, the top of the
    walk and the rung sort and drift run in full; of the work items below the top a random
    subset is walked, chosen with probability proportional to a cost proxy, and the walk time
    of all items is estimated from it (the Horvitz-Thompson total, sum of t_i / pi_i over the
    sample, spread over the threads by walk_makespan's simulation of their schedule).
    Returns (estimated seconds, details); the state advances as the
    step moves it (unsampled particles keep their rungs and velocities)."""
    import time

    if nthreads <= 0:
        nthreads = os.cpu_count() or 1
    rng = np.random.default_rng(seed)
    minrung = sp["minrung"]
    max_rung = max(sp["max_rung"], minrung)
    levels = list(range(max_rung, minrung, -1)) + [minrung]
    ascending, clip_top = True, False
    x, y, z, v, r = st["x"], st["y"], st["z"], st["v"], st["rung"]
    n = len(x)
    est = {"tree": 0.0, "top": 0.0, "walk": 0.0, "walk_sampled": 0.0, "sort": 0.0, "drift": 0.0, "kicks": 0, "active": 0, "items": 0, "sampled_items": 0}
    li = 0
    while li < len(levels):
        level = levels[li]
        top = level == minrung
        if top:
            ascending = False
        if not ascending and not top:
            st["stack"].append(st["rung_begin"])
        if not ascending:
            t = time.perf_counter()
            st["rung_begin"] = O.sort_by_rung(x, y, z, v, r, level, st["rung_begin"]) if level > 0 else 0
            est["sort"] += time.perf_counter() - t
        if top and minrung == sp["minrung0"]:
            counts = np.bincount(np.clip(r, 0, 15), minlength=16)
            if np.nonzero(counts)[0].max() > sp["minrung0"]:
                fast = counts[sp["minrung0"] + 1:].sum()
                slow = counts[sp["minrung0"]]
                if 3 * fast > slow:
                    clip_top = not sp["nocrop"]
        b = st["rung_begin"]
        t = time.perf_counter()
        nodes = O.tree_build(x, y, z, v, r, sp["theta"], sp["hsoft"], sp["bucket"], order=order, begin=b, nthreads=nthreads)
        est["tree"] += time.perf_counter() - t
        kp = KickParams(sign=sp["sign"], min_rung=level, a=sp["a"], t0=sp["t0"], theta=sp["theta"], h=sp["hsoft"], eta=sp["eta"], GM=sp["GM"],
                        max_dt=sp["max_dt"], save_force=0, first_call=int(sp["tau"] == 0.0), ascending=int(ascending or top),
                        descending=int(False if (clip_top and top) else ((not ascending) or top)),
                        top=int(True if (clip_top and level == sp["minrung0"] + 1) else top), do_phi=int(sp["do_phi"] and top))
        active = n - b
        mp = max_parts if max_parts else max(256, active // 2048)
        plan = O.plan(kp, nodes, x, y, z, order=order, max_parts=mp, nthreads=nthreads)
        est["top"] += plan.top_seconds
        mask, pi = pps_select(item_proxy(plan), frac, rng, min_items=2 * nthreads)
        _, kr, _, secs = plan.run(v, r, select=mask, save_force=False)
        plan.close()
        est["walk"] += walk_makespan(item_proxy(plan), mask, pi, secs, nthreads)
        est["walk_sampled"] += float(np.sum(secs[mask]))
        est["kicks"] += 1
        est["active"] += active
        est["items"] += plan.nitems
        est["sampled_items"] += int(mask.sum())
        if clip_top and top:
            np.maximum(r, sp["minrung0"] + 1, out=r)
        if clip_top and top:
            levels.append(sp["minrung0"] + 1)
        elif (not ascending) or top:
            # the rung ladder follows the highest rung; unsampled particles keep theirs
            max_rung = max(kr.max_rung, int(r[b:].max()) if active else 0)
            if max_rung > level:
                levels.append(level + 1)
        if ((not ascending) or top) and not (clip_top and top):
            t = time.perf_counter()
            O.drift(x, y, z, v, r, level, sp["a"], (1.0 / (1 << level)) * sp["t0"], sp["drag"])
            est["drift"] += time.perf_counter() - t
        if ascending and not top:
            st["rung_begin"] = st["stack"].pop()
        li += 1
    if clip_top:
        minrung += 1
    st["minrung"], st["max_rung"] = minrung, max_rung
    seconds = est["tree"] + est["top"] + est["walk"] + est["sort"] + est["drift"]
    est["threads"] = nthreads
    return seconds, est


def rung_state_from_forces(O, st, g, t0, eta, h, a=1.0, minrung0=0):
    """Rungs of a state whose forces g (N, 3) are known, by the rung rule of do_kick
    (dt = min(eta sqrt(a h / |g|), t0), rung = ceil(log2(t0 / dt)); kick.cu:133-140) applied
    with the full forces at every level of the first step's descending ladder; the lowest rung
    is raised as the ladder's top clip raises it (driver.cpp:442-462), and the active range and
    rung stack are those the descending partitions leave (particles_push_rungs before each
    particles_sort_by_rung).  Fills st's rung, rung_begin and stack; returns (minrung, max_rung)."""
    gm = np.sqrt(np.sum(np.asarray(g, np.float64) ** 2, axis=1))
    dt = np.minimum(eta * np.sqrt(a * h / np.maximum(gm, 1e-300)), t0)
    lv = np.ceil(np.log2(t0 / dt) - 1e-12)
    rung = np.clip(lv, minrung0, 15).astype(np.int8)
    counts = np.bincount(rung, minlength=16)
    minrung = minrung0
    if counts[minrung0 + 1:].sum() * 3 > counts[minrung0] and counts[minrung0 + 1:].sum() > 0:
        rung = np.maximum(rung, minrung0 + 1).astype(np.int8)
        minrung = minrung0 + 1
    st["rung"][:] = rung
    max_rung = int(rung.max())
    st["rung_begin"] = 0
    st["stack"] = []
    x, y, z, v, r = st["x"], st["y"], st["z"], st["v"], st["rung"]
    for level in range(minrung + 1, max_rung + 1):
        st["stack"].append(st["rung_begin"])
        st["rung_begin"] = O.sort_by_rung(x, y, z, v, r, level, st["rung_begin"])
    return minrung, max_rung
