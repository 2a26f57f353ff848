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
    def tree_build(self, x, y, z, v, rung, theta, hsoft, bucket=128, order=7, begin=0):
        n = len(x)
        max_nodes = max(64, 8 * n // max(bucket // 4, 1) + 1024)
        while True:
            nodes = np.zeros(max_nodes, NODE_DTYPE)
            cnt = self.lib.ct_or_tree_build(
                ctypes.c_int(order), ctypes.c_int(n), ctypes.c_int(begin), _p(x), _p(y), _p(z), _p(v), _p(rung),
                ctypes.c_double(theta), ctypes.c_double(hsoft), ctypes.c_int(bucket), _p(nodes), ctypes.c_int(max_nodes))
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

    def kick_sampled(self, params, nodes, x, y, z, v, rung, stride, order=7, nthreads=0):
        """Kick of every stride-th top-level work item; returns (seconds, particles kicked, flops)."""
        import time

        n = len(x)
        g = [np.zeros(n, np.float32) for _ in range(4)]
        rc = KickReturn()
        flops = ctypes.c_double(0)
        sampled = ctypes.c_int64(0)
        t = time.perf_counter()
        err = self.lib.ct_or_kick_sampled(ctypes.c_int(order), ctypes.byref(params), ctypes.c_int(len(nodes)), _p(nodes), _p(x), _p(y), _p(z), _p(v),
                                          _p(rung), *[_p(a) for a in g], ctypes.byref(rc), ctypes.c_int(nthreads), ctypes.byref(flops),
                                          ctypes.c_int(stride), ctypes.byref(sampled))
        dt = time.perf_counter() - t
        if err:
            raise RuntimeError("oracle kick error %d" % err)
        return dt, sampled.value, flops.value

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
