"""ctypes binding of oracle/_ref/libctref_gpu.so: the reference's own CUDA kick and drift
(src/kick.cu, src/gravity.cu, src/drift.cu and the rest of its device code, compiled from the
reference's sources for sm_100a by `make -C oracle refgpu`) behind a small host harness
(oracle/ref_gpu_shim.cu).  Test infrastructure only.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "libctref_gpu.so")


class RefKickParams(ctypes.Structure):
    """kick_params fields in the reference's meaning (cosmictiger/kick.hpp:138-186)."""
    _fields_ = [("sign", ctypes.c_float), ("min_rung", ctypes.c_int), ("a", ctypes.c_float), ("t0", ctypes.c_float), ("theta", ctypes.c_float),
                ("h", ctypes.c_float), ("eta", ctypes.c_float), ("GM", ctypes.c_float), ("max_dt", ctypes.c_float), ("save_force", ctypes.c_int),
                ("first_call", ctypes.c_int), ("ascending", ctypes.c_int), ("descending", ctypes.c_int), ("top", ctypes.c_int), ("do_phi", ctypes.c_int)]


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def available():
    return os.path.exists(LIB)


class ReferenceGPU:
    """The reference's device heap (cuda_mem_init) is set up once per process, with the size of
    the first instance.  Its allocator traps the kernel when the heap runs out
    (device_vector.hpp:197-200), so the default is far above what the kernel's lists take:
    about 80 KB per resident warp of the kick grid (20 x 148 warps on a B200) for the
    production work items, a few MB for the single-root walk; managed memory, populated only
    where it is touched."""

    def __init__(self, heap_bytes=8 << 30):
        L = ctypes.CDLL(LIB)
        vp, i64 = ctypes.c_void_p, ctypes.c_int64
        L.ctref_init.argtypes = [ctypes.c_double]
        L.ctref_kick.argtypes = [i64, vp, vp, vp, vp, vp, i64, vp, ctypes.POINTER(RefKickParams), vp, vp, vp, vp, vp]
        L.ctref_drift.argtypes = [i64, i64, vp, vp, vp, vp, vp, ctypes.c_int, ctypes.c_float, ctypes.c_float]
        rc = L.ctref_init(float(heap_bytes))
        if rc != 0:
            raise RuntimeError("reference harness set-up failed (%d)" % rc)
        self.lib = L

    def kick(self, state, nodes, params):
        """Kick every particle with the reference's kernel (whole walk from the root).
        state: tree-ordered x, y, z (uint32), v (float32 (n,3)), rung (int8); nodes: the tree
        as exported by Box.tree() (breadth-first, root first)."""
        x, y, z = (np.ascontiguousarray(state[k], np.uint32) for k in "xyz")
        v = np.ascontiguousarray(state["v"], np.float32).copy()
        r = np.ascontiguousarray(state["rung"], np.int8).copy()
        n = len(x)
        g = [np.zeros(n, np.float32) for _ in range(4)]
        ret = np.zeros(8)
        nodes = np.ascontiguousarray(nodes)
        rc = self.lib.ctref_kick(n, _p(x), _p(y), _p(z), _p(v), _p(r), len(nodes), _p(nodes), ctypes.byref(params), *[_p(a) for a in g], _p(ret))
        if rc != 0:
            raise RuntimeError("reference kick failed (%d)" % rc)
        return {"v": v, "rung": r, "gx": g[0], "gy": g[1], "gz": g[2], "pot": g[3], "max_rung": int(ret[0]), "pot_sum": ret[1], "kin": ret[2]}

    def kick_block_count(self):
        """Blocks of the reference's kick grid (occupancy x SMs)."""
        self.lib.ctref_kick_block_count.restype = ctypes.c_int
        return int(self.lib.ctref_kick_block_count())

    def max_parts(self, active, bucket=128):
        """Largest subtree the reference's CPU top hands to the GPU (kick.cpp:173-177,
        CUDA_KICK_PARTS_MAX 16384, defs.hpp:71)."""
        return int(min(16384, max(active // max(self.kick_block_count(), 1), bucket)))

    def kick_items(self, state, nodes, params, items, repeats=2):
        """The reference's kick in production form: cuda_execute_kicks on work items (a dict as
        tests/oracle_lib.KickPlan.export returns: the subtrees below the CPU top of the walk with
        their parent expansions and check lists) over `nodes` (ct_node layout, which the items
        index).  The kick runs `repeats` times in a row on one particle copy; returns the last
        call's results and every call's milliseconds (CUDA events around cuda_execute_kicks)."""
        x, y, z = (np.ascontiguousarray(state[k], np.uint32) for k in "xyz")
        v = np.ascontiguousarray(state["v"], np.float32).copy()
        r = np.ascontiguousarray(state["rung"], np.int8).copy()
        n = len(x)
        g = [np.zeros(n, np.float32) for _ in range(4)]
        ret = np.zeros(8)
        ms = np.zeros(repeats, np.float32)
        nodes = np.ascontiguousarray(nodes)
        it = {k: np.ascontiguousarray(items[k]) for k in ("self", "L", "pos", "doff", "dlist", "eoff", "elist")}
        f = self.lib.ctref_kick_items
        vp, i64 = ctypes.c_void_p, ctypes.c_int64
        f.argtypes = [i64, vp, vp, vp, vp, vp, i64, vp, ctypes.POINTER(RefKickParams), i64, vp, vp, vp, vp, vp, vp, vp, ctypes.c_int, vp, vp, vp, vp, vp, vp]
        rc = f(n, _p(x), _p(y), _p(z), _p(v), _p(r), len(nodes), _p(nodes), ctypes.byref(params), len(it["self"]), _p(it["self"]), _p(it["L"]),
               _p(it["pos"]), _p(it["doff"]), _p(it["dlist"]), _p(it["eoff"]), _p(it["elist"]), int(repeats), *[_p(a) for a in g], _p(ret), _p(ms))
        if rc != 0:
            raise RuntimeError("reference kick (work items) failed (%d)" % rc)
        return {"v": v, "rung": r, "gx": g[0], "gy": g[1], "gz": g[2], "pot": g[3], "max_rung": int(ret[0]), "pot_sum": ret[1], "kin": ret[2],
                "ms": [float(q) for q in ms]}

    def drift_lc(self, x, y, z, v, rung, level, a, dt, tau0, tau1, tau_max, nside, create_glass=False, rung_begin=0, max_out=None):
        """The reference's drift with its lightcone capture; returns (x, y, z, v, entries)."""
        from tests.oracle_lib import LC_ENTRY

        x, y, z = (np.ascontiguousarray(q, np.uint32).copy() for q in (x, y, z))
        v = np.ascontiguousarray(v, np.float32).copy()
        rung = np.ascontiguousarray(rung, np.int8)
        cap = max_out if max_out is not None else 8 * len(x)
        out = np.zeros(max(cap, 1), LC_ENTRY)
        nout = ctypes.c_int64(0)
        f = self.lib.ctref_drift_lc
        f.argtypes = [ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                      ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                      ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]
        rc = f(len(x), rung_begin, _p(x), _p(y), _p(z), _p(v), _p(rung), level, a, dt, tau0, tau1, tau_max, nside, int(create_glass), _p(out), cap,
               ctypes.byref(nout))
        if rc != 0:
            raise RuntimeError("reference lightcone drift failed (%d)" % rc)
        if nout.value > cap:
            raise RuntimeError("reference lightcone: %d entries, room for %d" % (nout.value, cap))
        return x, y, z, v, out[:nout.value]

    def drift(self, x, y, z, v, rung, level, a, dt, rung_begin=0):
        """Drift (in place on copies) the particles in [rung_begin, n) of rung `level`."""
        x, y, z = (np.ascontiguousarray(q, np.uint32).copy() for q in (x, y, z))
        v = np.ascontiguousarray(v, np.float32)
        rung = np.ascontiguousarray(rung, np.int8)
        rc = self.lib.ctref_drift(len(x), rung_begin, _p(x), _p(y), _p(z), _p(v), _p(rung), level, a, dt)
        if rc != 0:
            raise RuntimeError("reference drift failed (%d)" % rc)
        return x, y, z
