"""B200-native gravity step of CosmicTiger: tree build, kick, drift behind a C ABI.

The compute path is libct_gravity.so (hand-written sm_100a CUDA, include/ct_gravity.h).  This
module is the host-side mirror of the reference's call surface for that path:

    reference (dmarce1/cosmictiger)                      here
    particles_sort_by_rung(minrung)  particles.cpp:1029   Box.sort_by_rung(minrung)
    tree_create(tree_create_params)  tree.cpp:273         Box.tree_create(theta, hsoft, bucket, min_rung)
    kick(kick_params, L, pos, root, {root}, {root})       Box.kick(KickParams) -> KickReturn
                                     kick.cpp:150
    drift(scale, dt, ..., rung)      drift.cpp:33         Box.drift(rung, a, dt, drag)

There is no CPU fallback: importing works without a GPU, but creating a Context requires the
built library and a CUDA device and raises otherwise.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libct_gravity.so")

CT_OK = 0
_ERRORS = {-1: "invalid argument", -2: "CUDA error", -3: "out of device memory / HBM budget", -4: "capacity exceeded", -5: "call out of order"}


class GravityError(RuntimeError):
    pass


class KickParams(ctypes.Structure):
    """Mirror of kick_params (cosmictiger/kick.hpp:138-186)."""

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

    @classmethod
    def make(cls, theta, h, GM, eta, min_rung=0, a=1.0, t0=1.0, max_dt=1e30, save_force=True, first_call=True, ascending=True,
             descending=True, top=True, do_phi=True, sign=1.0):
        return cls(sign=sign, min_rung=min_rung, a=a, t0=t0, theta=theta, h=h, eta=eta, GM=GM, max_dt=max_dt, save_force=int(save_force),
                   first_call=int(first_call), ascending=int(ascending), descending=int(descending), top=int(top), do_phi=int(do_phi))


class KickReturn(ctypes.Structure):
    """Mirror of kick_return (cosmictiger/kick.hpp:92-136)."""

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


class TreeParams(ctypes.Structure):
    _fields_ = [("min_rung", ctypes.c_int), ("theta", ctypes.c_double), ("hsoft", ctypes.c_double), ("bucket", ctypes.c_int)]


class StepParams(ctypes.Structure):
    """Parameters of one hierarchical step (kick_step_hierarchical, src/driver.cpp:382)."""

    _fields_ = [("minrung", ctypes.c_int), ("minrung0", ctypes.c_int), ("max_rung", ctypes.c_int), ("a", ctypes.c_double), ("tau", ctypes.c_double),
                ("t0", ctypes.c_double), ("theta", ctypes.c_double), ("hsoft", ctypes.c_double), ("bucket", ctypes.c_int), ("eta", ctypes.c_float),
                ("GM", ctypes.c_float), ("max_dt", ctypes.c_float), ("do_phi", ctypes.c_int), ("nocrop", ctypes.c_int), ("drag", ctypes.c_double),
                ("sign", ctypes.c_float)]


class StepReturn(ctypes.Structure):
    _fields_ = [("kr", KickReturn), ("minrung", ctypes.c_int), ("max_rung", ctypes.c_int), ("particles_kicked", ctypes.c_double), ("kicks", ctypes.c_int),
                ("particles_drifted_levels", ctypes.c_int)]


class Tuning(ctypes.Structure):
    """Mirror of ct_tuning: P2P cell-list size, warps per sink tile, sinks per tile."""

    _fields_ = [("p2p_stage", ctypes.c_int), ("warps_per_tile", ctypes.c_int), ("tile_width", ctypes.c_int)]


class Counters(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in (
        "pp_pairs", "cc_direct", "cc_ewald", "cp_pairs", "pc_pairs", "nodes", "leaves", "flops", "flops_pp", "flops_cc",
        "ms_tree", "ms_walk", "ms_m2l", "ms_l2l", "ms_leaf", "ms_drift", "ms_leafkick", "pp_near")]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


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

# one lightcone crossing (ct_lc_entry; the reference's lc_entry, cosmictiger/lightcone.hpp:54-58):
# position fixed<int,31> relative to the observer, velocity after drag, HEALPix nested pixel
LC_ENTRY = np.dtype([("x", "<i4"), ("y", "<i4"), ("z", "<i4"), ("vx", "<f4"), ("vy", "<f4"), ("vz", "<f4"), ("pix", "<i4")])


class LcParams(ctypes.Structure):
    _fields_ = [("tau0", ctypes.c_float), ("tau1", ctypes.c_float), ("tau_max", ctypes.c_float), ("nside", ctypes.c_int)]


class ICParams(ctypes.Structure):
    _fields_ = [("nfour", ctypes.c_int), ("box_size", ctypes.c_double), ("omega_m", ctypes.c_double), ("z0", ctypes.c_double),
                ("hubble", ctypes.c_double), ("sigma8", ctypes.c_double), ("H0", ctypes.c_double), ("twolpt", ctypes.c_int),
                ("table_k", ctypes.c_void_p), ("table_p", ctypes.c_void_p), ("ntable", ctypes.c_int)]


class ICReturn(ctypes.Structure):
    _fields_ = [("D1", ctypes.c_double), ("D2", ctypes.c_double), ("prefac1", ctypes.c_double), ("prefac2", ctypes.c_double),
                ("norm", ctypes.c_double), ("dxmax", ctypes.c_float * 3), ("dxmax2", ctypes.c_float * 3)]


_lib = None


def library():
    """Load libct_gravity.so; raises if it is missing (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise GravityError("libct_gravity.so is not built (run __graft_entry__.build() or python cosmictiger_b200/build.py)")
    L = ctypes.CDLL(LIB_PATH)
    vp, i64, i32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int
    L.ct_ctx_create.argtypes = [ctypes.POINTER(vp), i32, ctypes.c_size_t, i32]
    L.ct_ctx_destroy.argtypes = [vp]
    L.ct_ctx_destroy.restype = None
    L.ct_last_error.argtypes = [vp]
    L.ct_last_error.restype = ctypes.c_char_p
    L.ct_box_create.argtypes = [vp, i64, ctypes.POINTER(i32)]
    L.ct_box_destroy.argtypes = [vp, i32]
    L.ct_box_size.argtypes = [vp, i32]
    L.ct_box_size.restype = i64
    L.ct_box_upload.argtypes = [vp, i32, vp, vp, vp, vp, vp]
    L.ct_box_upload_device.argtypes = [vp, i32, vp, vp, vp, vp, vp]
    L.ct_box_download.argtypes = [vp, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    L.ct_box_download_device.argtypes = [vp, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    L.ct_sort_by_rung.argtypes = [vp, i32, i32, ctypes.POINTER(i64)]
    L.ct_ctx_set_compensated.argtypes = [vp, i32]
    L.ct_ctx_set_priority.argtypes = [vp, i32]
    L.ct_ensemble_reshape.argtypes = [vp, i32, i32, ctypes.POINTER(i64)]
    L.ct_box_get_rung_state.argtypes = [vp, i32, ctypes.POINTER(i64), vp, ctypes.POINTER(i32)]
    L.ct_box_set_rung_state.argtypes = [vp, i32, i64, vp, i32]
    L.ct_tree_create.argtypes = [vp, i32, ctypes.POINTER(TreeParams), ctypes.POINTER(i64)]
    L.ct_kick.argtypes = [vp, i32, ctypes.POINTER(KickParams), ctypes.POINTER(KickReturn)]
    L.ct_drift.argtypes = [vp, i32, i32, ctypes.c_float, ctypes.c_float, ctypes.c_double]
    L.ct_tree_download.argtypes = [vp, i32, vp, i64, ctypes.POINTER(i64)]
    L.ct_get_counters.argtypes = [vp, i32, ctypes.POINTER(Counters)]
    L.ct_synchronize.argtypes = [vp]
    L.ct_ensemble_create.argtypes = [vp, i32, ctypes.POINTER(i64), ctypes.POINTER(i32)]
    L.ct_box_count.argtypes = [vp, i32]
    L.ct_ensemble_set_params.argtypes = [vp, i32, vp, vp]
    L.ct_kick_ensemble.argtypes = [vp, i32, ctypes.POINTER(KickParams), ctypes.POINTER(KickReturn)]
    L.ct_ensemble_set_first_call.argtypes = [vp, i32, vp]
    L.ct_ensemble_gather.argtypes = [vp, i32, ctypes.POINTER(i32), i32]
    L.ct_ensemble_scatter.argtypes = [vp, i32, ctypes.POINTER(i32), i32]
    L.ct_bytes_in_use.argtypes = [vp]
    L.ct_bytes_in_use.restype = ctypes.c_size_t
    L.ct_step_hierarchical.argtypes = [vp, i32, ctypes.POINTER(StepParams), ctypes.POINTER(StepReturn)]
    L.ct_rung_counts.argtypes = [vp, i32, vp]
    L.ct_launch_count.argtypes = [vp]
    L.ct_launch_count.restype = ctypes.c_ulonglong
    L.ct_order.argtypes = [vp]
    L.ct_stream.argtypes = [vp]
    L.ct_stream.restype = vp  # a cudaStream_t: a 64-bit handle, not an int
    L.ct_fp32_peak.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
    L.ct_ctx_set_tuning.argtypes = [vp, ctypes.POINTER(Tuning)]
    L.ct_ctx_get_tuning.argtypes = [vp, ctypes.POINTER(Tuning)]
    L.ct_sort_by_rung_noalloc.argtypes = [i64, i64, i32, vp, vp, vp, vp, vp, vp, vp, ctypes.POINTER(i64), vp]
    L.ct_direct_ewald.argtypes = [vp, i32, i64, vp, vp, vp, ctypes.c_double, vp, vp, vp, vp]
    L.ct_drift_lightcone.argtypes = [vp, i32, i32, ctypes.c_float, ctypes.c_float, ctypes.c_double, ctypes.POINTER(LcParams), ctypes.POINTER(i64)]
    L.ct_lightcone_count.argtypes = [vp, i32, ctypes.POINTER(i64)]
    L.ct_lightcone_download.argtypes = [vp, i32, vp, i64, ctypes.POINTER(i64), i32]
    L.ct_lightcone_reserve.argtypes = [vp, i32, i64]
    L.ct_initialize.argtypes = [vp, i32, ctypes.POINTER(ICParams), ctypes.POINTER(ICReturn)]
    fp = ctypes.POINTER(ctypes.c_float)
    L.ct_power_spectrum.argtypes = [vp, i32, i32, i32, ctypes.c_double, i32, vp, vp, vp, ctypes.POINTER(i32)]
    _lib = L
    return L


def _p(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data if isinstance(a, np.ndarray) else int(a))


class Context:
    """One device, one stream, device-resident boxes (ct_ctx_create)."""

    def __init__(self, device=0, hbm_budget=0, order=7):
        self.lib = library()
        h = ctypes.c_void_p()
        rc = self.lib.ct_ctx_create(ctypes.byref(h), device, hbm_budget, order)
        if rc != CT_OK:
            raise GravityError("ct_ctx_create failed (%s)" % _ERRORS.get(rc, rc))
        self.h = h
        self.order = order

    def check(self, rc, what):
        if rc != CT_OK:
            raise GravityError("%s: %s (%s)" % (what, self.lib.ct_last_error(self.h).decode(), _ERRORS.get(rc, rc)))

    def box(self, n):
        return Box(self, n)

    def ensemble(self, counts):
        """Independent periodic boxes handled together (ct_ensemble_create)."""
        return Box(self, int(np.sum(counts)), counts=counts)

    def bytes_in_use(self):
        return int(self.lib.ct_bytes_in_use(self.h))

    def launches(self):
        """Kernels of libct_gravity launched on this context so far."""
        return int(self.lib.ct_launch_count(self.h))

    def set_tuning(self, p2p_stage=128, warps_per_tile=1, tile_width=32):
        """Launch shape of the P2P and leaf-kick kernels (ct_ctx_set_tuning)."""
        t = Tuning(p2p_stage, warps_per_tile, tile_width)
        self.check(self.lib.ct_ctx_set_tuning(self.h, ctypes.byref(t)), "ct_ctx_set_tuning")

    def tuning(self):
        t = Tuning()
        self.check(self.lib.ct_ctx_get_tuning(self.h, ctypes.byref(t)), "ct_ctx_get_tuning")
        return {"p2p_stage": t.p2p_stage, "warps_per_tile": t.warps_per_tile, "tile_width": t.tile_width}

    def set_priority(self, priority):
        """CUDA stream priority of the context (0 default and lowest, negative higher; clamped
        to the device's range).  Drains the context and replaces its streams."""
        self.check(self.lib.ct_ctx_set_priority(self.h, int(priority)), "ct_ctx_set_priority")

    def set_compensated(self, on):
        """Neumaier-compensated (True, default) or plain FP32 sums of the P2P source batches."""
        self.check(self.lib.ct_ctx_set_compensated(self.h, int(bool(on))), "ct_ctx_set_compensated")

    def synchronize(self):
        self.check(self.lib.ct_synchronize(self.h), "ct_synchronize")

    def stream_handle(self):
        """The context's cudaStream_t as an integer (ct_stream), e.g. for
        torch.cuda.ExternalStream, to order other work or events with the library's."""
        return int(self.lib.ct_stream(self.h) or 0)

    def fp32_peak(self):
        """Measured FP32 FMA throughput of the device, TFLOP/s (ct_fp32_peak)."""
        pk = ctypes.c_double(0)
        self.check(self.lib.ct_fp32_peak(self.h, ctypes.byref(pk)), "ct_fp32_peak")
        return pk.value

    def device_order(self):
        """Expansion order the context was created with (ct_order)."""
        return int(self.lib.ct_order(self.h))

    def close(self):
        if getattr(self, "h", None):
            self.lib.ct_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Box:
    """A periodic unit box of particles with its tree, resident on the device."""

    def __init__(self, ctx, n, counts=None):
        self.ctx = ctx
        self.n = int(n)
        bid = ctypes.c_int()
        if counts is None:
            ctx.check(ctx.lib.ct_box_create(ctx.h, self.n, ctypes.byref(bid)), "ct_box_create")
            self.counts = np.array([self.n], np.int64)
        else:
            self.counts = np.ascontiguousarray(counts, np.int64)
            ctx.check(ctx.lib.ct_ensemble_create(ctx.h, len(self.counts), self.counts.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), ctypes.byref(bid)),
                      "ct_ensemble_create")
        self.id = bid.value
        self.tree_params = None

    @property
    def nbox(self):
        return len(self.counts)

    def set_box_params(self, h, GM):
        """Per-box softening and GM of an ensemble."""
        h = np.ascontiguousarray(h, np.float32)
        GM = np.ascontiguousarray(GM, np.float32)
        self.ctx.check(self.ctx.lib.ct_ensemble_set_params(self.ctx.h, self.id, _p(h), _p(GM)), "ct_ensemble_set_params")

    def reshape(self, counts):
        """Re-batch an ensemble in place for boxes of `counts` particles (ct_ensemble_reshape);
        device arrays are reused while they are large enough."""
        c = np.ascontiguousarray(counts, np.int64)
        self.ctx.check(self.ctx.lib.ct_ensemble_reshape(self.ctx.h, self.id, len(c), c.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))),
                       "ct_ensemble_reshape")
        self.counts = c
        self.n = int(np.sum(c))
        self.tree_params = None

    def rung_state(self):
        """(active range start, saved starts of the enclosing ranges) of the rung ladder."""
        rb = ctypes.c_int64()
        depth = ctypes.c_int(0)
        self.ctx.check(self.ctx.lib.ct_box_get_rung_state(self.ctx.h, self.id, ctypes.byref(rb), None, ctypes.byref(depth)), "ct_box_get_rung_state")
        stack = np.zeros(max(depth.value, 1), np.int64)
        self.ctx.check(self.ctx.lib.ct_box_get_rung_state(self.ctx.h, self.id, ctypes.byref(rb), _p(stack), ctypes.byref(depth)), "ct_box_get_rung_state")
        return int(rb.value), [int(q) for q in stack[:depth.value]]

    def set_rung_state(self, rung_begin, stack):
        s = np.ascontiguousarray(stack if len(stack) else [0], np.int64)
        self.ctx.check(self.ctx.lib.ct_box_set_rung_state(self.ctx.h, self.id, int(rung_begin), _p(s), len(stack)), "ct_box_set_rung_state")

    def set_first_call(self, flags):
        f = np.ascontiguousarray(flags, np.int32)
        self.ctx.check(self.ctx.lib.ct_ensemble_set_first_call(self.ctx.h, self.id, _p(f)), "ct_ensemble_set_first_call")

    def gather(self, boxes):
        """Copy plain boxes (device-resident) into this ensemble's slots."""
        ids = (ctypes.c_int * len(boxes))(*[b.id for b in boxes])
        self.ctx.check(self.ctx.lib.ct_ensemble_gather(self.ctx.h, self.id, ids, len(boxes)), "ct_ensemble_gather")

    def scatter(self, boxes):
        """Copy this ensemble's slots back into plain boxes."""
        ids = (ctypes.c_int * len(boxes))(*[b.id for b in boxes])
        self.ctx.check(self.ctx.lib.ct_ensemble_scatter(self.ctx.h, self.id, ids, len(boxes)), "ct_ensemble_scatter")

    def kick_ensemble(self, params):
        """Per-box kick returns of an ensemble."""
        out = (KickReturn * self.nbox)()
        self.ctx.check(self.ctx.lib.ct_kick_ensemble(self.ctx.h, self.id, ctypes.byref(params), out), "ct_kick_ensemble")
        return list(out)

    def upload(self, x, y, z, vxyz, rung):
        """Host arrays: x,y,z uint32 fixed32; vxyz float32 (n,3); rung int8."""
        arrs = [np.ascontiguousarray(x, np.uint32), np.ascontiguousarray(y, np.uint32), np.ascontiguousarray(z, np.uint32),
                np.ascontiguousarray(vxyz, np.float32), np.ascontiguousarray(rung, np.int8)]
        for a in arrs[:3] + [arrs[4]]:
            if a.shape[0] != self.n:
                raise ValueError("array length differs from the box size")
        self.ctx.check(self.ctx.lib.ct_box_upload(self.ctx.h, self.id, *[_p(a) for a in arrs]), "ct_box_upload")

    def upload_device(self, x, y, z, vxyz, rung):
        """Device pointers (e.g. torch tensor data_ptr()) with the same layout."""
        self.ctx.check(self.ctx.lib.ct_box_upload_device(self.ctx.h, self.id, *[_p(a) for a in (x, y, z, vxyz, rung)]), "ct_box_upload_device")

    def download_device(self, x, y, z, vxyz, rung, gx=None, gy=None, gz=None, pot=None):
        """Copy the box's particles into device buffers the caller holds (data_ptr() integers or
        None to skip a field); gx..pot only after a kick with save_force."""
        ptrs = [_p(a) for a in (x, y, z, vxyz, rung, gx, gy, gz, pot)]
        self.ctx.check(self.ctx.lib.ct_box_download_device(self.ctx.h, self.id, *ptrs), "ct_box_download_device")

    def size(self):
        """Particles held by the box (ct_box_size)."""
        return int(self.ctx.lib.ct_box_size(self.ctx.h, self.id))

    def box_count(self):
        """Boxes in an ensemble, 1 for a plain box (ct_box_count)."""
        return int(self.ctx.lib.ct_box_count(self.ctx.h, self.id))

    def download(self, forces=False):
        n = self.n
        x, y, z = (np.empty(n, np.uint32) for _ in range(3))
        v = np.empty((n, 3), np.float32)
        r = np.empty(n, np.int8)
        g = [np.empty(n, np.float32) for _ in range(4)] if forces else [None] * 4
        self.ctx.check(self.ctx.lib.ct_box_download(self.ctx.h, self.id, _p(x), _p(y), _p(z), _p(v), _p(r), *[_p(a) for a in g]), "ct_box_download")
        out = {"x": x, "y": y, "z": z, "v": v, "rung": r}
        if forces:
            out.update(gx=g[0], gy=g[1], gz=g[2], pot=g[3])
        return out

    def sort_by_rung(self, min_rung):
        rb = ctypes.c_int64()
        self.ctx.check(self.ctx.lib.ct_sort_by_rung(self.ctx.h, self.id, min_rung, ctypes.byref(rb)), "ct_sort_by_rung")
        return rb.value

    def tree_create(self, theta, hsoft, bucket=128, min_rung=0):
        p = TreeParams(min_rung=min_rung, theta=theta, hsoft=hsoft, bucket=bucket)
        cnt = ctypes.c_int64()
        self.ctx.check(self.ctx.lib.ct_tree_create(self.ctx.h, self.id, ctypes.byref(p), ctypes.byref(cnt)), "ct_tree_create")
        self.tree_params = p
        return cnt.value

    def kick(self, params):
        rc = KickReturn()
        self.ctx.check(self.ctx.lib.ct_kick(self.ctx.h, self.id, ctypes.byref(params), ctypes.byref(rc)), "ct_kick")
        return rc

    def step_hierarchical(self, params):
        """One multistep step over the rung ladder; returns StepReturn."""
        r = StepReturn()
        self.ctx.check(self.ctx.lib.ct_step_hierarchical(self.ctx.h, self.id, ctypes.byref(params), ctypes.byref(r)), "ct_step_hierarchical")
        return r

    def rung_counts(self):
        c = np.zeros(16, np.uint64)
        self.ctx.check(self.ctx.lib.ct_rung_counts(self.ctx.h, self.id, _p(c)), "ct_rung_counts")
        return c

    def drift(self, rung, a, dt, drag=0.0):
        self.ctx.check(self.ctx.lib.ct_drift(self.ctx.h, self.id, rung, a, dt, drag), "ct_drift")

    def drift_lightcone(self, rung, a, dt, tau0, tau1, tau_max, nside, drag=0.0):
        """Drift with the lightcone capture (cuda_drift with do_lc); returns this call's count."""
        p = LcParams(tau0, tau1, tau_max, nside)
        n = ctypes.c_int64()
        self.ctx.check(self.ctx.lib.ct_drift_lightcone(self.ctx.h, self.id, rung, a, dt, drag, ctypes.byref(p), ctypes.byref(n)), "ct_drift_lightcone")
        return n.value

    def lightcone(self, clear=True):
        """The captured entries (LC_ENTRY rows); clear empties the device buffer."""
        n = ctypes.c_int64()
        self.ctx.check(self.ctx.lib.ct_lightcone_count(self.ctx.h, self.id, ctypes.byref(n)), "ct_lightcone_count")
        out = np.zeros(n.value, LC_ENTRY)
        self.ctx.check(self.ctx.lib.ct_lightcone_download(self.ctx.h, self.id, _p(out), n.value, ctypes.byref(n), int(clear)), "ct_lightcone_download")
        return out

    def initialize(self, nfour, box_size, table_k, table_p, omega_m=0.3111, z0=49.0, hubble=0.6732, sigma8=0.8607, H0=1.0, twolpt=True):
        """Lattice + Zel'dovich (+ 2LPT) initial conditions from a power.init table (k in h/Mpc,
        P in (Mpc/h)^3); returns the factors and largest displacements (ICReturn as a dict)."""
        k = np.ascontiguousarray(table_k, np.float32)
        P = np.ascontiguousarray(table_p, np.float32)
        prm = ICParams(nfour, box_size, omega_m, z0, hubble, sigma8, H0, int(twolpt), _p(k).value, _p(P).value, len(k))
        r = ICReturn()
        self.ctx.check(self.ctx.lib.ct_initialize(self.ctx.h, self.id, ctypes.byref(prm), ctypes.byref(r)), "ct_initialize")
        return {"D1": r.D1, "D2": r.D2, "prefac1": r.prefac1, "prefac2": r.prefac2, "norm": r.norm, "dxmax": list(r.dxmax), "dxmax2": list(r.dxmax2)}

    def power_spectrum(self, nfour, box_size, fold=1):
        """(k [1/Mpc], P, Perr) of the box's particles on an nfour^3 grid (power_spectrum_compute)."""
        nb = ctypes.c_int()
        self.ctx.check(self.ctx.lib.ct_power_spectrum(self.ctx.h, self.id, nfour, fold, box_size, 0, None, None, None, ctypes.byref(nb)),
                       "ct_power_spectrum")
        k, P, e = (np.zeros(nb.value, np.float32) for _ in range(3))
        self.ctx.check(self.ctx.lib.ct_power_spectrum(self.ctx.h, self.id, nfour, fold, box_size, nb.value, _p(k), _p(P), _p(e), ctypes.byref(nb)),
                       "ct_power_spectrum")
        return k, P, e

    def lightcone_clear(self):
        """Empties the device buffer without copying it out."""
        n = ctypes.c_int64()
        self.ctx.check(self.ctx.lib.ct_lightcone_download(self.ctx.h, self.id, None, 0, ctypes.byref(n), 1), "ct_lightcone_download")
        return n.value

    def lightcone_reserve(self, entries):
        self.ctx.check(self.ctx.lib.ct_lightcone_reserve(self.ctx.h, self.id, entries), "ct_lightcone_reserve")

    def tree(self):
        cnt = ctypes.c_int64()
        self.ctx.check(self.ctx.lib.ct_tree_download(self.ctx.h, self.id, None, 0, ctypes.byref(cnt)), "ct_tree_download")
        nodes = np.zeros(cnt.value, NODE_DTYPE)
        self.ctx.check(self.ctx.lib.ct_tree_download(self.ctx.h, self.id, _p(nodes), cnt.value, ctypes.byref(cnt)), "ct_tree_download")
        return nodes

    def counters(self):
        c = Counters()
        self.ctx.check(self.ctx.lib.ct_get_counters(self.ctx.h, self.id, ctypes.byref(c)), "ct_get_counters")
        return c.as_dict()

    def direct_ewald(self, sx, sy, sz, h):
        ns = len(sx)
        out = [np.empty(ns) for _ in range(4)]
        sx, sy, sz = (np.ascontiguousarray(a, np.uint32) for a in (sx, sy, sz))
        self.ctx.check(self.ctx.lib.ct_direct_ewald(self.ctx.h, self.id, ns, _p(sx), _p(sy), _p(sz), h, *[_p(a) for a in out]), "ct_direct_ewald")
        return out

    def close(self):
        if self.ctx is not None and self.ctx.h is not None and self.id is not None:
            self.ctx.lib.ct_box_destroy(self.ctx.h, self.id)
            self.id = None
