"""The reference's checkpoint file, so that states move between the two codes.

A checkpoint written by write_checkpoint (src/driver.cpp:1143-1173) for one rank holds, in
order and in the rank's native byte order:

  driver_params            the driver's state (cosmictiger/driver.hpp:26-43), a C struct with
                           natural alignment: 176 bytes
  particles_save           (src/particles.cpp:1206-1227) part_int N; fixed32 x[N], y[N], z[N];
                           float v[N][3]; char rung[N]; [group_int lastgroup[N] with groups]
                           [char tracer[N] with tracers]; int depth; int rung_begin;
                           int rung_begins[depth]
  domains_save             (src/domain.cpp:87-94) size_t count; count x {size_t key; domain_t};
                           domain_local[ranks]
  lc_save                  only with lightcone output (not part of this path: refused here)

part_int is int unless the reference was built with LONG_LONG_PART_INT.  The particle
section maps one to one onto this library's box state: positions, velocities (AoS at the
ABI), rungs, and the rung ladder's active range and saved range starts
(ct_box_set_rung_state).  This module reads and writes that layout; a box's state goes in
and out through Box.upload/download and Box.rung_state/set_rung_state.
"""
import numpy as np

ENERGIES = [("pot", "<f8"), ("kin", "<f8"), ("tckin", "<f8"), ("xmom", "<f8"), ("ymom", "<f8"), ("cosmic", "<f8"), ("zmom", "<f8"), ("nmom", "<f8")]

# driver_params (cosmictiger/driver.hpp:26-43) with the C compiler's natural alignment
DRIVER_PARAMS = np.dtype([("a", "<f8"), ("adot", "<f8"), ("dummy", "<f8"), ("tau", "<f8"), ("tau_max", "<f8"), ("energy0", "<f8"),
                          ("energies", ENERGIES), ("max_rung", "<i4"), ("iter", "<i4"), ("minrung0", "<i4"), ("step", "<i4"), ("bucket_size", "<i4"),
                          ("total_processed", "<u8"), ("flops", "<f8"), ("runtime", "<f8"), ("years", "<f8"), ("itime", "<u8")], align=True)

# domain_t (cosmictiger/domain.hpp:39-48) and domain_local (:61-66)
RANGE = [("begin", "<f8", 3), ("end", "<f8", 3)]
DOMAIN_ENTRY = np.dtype([("key", "<u8"), ("box", RANGE), ("midx", "<f8"), ("rank", "<i4")], align=True)


def domain_local_dtype(part_int64):
    pi = "<i8" if part_int64 else "<i4"
    return np.dtype([("box", RANGE), ("proc_range", "<i4", 2), ("part_range", pi, 2), ("depth", "<i4")], align=True)


class CheckpointError(ValueError):
    pass


def default_params(**kw):
    """A driver_params record with the given fields set (others zero)."""
    p = np.zeros((), DRIVER_PARAMS)
    for k, v in kw.items():
        p[k] = v
    return p


def read_checkpoint(path, part_int64=False, groups=False, group_int64=False, tracers=False, lightcone=False):
    """Read a one-rank checkpoint.  Returns {"params": structured scalar, "x", "y", "z" (uint32),
    "v" (float32 (N, 3)), "rung" (int8), "rung_begin": int, "rung_begins": [int],
    "domains": structured array, "domain_local": structured array, and "lastgroup"/"tracer"
    when present}."""
    if lightcone:
        raise CheckpointError("lightcone sections (lc_save) are not part of the gravity step")
    raw = np.fromfile(path, np.uint8)
    pos = 0

    def take(dtype, count=1):
        nonlocal pos
        dt = np.dtype(dtype)
        nbytes = dt.itemsize * count
        if pos + nbytes > len(raw):
            raise CheckpointError("%s: truncated (need %d bytes at offset %d, file has %d)" % (path, nbytes, pos, len(raw)))
        a = raw[pos:pos + nbytes].view(dt)
        pos += nbytes
        return a.copy()

    out = {"params": take(DRIVER_PARAMS)[0]}
    n = int(take("<i8" if part_int64 else "<i4")[0])
    if n < 0:
        raise CheckpointError("%s: negative particle count" % path)
    out["x"], out["y"], out["z"] = take("<u4", n), take("<u4", n), take("<u4", n)
    out["v"] = take("<f4", 3 * n).reshape(n, 3)
    out["rung"] = take("<i1", n)
    if groups:
        out["lastgroup"] = take("<u8" if group_int64 else "<u4", n)
    if tracers:
        out["tracer"] = take("<i1", n)
    depth = int(take("<i4")[0])
    out["rung_begin"] = int(take("<i4")[0])
    out["rung_begins"] = [int(q) for q in take("<i4", depth)] if depth > 0 else []
    ndom = int(take("<u8")[0])
    out["domains"] = take(DOMAIN_ENTRY, ndom)
    out["domain_local"] = take(domain_local_dtype(part_int64), 1)
    if pos != len(raw):
        raise CheckpointError("%s: %d bytes left after the last section" % (path, len(raw) - pos))
    return out


def write_checkpoint(path, params, x, y, z, v, rung, rung_begin=0, rung_begins=(), part_int64=False):
    """Write a one-rank checkpoint in the reference's layout.  The domain section describes
    the single rank owning the unit box and all particles, as the reference's one-rank domain
    decomposition leaves it (domains_rebound, src/domain.cpp:211-330: key 1, the unit box, rank
    0; the split coordinate midx is set only for domains it splits, so it stays 0) -- the file
    is byte for byte the one the reference's write_checkpoint writes for the same state."""
    n = len(x)
    v = np.ascontiguousarray(v, np.float32).reshape(n, 3)
    dom = np.zeros(1, DOMAIN_ENTRY)
    dom["key"] = 1
    dom["box"]["end"] = 1.0
    loc = np.zeros(1, domain_local_dtype(part_int64))
    loc["box"]["end"] = 1.0
    loc["proc_range"] = (0, 1)
    loc["part_range"] = (0, n)
    with open(path, "wb") as f:
        f.write(np.asarray(params, DRIVER_PARAMS).tobytes())
        f.write(np.array([n], "<i8" if part_int64 else "<i4").tobytes())
        for a in (x, y, z):
            f.write(np.ascontiguousarray(a, "<u4").tobytes())
        f.write(v.astype("<f4").tobytes())
        f.write(np.ascontiguousarray(rung, "<i1").tobytes())
        rb = list(rung_begins)
        f.write(np.array([len(rb), rung_begin] + rb, "<i4").tobytes())
        f.write(np.array([1], "<u8").tobytes())
        f.write(dom.tobytes())
        f.write(loc.tobytes())


def save_box(path, box, params):
    """Write a box's particles and rung-ladder state as a checkpoint."""
    st = box.download()
    rb, stack = box.rung_state()
    write_checkpoint(path, params, st["x"], st["y"], st["z"], st["v"], st["rung"], rb, stack)


def load_box(ctx, path, **kw):
    """A new box holding a checkpoint's particles and rung-ladder state; returns (box, params)."""
    c = read_checkpoint(path, **kw)
    box = ctx.box(len(c["x"]))
    try:
        box.upload(c["x"], c["y"], c["z"], c["v"], c["rung"])
        box.set_rung_state(c["rung_begin"], c["rung_begins"])
    except Exception:
        box.close()  # a state the library refuses (e.g. rung_begin beyond N) frees its box
        raise
    return box, c["params"]
