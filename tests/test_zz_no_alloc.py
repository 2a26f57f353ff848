"""The allocation-free rung partition (ct_sort_by_rung_noalloc) against ct_sort_by_rung.

ct_sort_by_rung_noalloc serves callers that cannot allocate device memory when they
partition rungs (a driver inside a memory pool it does not own, or one that keeps its device
footprint fixed): it works on device arrays the caller holds and keeps its temporary storage
in a fixed file-scope device array.  This file is collected last so that a failure here comes
after every other test has run; it passes alone and after the others.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(lib):
    f = lib.ct_sort_by_rung_noalloc
    vp = ctypes.c_void_p
    f.argtypes = [ctypes.c_int64, ctypes.c_int64, ctypes.c_int, vp, vp, vp, vp, vp, vp, vp, ctypes.POINTER(ctypes.c_int64), vp]
    f.restype = ctypes.c_int
    return f


def test_noalloc_rung_partition_matches_allocating_entry_point():
    import torch

    import cosmictiger_b200 as ct

    lib = ct.library()
    f = _noalloc(lib)
    rng = np.random.default_rng(2024)
    N = 300001
    x, y, z = (rng.integers(0, 2 ** 32, N, dtype=np.uint64).astype(np.uint32) for _ in range(3))
    v = rng.standard_normal((N, 3)).astype(np.float32)
    r = rng.integers(0, 5, N).astype(np.int8)

    # the existing entry point, on a context-owned box
    ctx = ct.Context(order=7)
    box = ctx.box(N)
    box.upload(x, y, z, v, r)
    ref_begin = [box.sort_by_rung(1), box.sort_by_rung(3)]
    ref = box.download()
    box.close()
    ctx.close()

    # the allocation-free entry point on caller-held device arrays, two calls in a row
    dev = torch.device("cuda", 0)
    tx, ty, tz = (torch.from_numpy(a.view(np.int32).copy()).to(dev) for a in (x, y, z))
    tv = [torch.from_numpy(np.ascontiguousarray(v[:, d])).to(dev) for d in range(3)]
    tr = torch.from_numpy(r.copy()).to(dev)
    stream = torch.cuda.current_stream(dev)
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    begin = 0
    got_begin = []
    for minrung in (1, 3):
        rb = ctypes.c_int64(-1)
        rc = f(begin, N, minrung, ptr(tx), ptr(ty), ptr(tz), ptr(tv[0]), ptr(tv[1]), ptr(tv[2]), ptr(tr), ctypes.byref(rb),
               ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0
        begin = rb.value
        got_begin.append(begin)
    torch.cuda.synchronize()
    assert got_begin == ref_begin
    assert np.array_equal(tx.cpu().numpy().view(np.uint32), ref["x"])
    assert np.array_equal(ty.cpu().numpy().view(np.uint32), ref["y"])
    assert np.array_equal(tz.cpu().numpy().view(np.uint32), ref["z"])
    for d in range(3):
        assert np.array_equal(tv[d].cpu().numpy(), ref["v"][:, d])
    assert np.array_equal(tr.cpu().numpy(), ref["rung"])


def test_noalloc_rejects_oversize():
    import cosmictiger_b200 as ct

    f = _noalloc(ct.library())
    rb = ctypes.c_int64(-1)
    n = (1 << 20) + 1
    rc = f(0, n, 1, None, None, None, None, None, None, None, ctypes.byref(rb), None)
    assert rc == -4  # CT_ERR_CAPACITY, before any device work
    assert rb.value == -1


def test_noalloc_full_capacity_from_an_offset():
    """The largest call the fixed scratch array allows (exactly CT_NOALLOC_MAX_PARTICLES
    particles) on a range that starts past the beginning of the caller's arrays, against
    ct_sort_by_rung on the same data: the active range of a previous partition (rung 0 moved
    to the front) is partitioned again at min_rung 3."""
    import torch

    import cosmictiger_b200 as ct

    lib = ct.library()
    f = _noalloc(lib)
    cap = 1 << 20
    n0 = 5003  # particles on rung 0, in front of the active range after the first partition
    N = n0 + cap
    rng = np.random.default_rng(77)
    x, y, z = (rng.integers(0, 2 ** 32, N, dtype=np.uint64).astype(np.uint32) for _ in range(3))
    v = rng.standard_normal((N, 3)).astype(np.float32)
    r = rng.integers(1, 6, N).astype(np.int8)
    r[rng.choice(N, n0, replace=False)] = 0

    ctx = ct.Context(order=7)
    box = ctx.box(N)
    box.upload(x, y, z, v, r)
    b1 = box.sort_by_rung(1)
    assert b1 == n0
    mid = box.download()
    b3 = box.sort_by_rung(3)
    ref = box.download()
    box.close()
    ctx.close()

    dev = torch.device("cuda", 0)
    tx, ty, tz = (torch.from_numpy(mid[c].view(np.int32).copy()).to(dev) for c in "xyz")
    tv = [torch.from_numpy(np.ascontiguousarray(mid["v"][:, d])).to(dev) for d in range(3)]
    tr = torch.from_numpy(mid["rung"].copy()).to(dev)
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    stream = torch.cuda.current_stream(dev)
    rb = ctypes.c_int64(-1)
    rc = f(b1, N, 3, ptr(tx), ptr(ty), ptr(tz), ptr(tv[0]), ptr(tv[1]), ptr(tv[2]), ptr(tr), ctypes.byref(rb), ctypes.c_void_p(stream.cuda_stream))
    assert rc == 0
    torch.cuda.synchronize()
    assert rb.value == b3
    for c, t in zip("xyz", (tx, ty, tz)):
        assert np.array_equal(t.cpu().numpy().view(np.uint32), ref[c]), c
    for d in range(3):
        assert np.array_equal(tv[d].cpu().numpy(), ref["v"][:, d])
    assert np.array_equal(tr.cpu().numpy(), ref["rung"])
