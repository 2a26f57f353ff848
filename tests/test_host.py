"""Host-side checks that need no GPU: the C ABI library loads and exports every declared
entry point, the package fails loudly without a device, box sharding and the multi-rank
aggregation (gloo, world size 2), and the initial-condition generators."""
import os
import re
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "ct_gravity.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ct_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from cosmictiger_b200 import LIB_PATH, build

    if not os.path.exists(LIB_PATH):
        build.build()
    out = subprocess.check_output(["nm", "-D", "--defined-only", LIB_PATH], text=True)
    exported = set(ln.split()[-1] for ln in out.splitlines() if ln.strip())
    want = declared_symbols()
    assert len(want) >= 15
    missing = [s for s in want if s not in exported]
    assert not missing, missing


def test_library_loads_and_context_needs_a_device():
    import cosmictiger_b200 as ct

    ct.library()
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(ct.GravityError):
        ct.Context(device=0)


def test_shard_boxes_partition():
    from cosmictiger_b200.ensemble import shard_boxes

    rng = np.random.default_rng(0)
    sizes = (np.exp(rng.uniform(np.log(16), np.log(128), 512)).astype(int)) ** 3
    for world in (1, 2, 3, 8):
        parts = [shard_boxes(sizes, world, r) for r in range(world)]
        allidx = np.sort(np.concatenate(parts))
        assert np.array_equal(allidx, np.arange(len(sizes)))
        loads = [sizes[p].sum() for p in parts]
        assert max(loads) - min(loads) <= sizes.max()


_GLOO = r'''
import os, sys
sys.path.insert(0, %r)
import torch.distributed as dist
from cosmictiger_b200.ensemble import aggregate, shard_boxes
dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d", rank=int(sys.argv[1]), world_size=2)
r = dist.get_rank()
mine = shard_boxes([10, 20, 30, 40, 50], 2, r)
ms = 100.0 + 50.0 * r
val, tmax = aggregate(ms, 1000.0 * (r + 1), dist)
print("RESULT", r, list(mine), val, tmax, flush=True)
dist.barrier()
dist.destroy_process_group()
'''


def test_two_rank_aggregation_gloo(tmp_path):
    import socket

    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    script = tmp_path / "agg.py"
    script.write_text(_GLOO % (ROOT, port))
    procs = [subprocess.Popen([sys.executable, str(script), str(r)], stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True) for r in range(2)]
    outs = [p.communicate(timeout=120)[0] for p in procs]
    assert all(p.returncode == 0 for p in procs), outs
    res = {}
    for o in outs:
        for ln in o.splitlines():
            if ln.startswith("RESULT"):
                f = ln.split(maxsplit=3)
                res[int(f[1])] = f
    assert set(res) == {0, 1}
    # sum of particle-steps 3000 over the max time 150 ms
    for r in (0, 1):
        tail = res[r][3].rsplit(" ", 2)
        assert abs(float(tail[1]) - 3000.0 / 0.15) < 1e-6
        assert abs(float(tail[2]) - 150.0) < 1e-9


def test_ics_fixed_point_and_shapes():
    from cosmictiger_b200 import ics

    x, y, z, v, r = ics.zeldovich_lattice(8, index=-2.0, rms_spacing=0.25, seed=1)
    assert x.dtype == np.uint32 and v.shape == (512, 3) and r.dtype == np.int8
    disp = ics.fixed32_to_double(x) - np.repeat(np.arange(8) / 8.0, 64)
    disp = (disp + 0.5) % 1.0 - 0.5
    assert 0.0 < np.sqrt(np.mean(disp ** 2)) < 0.25 / 8
    cx, cy, cz, cv, cr = ics.clustered_box(16, nspheres=20, seed=2)
    assert len(cx) == 16 ** 3
    assert ics.to_fixed32(np.array([0.0, 0.5, 1.0 - 1e-12, -0.25]))[1] == 2 ** 31


def _header_prototypes():
    """name -> number of parameters of every function declared in include/ct_gravity.h."""
    src = open(os.path.join(ROOT, "include", "ct_gravity.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    out = {}
    for m in re.finditer(r"\b(ct_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", src):
        params = m.group(2).strip()
        out[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def test_ctypes_bindings_match_the_header():
    """Every function the header declares has an argtypes list in the Python binding with as many
    entries as the C prototype has parameters (a mismatch, or a missing list, would pass
    truncated or shifted values through the ABI without an error)."""
    import cosmictiger_b200 as ct

    L = ct.library()
    protos = _header_prototypes()
    assert len(protos) >= 40
    for name, nparams in protos.items():
        fn = getattr(L, name)
        assert fn.argtypes is not None, name
        assert len(fn.argtypes) == nparams, (name, len(fn.argtypes), nparams)
    # returns wider than int keep their width (ctypes' default restype is a 32-bit int)
    import ctypes

    for name, rt in (("ct_stream", ctypes.c_void_p), ("ct_last_error", ctypes.c_char_p), ("ct_launch_count", ctypes.c_ulonglong)):
        assert getattr(L, name).restype is rt, name
    assert ctypes.sizeof(L.ct_box_size.restype) == 8 and ctypes.sizeof(L.ct_bytes_in_use.restype) == 8


_NULL_CTX = r'''
import ctypes, sys
sys.path.insert(0, %r)
import cosmictiger_b200 as ct
L = ct.library()
numbers = (ctypes.c_int, ctypes.c_int64, ctypes.c_float, ctypes.c_double, ctypes.c_size_t, ctypes.c_ulonglong)
for name in %r:
    fn = getattr(L, name)
    r = fn(*[0 if t in numbers else None for t in fn.argtypes])
    print(name, r, flush=True)
'''


def test_entry_points_reject_a_null_context():
    """Every ct_status entry point taking a context returns an error for a NULL context and null
    arguments instead of dereferencing them (run in a child process, so that a crash is a test
    failure rather than the end of the test run).  No device is touched."""
    import cosmictiger_b200 as ct

    ct.library()
    src = open(os.path.join(ROOT, "include", "ct_gravity.h")).read()
    names = sorted(n for n in _header_prototypes() if re.search(r"ct_status\s+" + n + r"\s*\(\s*ct_ctx\s*\*", src) and n != "ct_ctx_create")
    assert len(names) >= 30
    out = subprocess.run([sys.executable, "-c", _NULL_CTX % (ROOT, names)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr[-2000:]
    got = dict(ln.split() for ln in out.stdout.splitlines())
    assert sorted(got) == names
    assert all(int(v) < 0 for v in got.values()), got


_ABI_PROGRAM = r'''
#include <stdio.h>
#include "ct_gravity.h"
int main(void) {
	ct_ctx* ctx = NULL;
	ct_status s = ct_ctx_create(&ctx, 0, 0, 7);
	if (s == CT_OK) {
		printf("context order %d\n", ct_order(ctx));
		ct_ctx_destroy(ctx);
		return 0;
	}
	printf("status %d\n", (int) s);
	return s < 0 ? 0 : 1;
}
'''


@pytest.mark.parametrize("compiler,std", [("gcc", "-std=c99"), ("g++", "-std=c++17")])
def test_header_compiles_and_links_from_c_and_cpp(tmp_path, compiler, std):
    """include/ct_gravity.h is plain C (and C++): a program written against it alone compiles
    with warnings as errors, links against libct_gravity.so and runs; without a device the
    context call returns an error status instead of failing."""
    import shutil

    from cosmictiger_b200 import LIB_PATH, build

    if shutil.which(compiler) is None:
        pytest.skip(compiler + " not installed")
    if not os.path.exists(LIB_PATH):
        build.build()
    src = tmp_path / ("abi.c" if compiler == "gcc" else "abi.cpp")
    src.write_text(_ABI_PROGRAM)
    exe = tmp_path / "abi"
    libdir = os.path.dirname(LIB_PATH)
    cmd = [compiler, std, "-Wall", "-Wextra", "-pedantic", "-Werror", "-I" + os.path.join(ROOT, "include"), str(src), "-L" + libdir, "-lct_gravity",
           "-Wl,-rpath," + libdir, "-o", str(exe)]
    cc = subprocess.run(cmd, capture_output=True, text=True, timeout=120)
    assert cc.returncode == 0, cc.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0, run.stdout + run.stderr
    assert run.stdout.startswith(("context order 7", "status -")), run.stdout


def test_noalloc_rung_partition_rejects_bad_arguments_before_device_work():
    """ct_sort_by_rung_noalloc checks its arguments before it touches a device: a negative
    begin, n below begin, min_rung outside 0-15, NULL arrays for a non-empty range and a null
    result pointer give CT_ERR_ARG; a range above the fixed capacity gives CT_ERR_CAPACITY;
    min_rung 0 and an empty range succeed without device work.  None of these calls needs a
    GPU, so they run here (in a child process, so that a crash fails the test)."""
    import cosmictiger_b200 as ct

    ct.library()
    prog = r'''
import ctypes, sys
sys.path.insert(0, %r)
import cosmictiger_b200 as ct
f = ct.library().ct_sort_by_rung_noalloc
vp = ctypes.c_void_p
f.argtypes = [ctypes.c_int64, ctypes.c_int64, ctypes.c_int, vp, vp, vp, vp, vp, vp, vp, ctypes.POINTER(ctypes.c_int64), vp]
f.restype = ctypes.c_int
buf = (ctypes.c_uint8 * 64)()
a = ctypes.cast(buf, vp)
def call(begin, n, mr, arrays=True, out=True):
    rb = ctypes.c_int64(-7)
    args = [a] * 7 if arrays else [None] * 7
    rc = f(begin, n, mr, *args, ctypes.byref(rb) if out else None, None)
    return rc, rb.value
cap = 1 << 20
print(call(-1, 10, 1)[0], call(5, 4, 1)[0], call(0, 10, 16)[0], call(0, 10, -1)[0], call(0, 10, 1, arrays=False)[0], call(0, 10, 1, out=False)[0])
print(call(3, 3 + cap + 1, 1)[0], call(0, cap + 1, 1, arrays=False)[0])
print(*call(4, 100, 0), *call(9, 9, 2))
''' % ROOT
    out = subprocess.run([sys.executable, "-c", prog], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = out.stdout.split("\n")
    arg = [int(t) for t in lines[0].split()]
    assert arg == [-1] * 6, arg  # CT_ERR_ARG
    assert [int(t) for t in lines[1].split()] == [-4, -4]  # CT_ERR_CAPACITY
    # min_rung 0 resets the active range to 0; an empty range leaves it at begin
    assert [int(t) for t in lines[2].split()] == [0, 0, 0, 9]
