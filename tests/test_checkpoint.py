"""The reference's checkpoint layout (write_checkpoint, src/driver.cpp:1143-1173; particles_save,
src/particles.cpp:1206-1227; domains_save, src/domain.cpp:87-94): struct sizes and offsets,
byte-level layout of the particle section, round trips, resuming a hierarchical run from a
checkpoint on the device, and files written and read by the reference's own code
(oracle/ckpt_probe.cpp): byte-identical in both directions."""
import struct

import numpy as np
import pytest

from cosmictiger_b200 import checkpoint as ck


def test_struct_layouts():
    d = ck.DRIVER_PARAMS
    assert d.itemsize == 176
    assert d.fields["energies"][1] == 48 and d.fields["max_rung"][1] == 112 and d.fields["bucket_size"][1] == 128
    assert d.fields["total_processed"][1] == 136 and d.fields["flops"][1] == 144 and d.fields["itime"][1] == 168
    assert ck.DOMAIN_ENTRY.itemsize == 72  # pair<size_t, domain_t>: 8 + (48 + 8 + 4 + 4)
    assert ck.domain_local_dtype(False).itemsize == 72 and ck.domain_local_dtype(True).itemsize == 80


def test_particle_section_bytes(tmp_path):
    """The bytes after driver_params follow particles_save field by field."""
    x = np.array([1, 2, 3], np.uint32)
    y = np.array([4, 5, 6], np.uint32)
    z = np.array([7, 8, 2 ** 32 - 1], np.uint32)
    v = np.arange(9, dtype=np.float32).reshape(3, 3)
    r = np.array([0, 2, 1], np.int8)
    p = tmp_path / "c.dat"
    ck.write_checkpoint(str(p), ck.default_params(a=0.5, iter=7), x, y, z, v, r, rung_begin=1, rung_begins=[0])
    raw = p.read_bytes()
    body = raw[176:]
    want = struct.pack("<i", 3) + struct.pack("<3I", 1, 2, 3) + struct.pack("<3I", 4, 5, 6) + struct.pack("<3I", 7, 8, 2 ** 32 - 1)
    want += struct.pack("<9f", *range(9)) + struct.pack("<3b", 0, 2, 1) + struct.pack("<3i", 1, 1, 0)
    assert body[:len(want)] == want
    # domains: one entry (key 1, unit box, midx 0, rank 0) and one domain_local
    dom = body[len(want):]
    assert len(dom) == 8 + 72 + 72
    assert struct.unpack("<Q", dom[:8])[0] == 1
    params = np.frombuffer(raw[:176], ck.DRIVER_PARAMS)[0]
    assert params["a"] == 0.5 and params["iter"] == 7


def test_round_trip_and_truncation(tmp_path):
    rng = np.random.default_rng(3)
    n = 1000
    x, y, z = (rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32) for _ in range(3))
    v = rng.standard_normal((n, 3)).astype(np.float32)
    r = rng.integers(0, 5, n).astype(np.int8)
    p = tmp_path / "c.dat"
    params = ck.default_params(a=1.0, tau=0.25, max_rung=4, minrung0=1, step=3, bucket_size=128)
    ck.write_checkpoint(str(p), params, x, y, z, v, r, rung_begin=700, rung_begins=[0, 300, 600])
    c = ck.read_checkpoint(str(p))
    for k, a in (("x", x), ("y", y), ("z", z), ("v", v), ("rung", r)):
        assert np.array_equal(c[k], a), k
    assert c["rung_begin"] == 700 and c["rung_begins"] == [0, 300, 600]
    assert c["params"]["max_rung"] == 4 and c["params"]["tau"] == 0.25
    assert c["domain_local"]["part_range"][0].tolist() == [0, n]
    raw = p.read_bytes()
    (tmp_path / "t.dat").write_bytes(raw[:-5])
    with pytest.raises(ck.CheckpointError):
        ck.read_checkpoint(str(tmp_path / "t.dat"))
    with pytest.raises(ck.CheckpointError):
        ck.read_checkpoint(str(p), lightcone=True)


@pytest.mark.gpu
def test_resume_hierarchical_run_from_checkpoint(tmp_path):
    """Two hierarchical steps, checkpoint, two more, against the same four steps with a reload
    from the checkpoint in between: bit-identical particles and rung-ladder state."""
    import cosmictiger_b200 as ct
    from cosmictiger_b200 import ics

    x, y, z, v, r = ics.clustered_box(16, nspheres=20, seed=41)
    N = len(x)
    h = ics.softening(N, 0.02)
    ctx = ct.Context(order=7)

    def run(box, steps, state):
        for _ in range(steps):
            sp = ct.StepParams(minrung=state["minrung"], minrung0=0, max_rung=state["max_rung"], a=1.0, tau=state["tau"], t0=0.01, theta=0.55, hsoft=h,
                               bucket=128, eta=ics.eta_default(), GM=1.0 / N, max_dt=1e30, do_phi=1, nocrop=1, drag=0.0, sign=1.0)
            res = box.step_hierarchical(sp)
            state.update(minrung=res.minrung, max_rung=res.max_rung, tau=state["tau"] + 0.01)

    a = ctx.box(N)
    a.upload(x, y, z, v, r)
    sa = {"minrung": 0, "max_rung": 0, "tau": 0.0}
    run(a, 2, sa)
    path = str(tmp_path / "ck.dat")
    ck.save_box(path, a, ck.default_params(a=1.0, tau=sa["tau"], max_rung=sa["max_rung"], minrung0=sa["minrung"], step=2, bucket_size=128))
    run(a, 2, sa)
    b, params = ck.load_box(ctx, path)
    sb = {"minrung": int(params["minrung0"]), "max_rung": int(params["max_rung"]), "tau": float(params["tau"])}
    run(b, 2, sb)
    oa, ob = a.download(), b.download()
    for f in ("x", "y", "z", "v", "rung"):
        assert np.array_equal(oa[f], ob[f]), f
    assert a.rung_state() == b.rung_state()
    assert sa == sb
    ctx.close()


def test_layouts_match_the_reference_compiler():
    """The record layouts used here equal the reference's as its compiler lays them out
    (tests/golden/ref_layouts.json, printed by oracle/layout_probe.cu built against the
    reference's headers): driver_params, domain_t and the lightcone's lc_entry."""
    import json
    import os

    import cosmictiger_b200 as ct

    ref = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_layouts.json")))
    d, dp = ck.DRIVER_PARAMS, ref["driver_params"]
    assert d.itemsize == dp["size"]
    for f in ("energies", "max_rung", "bucket_size", "total_processed", "flops", "itime"):
        assert d.fields[f][1] == dp[f], f
    assert ck.DOMAIN_ENTRY.itemsize == 8 + ref["domain_t"]  # pair<size_t key, domain_t>
    lc = ct.LC_ENTRY
    assert lc.itemsize == ref["lc_entry"]["size"]
    assert lc.fields["vx"][1] == ref["lc_entry"]["vx"] and lc.fields["pix"][1] == ref["lc_entry"]["pix"]


def test_load_box_frees_the_box_when_the_state_is_refused(tmp_path):
    """A checkpoint whose rung state the library refuses leaves no box behind (a fake context
    stands in for the device)."""

    class FakeBox:
        closed = False

        def upload(self, *a):
            pass

        def set_rung_state(self, rung_begin, stack):
            raise RuntimeError("rung_begin beyond the box")

        def close(self):
            self.closed = True

    class FakeCtx:
        def box(self, n):
            self.made = FakeBox()
            return self.made

    n = 8
    x = np.arange(n, dtype=np.uint32)
    path = str(tmp_path / "bad.chk")
    ck.write_checkpoint(path, ck.default_params(a=1.0), x, x, x, np.zeros((n, 3), np.float32), np.zeros(n, np.int8), rung_begin=99)
    ctx = FakeCtx()
    with pytest.raises(RuntimeError):
        ck.load_box(ctx, path)
    assert ctx.made.closed


@pytest.mark.parametrize("probe,fixture", [("layout_probe", "ref_layouts.json"), ("func_probe", "ref_functions.json")])
def test_reference_fixtures_equal_their_probes(probe, fixture):
    """Where the probes built from the reference's sources are present (oracle/_ref, made by
    `make -C oracle layout funcs`), their output equals the committed fixture byte for byte, so
    the fixtures cannot drift from the reference they were recorded from."""
    import os
    import subprocess

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = os.path.join(root, "oracle", "_ref", probe)
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref/%s not built (needs the reference's sources)" % probe)
    out = subprocess.run([exe], capture_output=True, timeout=60)
    assert out.returncode == 0
    with open(os.path.join(root, "tests", "golden", fixture), "rb") as f:
        assert out.stdout == f.read()


# ---------------------------------------------------------------- against the reference's own writer
# tests/golden/ref_checkpoint.npz: files the reference's write_checkpoint wrote for one rank
# (oracle/ckpt_probe.cpp; tests/golden/make_ckpt_golden.py), with the states they came from.
def _ref_ckpt():
    import os

    return np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_checkpoint.npz"))


def _ref_cases():
    return sorted({k.split("/")[0] for k in _ref_ckpt().files})


@pytest.mark.parametrize("name", _ref_cases())
def test_reference_written_checkpoint_reads_and_rewrites_byte_for_byte(tmp_path, name):
    """A checkpoint the reference wrote reads back to its state -- driver_params, the particles
    in the order the reference's rung partition left them (this project's CPU oracle applies the
    same operations to the same particles and gets the same order, range start and saved
    starts), the one-rank domain section -- and write_checkpoint of that state gives the
    reference's file byte for byte."""
    from tests import oracle_lib

    fx = _ref_ckpt()
    raw = fx[name + "/file"].tobytes()
    path = tmp_path / "ref.dat"
    path.write_bytes(raw)
    c = ck.read_checkpoint(str(path))
    assert np.asarray(c["params"], ck.DRIVER_PARAMS).tobytes() == fx[name + "/params"].tobytes()
    x, y, z = (fx[name + "/x"][k].copy() for k in range(3))
    v = fx[name + "/v"].copy()
    r = fx[name + "/rung"].copy()
    begin, stack = 0, []
    if len(x):
        orc = oracle_lib.load()
        for op in fx[name + "/ops"]:
            if op == "push":
                stack.append(begin)
            elif op == "pop":
                begin = stack.pop()
            else:
                m = int(op)
                begin = 0 if m == 0 else orc.sort_by_rung(x, y, z, v, r, m, begin)
    assert np.array_equal(c["x"], x) and np.array_equal(c["y"], y) and np.array_equal(c["z"], z)
    assert np.array_equal(c["v"], v) and np.array_equal(c["rung"], r)
    assert c["rung_begin"] == begin and c["rung_begins"] == stack
    assert len(c["domains"]) == 1 and c["domains"]["key"][0] == 1 and c["domains"]["rank"][0] == 0
    assert c["domain_local"]["part_range"][0].tolist() == [0, len(x)]
    out = tmp_path / "ours.dat"
    ck.write_checkpoint(str(out), c["params"], c["x"], c["y"], c["z"], c["v"], c["rung"], c["rung_begin"], c["rung_begins"])
    assert out.read_bytes() == raw


def _ckpt_probe():
    import os

    exe = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "ckpt_probe")
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref/ckpt_probe not built (needs the reference's sources)")
    return exe


def test_reference_reads_and_rewrites_our_checkpoint():
    """Where the probe is built: the reference's read_checkpoint loads a file this module wrote
    (a state with a rung ladder) and its write_checkpoint writes the same bytes back."""
    import importlib.util
    import os

    _ckpt_probe()
    spec = importlib.util.spec_from_file_location("make_ckpt_golden", os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "make_ckpt_golden.py"))
    g = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(g)
    import tempfile

    rng = np.random.default_rng(11)
    n = 101
    x, y, z = (rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32) for _ in range(3))
    v = rng.standard_normal((n, 3)).astype(np.float32)
    r = np.sort(rng.integers(0, 4, n)).astype(np.int8)
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "ours.dat")
        ck.write_checkpoint(path, ck.default_params(a=0.25, tau=1.5, iter=g.ITER, step=3), x, y, z, v, r, rung_begin=40, rung_begins=[0, 17])
        mine = np.fromfile(path, np.uint8)
    assert np.array_equal(g.resave(mine), mine)


def test_checkpoint_fixture_equals_a_fresh_run_of_the_reference():
    """Where the probe is built, a fresh recording from the reference's code equals the committed
    fixture (guards the fixture against drift of the generator or the probe)."""
    import os
    import subprocess
    import sys

    _ckpt_probe()
    here = os.path.dirname(os.path.abspath(__file__))
    res = subprocess.run([sys.executable, os.path.join(here, "golden", "make_ckpt_golden.py"), "--check"], capture_output=True, text=True,
                         cwd=os.path.dirname(here))
    assert res.returncode == 0, res.stdout + res.stderr
