"""Record the reference's own tree build as fixtures (tests/golden/ref_tree.npz).

The reference's tree_create (src/tree.cpp:273-601) and particles_sort (src/particles.cpp:
979-1018) are compiled where they lie by `make -C oracle tree` (oracle/tree_probe.cpp with the
single-threaded HPX stand-in of oracle/stub/hpx) in two builds: IEEE arithmetic
(oracle/_ref/tree_probe) and the reference's own flags, --fast-math -march=native
(oracle/_ref/tree_probe_native).  For each case below this script writes the seeded input
positions, the IEEE build's tree (ct_or_node fields: heap keys, particle ranges, children,
centres, radii, boxes, leaf flags, depths) and particle order, and how far the native build's
centres (in units of 2^-32) and radii (in units in the last place) are from them -- its keys,
ranges, boxes, leaf flags, depths and particle order are required to be the same; a case where the reference throws (more than a bucket of coincident particles,
"Maximum depth exceeded", tree.cpp:285-286) records the error instead.  The same probe runs
the reference's rung partition (particles_sort_by_rung with push/pop of the active range,
src/particles.cpp:218-235,1029-1076) through RUNG_OPS on seeded particles ("rungs/..." entries).

    python tests/golden/make_tree_golden.py            # writes tests/golden/ref_tree.npz
    python tests/golden/make_tree_golden.py --check    # compares a fresh recording with it

Needs the reference tree at CT_REFERENCE_DIR (default /root/reference) and the probes built.
"""
import argparse
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

OUT = os.path.join(HERE, "ref_tree.npz")
# the rung partition's operation sequence: minimum rungs of particles_sort_by_rung, with the
# active-range stack of particles_push_rungs / particles_pop_rungs between them (a ladder of
# the kind kick_step_hierarchical runs, driver.cpp:382-593, and some restarts from wider ranges)
RUNG_OPS = ["1", "push", "2", "push", "3", "push", "4", "pop", "pop", "3", "pop", "2", "0", "2", "push", "5", "pop", "1"]
PROBE = os.path.join(ROOT, "oracle", "_ref", "tree_probe")
PROBE_NATIVE = os.path.join(ROOT, "oracle", "_ref", "tree_probe_native")
FIELDS = ("key", "part_begin", "part_end", "child_left", "child_right", "pos", "radius", "box_begin", "box_end", "leaf", "depth")


def cases():
    """(name, x, y, z, theta, hsoft, bucket): small seeded boxes covering the tree rules."""
    from cosmictiger_b200 import ics

    out = []
    x, y, z, _, _ = ics.clustered_box(10, nspheres=3, seed=21)
    out.append(("clustered10", x, y, z, 0.55, ics.softening(len(x), 0.02), 128))
    x, y, z, _, _ = ics.zeldovich_lattice(10, index=-2.0, rms_spacing=0.25, seed=22)
    out.append(("lattice10", x, y, z, 0.7, ics.softening(len(x), 0.02), 128))
    # a tight core (a Plummer-like clump of 1000 particles of radius 1e-3 on 200 uniform ones):
    # deep splits by particle count below the Ewald depth, and a small bucket
    rng = np.random.default_rng(23)
    u = rng.random(200 * 3).reshape(3, 200)
    c = np.array([0.31, 0.62, 0.17])
    d = rng.normal(0.0, 1e-3, (3, 1000))
    pts = np.concatenate([u, (c[:, None] + d) % 1.0], axis=1)
    x, y, z = ((pts[k] * 2.0 ** 32).astype(np.uint64).astype(np.uint32) for k in range(3))
    out.append(("core1200", x, y, z, 0.55, 1e-4, 32))
    # one particle: split by the Ewald criterion alone
    out.append(("one", np.array([123456789], np.uint32), np.array([987654321], np.uint32), np.array([2 ** 31], np.uint32), 0.55, 1e-3, 128))
    # a full bucket of coincident particles (one leaf once the Ewald criterion holds)
    k = 128
    out.append(("coincident128", np.full(k, 3 ** 19, np.uint32), np.full(k, 5 ** 13, np.uint32), np.full(k, 7 ** 11, np.uint32), 0.55, 1e-3, 128))
    # one more than a bucket: the reference throws "Maximum depth exceeded"
    k = 129
    out.append(("coincident129", np.full(k, 3 ** 19, np.uint32), np.full(k, 5 ** 13, np.uint32), np.full(k, 7 ** 11, np.uint32), 0.55, 1e-3, 128))
    return out


def run_probe(probe, x, y, z, theta, hsoft, bucket):
    """The reference's tree over (x, y, z): (nodes, x, y, z after the build), or None if it threw."""
    from oracle_lib import NODE_DTYPE

    n = len(x)
    with tempfile.TemporaryDirectory() as tmp:
        fin, fout = os.path.join(tmp, "in.bin"), os.path.join(tmp, "out.bin")
        with open(fin, "wb") as f:
            np.array([n], np.int64).tofile(f)
            for a in (x, y, z):
                np.ascontiguousarray(a, np.uint32).tofile(f)
        res = subprocess.run([probe, fin, fout, repr(float(theta)), repr(float(hsoft)), str(int(bucket))], capture_output=True, text=True)
        if res.returncode == 3:
            # the reference stopped with an error message (THROW_ERROR); only this one is expected
            if "Maximum depth exceeded" not in res.stdout:
                raise RuntimeError("tree probe stopped with an unexpected error: %s" % res.stdout[-400:])
            return None
        if res.returncode != 0:
            raise RuntimeError("tree probe failed (%d): %s" % (res.returncode, res.stderr[-400:]))
        with open(fout, "rb") as f:
            cnt = int(np.fromfile(f, np.int64, 1)[0])
            nodes = np.fromfile(f, NODE_DTYPE, cnt)
            after = [np.fromfile(f, np.uint32, n) for _ in range(3)]
    return nodes, after


def rung_case():
    """1,500 particles with rungs 0-5 (more on the low rungs), seeded positions and velocities."""
    rng = np.random.default_rng(31)
    n = 1500
    x, y, z = (rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32) for _ in range(3))
    v = rng.standard_normal((n, 3)).astype(np.float32)
    r = np.minimum(rng.geometric(0.45, n) - 1, 5).astype(np.int8)
    return x, y, z, v, r


def run_rungs(probe, x, y, z, v, r, ops):
    """The reference's rung partition: (active-range start after each op, x, y, z, v, rung)."""
    n = len(x)
    with tempfile.TemporaryDirectory() as tmp:
        fin, fout = os.path.join(tmp, "in.bin"), os.path.join(tmp, "out.bin")
        with open(fin, "wb") as f:
            np.array([n], np.int64).tofile(f)
            for a in (x, y, z):
                np.ascontiguousarray(a, np.uint32).tofile(f)
            np.ascontiguousarray(v, np.float32).tofile(f)
            np.ascontiguousarray(r, np.int8).tofile(f)
        res = subprocess.run([probe, "--rungs", fin, fout] + list(ops), capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError("rung probe failed (%d): %s" % (res.returncode, res.stderr[-400:]))
        with open(fout, "rb") as f:
            cnt = int(np.fromfile(f, np.int64, 1)[0])
            begins = np.fromfile(f, np.int64, cnt)
            xs = [np.fromfile(f, np.uint32, n) for _ in range(3)]
            vs = np.fromfile(f, np.float32, 3 * n).reshape(n, 3)
            rs = np.fromfile(f, np.int8, n)
    return begins, xs, vs, rs


def record():
    data = {}
    x, y, z, v, r = rung_case()
    begins, xs, vs, rs = run_rungs(PROBE, x, y, z, v, r, RUNG_OPS)
    data["rungs/in_x"] = np.stack([x, y, z])
    data["rungs/in_v"] = v
    data["rungs/in_rung"] = r
    data["rungs/ops"] = np.array(RUNG_OPS)
    data["rungs/begins"] = begins
    data["rungs/x"] = np.stack(xs)
    data["rungs/v"] = vs
    data["rungs/rung"] = rs
    for name, x, y, z, theta, hsoft, bucket in cases():
        data[name + "/in"] = np.stack([x, y, z])
        data[name + "/params"] = np.array([theta, hsoft, bucket], np.float64)
        ieee = run_probe(PROBE, x, y, z, theta, hsoft, bucket)
        native = run_probe(PROBE_NATIVE, x, y, z, theta, hsoft, bucket)
        if (ieee is None) != (native is None):
            raise RuntimeError("%s: one build threw and the other did not" % name)
        data[name + "/threw"] = np.array(ieee is None)
        if ieee is None:
            continue
        nodes, after = ieee
        for f in FIELDS:
            data[name + "/" + f] = nodes[f]
        data[name + "/after"] = np.stack(after)
        nn, nafter = native
        for f in FIELDS:
            if f not in ("pos", "radius") and not np.array_equal(nn[f], nodes[f]):
                raise RuntimeError("%s: the native build's %s differs" % (name, f))
        if not np.array_equal(np.stack(nafter), data[name + "/after"]):
            raise RuntimeError("%s: the native build's particle order differs" % name)
        data[name + "/native_pos_delta"] = (nn["pos"].astype(np.int64) - nodes["pos"].astype(np.int64)).astype(np.int32)
        data[name + "/native_radius_ulps"] = nn["radius"].view(np.int32) - nodes["radius"].view(np.int32)
    return data


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--check", action="store_true")
    args = ap.parse_args()
    data = record()
    if args.check:
        old = np.load(OUT)
        assert sorted(old.files) == sorted(data), "fixture entries differ"
        for k in data:
            assert np.array_equal(old[k], data[k]), k
        print("fresh recording equals", OUT)
        return
    np.savez_compressed(OUT, **data)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
