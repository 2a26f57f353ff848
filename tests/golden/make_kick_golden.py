"""Record the work items of the reference's own CPU top of the kick as fixtures
(tests/golden/ref_kick_items.npz).

The reference's kick() (src/kick.cpp:150-507, its multipole interactions of src/gravity.cpp)
runs over its own tree build (src/tree.cpp) as the driver starts a step (driver.cpp:490-528:
zero expansion, the root as both check lists, every particle active), compiled where it lies by
`make -C oracle kick` (oracle/kick_probe.cpp; single-threaded HPX stand-in, the GPU workspace
replaced by a recorder).  Every subtree of at most max_parts = min(CUDA_KICK_PARTS_MAX,
max(N / blocks, bucket)) particles becomes a work item (kick.cpp:170-189), ordered by first
particle (kick_workspace.cpp:308-310).  For each case the fixture holds the input positions,
the parameters and the items: subtree root, incoming expansion, its centre, and the direct and
Ewald check lists (node indices of the depth-first tree, which is the order of this project's
CPU oracle's tree; CSR offsets).

    python tests/golden/make_kick_golden.py            # writes tests/golden/ref_kick_items.npz
    python tests/golden/make_kick_golden.py --check    # compares a fresh recording with it

Needs the reference tree at CT_REFERENCE_DIR (default /root/reference) and the probe built.
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

OUT = os.path.join(HERE, "ref_kick_items.npz")
PROBE = os.path.join(ROOT, "oracle", "_ref", "kick_probe")
NEXP = 50  # the reference's EXPANSION_SIZE at order 7


def cases():
    """(name, x (3, n), theta, hsoft, bucket, blocks)."""
    from cosmictiger_b200 import ics

    out = []
    x, y, z, _, _ = ics.clustered_box(16, nspheres=3, seed=21)
    out.append(("clustered16_b64", np.stack([x, y, z]), 0.55, ics.softening(len(x), 0.02), 128, 64))
    x, y, z, _, _ = ics.zeldovich_lattice(16, index=-2.0, rms_spacing=0.25, seed=22)
    out.append(("lattice16_b64", np.stack([x, y, z]), 0.7, ics.softening(len(x), 0.02), 128, 64))
    x, y, z, _, _ = ics.clustered_box(24, nspheres=20, seed=23)
    pts = np.stack([x, y, z])
    # a B200's kick block count (1,184 resident blocks): items of at most a bucket
    out.append(("clustered24_b1184", pts, 0.55, ics.softening(len(x), 0.02), 128, 1184))
    # few blocks: items of up to 1,728 particles, a deeper CPU top
    out.append(("clustered24_b8", pts, 0.55, ics.softening(len(x), 0.02), 128, 8))
    return out


def run_probe(x, theta, hsoft, bucket, blocks):
    """The reference's work items: dict of max_parts, self, L, pos, doff, dlist, eoff, elist."""
    from tests.oracle_lib import NODE_DTYPE

    n = x.shape[1]
    with tempfile.TemporaryDirectory() as tmp:
        fin, fout = os.path.join(tmp, "in.bin"), os.path.join(tmp, "out.bin")
        with open(fin, "wb") as f:
            f.write(np.int64(n).tobytes())
            f.write(np.ascontiguousarray(x, np.uint32).tobytes())
        subprocess.run([PROBE, fin, fout, repr(theta), repr(hsoft), str(bucket), str(blocks)], check=True, stdout=subprocess.DEVNULL)
        raw = open(fout, "rb").read()
    off = 0

    def take(dt, cnt):
        nonlocal off
        a = np.frombuffer(raw, dt, cnt, off)
        off += a.nbytes
        return a.copy()

    nn = int(take(np.int64, 1)[0])
    take(NODE_DTYPE, nn)
    take(np.uint32, 3 * n)
    max_parts = int(take(np.int64, 1)[0])
    ni = int(take(np.int64, 1)[0])
    it = {"self": np.zeros(ni, np.int32), "L": np.zeros((ni, NEXP), np.float32), "pos": np.zeros((ni, 3), np.uint32)}
    dl, el, doff, eoff = [], [], [0], [0]
    for i in range(ni):
        it["self"][i] = take(np.int32, 1)[0]
        it["L"][i] = take(np.float32, NEXP)
        it["pos"][i] = take(np.uint32, 3)
        nd = int(take(np.int32, 1)[0])
        dl.append(take(np.int32, nd))
        ne = int(take(np.int32, 1)[0])
        el.append(take(np.int32, ne))
        doff.append(doff[-1] + nd)
        eoff.append(eoff[-1] + ne)
    if off != len(raw):
        raise RuntimeError("kick_probe output has %d trailing bytes" % (len(raw) - off))
    it["max_parts"] = np.int64(max_parts)
    it["doff"], it["eoff"] = np.array(doff, np.int64), np.array(eoff, np.int64)
    it["dlist"] = np.concatenate(dl) if dl else np.zeros(0, np.int32)
    it["elist"] = np.concatenate(el) if el else np.zeros(0, np.int32)
    return it


def record():
    d = {}
    for name, x, theta, hsoft, bucket, blocks in cases():
        d[name + "/x"] = x
        d[name + "/params"] = np.array([theta, hsoft, bucket, blocks], np.float64)
        for k, v in run_probe(x, theta, hsoft, bucket, blocks).items():
            d[name + "/" + k] = v
    return d


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--check", action="store_true")
    a = ap.parse_args()
    d = record()
    if a.check:
        old = np.load(OUT)
        bad = [key for key in d if key not in old.files or not np.array_equal(d[key], old[key])]
        bad += [key for key in old.files if key not in d]
        if bad:
            print("differs from the committed fixture:", bad)
            sys.exit(1)
        print("fresh recording equals", OUT)
        return
    np.savez_compressed(OUT, **d)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
