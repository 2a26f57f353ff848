"""The CPU oracle's tree build (tree_create, src/tree.cpp:273-601, with the partition of
particles_sort, src/particles.cpp:979-1018) against an independent pure-Python restatement of
the same loop at small sizes, its structural invariants, and the edge cases the reference
defines: an empty box, a single particle, a bucket of coincident particles and one more than a
bucket (the reference throws "Maximum depth exceeded", tree.cpp:285-286, MAX_DEPTH 128 in
cosmictiger/defs.hpp:86).  The device build is compared with this oracle bit for bit in
test_gpu_parity.py."""
import numpy as np
import pytest


def _random_box(n, seed):
    rng = np.random.default_rng(seed)
    x, y, z = (rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32) for _ in range(3))
    v = rng.standard_normal(3 * n).astype(np.float32)
    r = rng.integers(0, 4, n).astype(np.int8)
    return x, y, z, v, r


def _py_partition(X, v, r, b, e, xm, xdim):
    """particles_sort (particles.cpp:979-1018): lo scans up; at an element >= xmid, hi scans
    down for one < xmid and the two swap.  xmid = fixed32(xm) truncates 2^32 xm."""
    xmid = int(np.uint64(np.float64(xm) * 4294967296.0))
    lo, hi = b, e
    d = X[xdim]
    while lo < hi:
        if d[lo] >= xmid:
            while lo != hi:
                hi -= 1
                if d[hi] < xmid:
                    for a in X:
                        a[hi], a[lo] = a[lo], a[hi]
                    v[3 * hi:3 * hi + 3], v[3 * lo:3 * lo + 3] = v[3 * lo:3 * lo + 3].copy(), v[3 * hi:3 * hi + 3].copy()
                    r[hi], r[lo] = r[lo], r[hi]
                    break
        lo += 1
    return hi


def _py_tree(X, v, r, theta, h, bucket):
    """Keys, particle ranges, leaf flags and depths of tree_create's recursion (tree.cpp:313-350):
    box_r accumulated in float, the Ewald leaf test, the split at the midpoint of the longest
    dimension (the first of equal spans, range.hpp:212-223)."""
    out = {}

    def rec(key, b, e, lo_box, hi_box, depth):
        box_r = np.float32(0.0)
        for d in range(3):
            s = 0.5 * (hi_box[d] - lo_box[d])
            box_r = np.float32(np.float64(box_r) + s * s)
        box_r = np.sqrt(box_r)
        ewald = float(box_r) < 0.25 * (theta / (1.0 + theta)) and float(box_r) < 0.125 - 0.25 * h
        n = e - b
        if n > bucket or (not ewald and n > 0):
            xdim, span = 0, -1.0
            for d in range(3):
                if hi_box[d] - lo_box[d] > span:
                    span, xdim = hi_box[d] - lo_box[d], d
            xm = 0.5 * (hi_box[xdim] + lo_box[xdim])
            mid = _py_partition(X, v, r, b, e, xm, xdim)
            lh, rl = list(hi_box), list(lo_box)
            lh[xdim] = rl[xdim] = xm
            rec(2 * key + 1, mid, e, rl, hi_box, depth + 1)
            rec(2 * key, b, mid, lo_box, lh, depth + 1)
            out[key] = (b, e, 0, depth)
        else:
            out[key] = (b, e, 1, depth)

    rec(1, 0, len(X[0]), [0.0] * 3, [1.0] * 3, 0)
    return out


@pytest.mark.parametrize("n,theta,bucket,seed", [(300, 0.7, 8, 1), (500, 0.55, 16, 2), (64, 0.4, 4, 3)])
def test_tree_matches_independent_restatement(oracle, n, theta, bucket, seed):
    x, y, z, v, r = _random_box(n, seed)
    h = 1e-3
    px = [x.astype(np.int64).tolist(), y.astype(np.int64).tolist(), z.astype(np.int64).tolist()]
    pv, pr = v.copy(), r.copy()
    want = _py_tree(px, pv, pr, theta, h, bucket)
    nodes = oracle.tree_build(x, y, z, v, r, theta, h, bucket)
    got = {int(nd["key"]): (int(nd["part_begin"]), int(nd["part_end"]), int(nd["leaf"]), int(nd["depth"])) for nd in nodes}
    assert got == want
    assert x.tolist() == px[0] and y.tolist() == px[1] and z.tolist() == px[2]
    assert np.array_equal(v, pv) and np.array_equal(r, pr)


def test_tree_structure_invariants(oracle):
    """Children split their parent's range at one point, leaves tile [0, n) in key order, no
    leaf holds more than a bucket, and the particles are a permutation of the input."""
    x, y, z, v, r = _random_box(4000, 7)
    orig = sorted(zip(x.tolist(), y.tolist(), z.tolist()))
    bucket = 32
    nodes = oracle.tree_build(x, y, z, v, r, 0.7, 1e-3, bucket)
    assert sorted(zip(x.tolist(), y.tolist(), z.tolist())) == orig
    by_key = {int(nd["key"]): nd for nd in nodes}
    assert len(by_key) == len(nodes)
    root = by_key[1]
    assert (root["part_begin"], root["part_end"], root["depth"]) == (0, 4000, 0)
    for k, nd in by_key.items():
        if nd["leaf"]:
            assert nd["part_end"] - nd["part_begin"] <= bucket
            assert 2 * k not in by_key and 2 * k + 1 not in by_key
            continue
        lc, rc = by_key[2 * k], by_key[2 * k + 1]
        assert lc["part_begin"] == nd["part_begin"] and rc["part_end"] == nd["part_end"]
        assert lc["part_end"] == rc["part_begin"]
        assert lc["depth"] == rc["depth"] == nd["depth"] + 1
    # every particle lies inside its leaf's tight box (fixed<int,29>: 2^-29 box units)
    for nd in nodes[nodes["leaf"] == 1]:
        b, e = int(nd["part_begin"]), int(nd["part_end"])
        for d, a in enumerate((x, y, z)):
            q = a[b:e].astype(np.int64) >> 3
            if e > b:
                assert q.min() >= nd["box_begin"][d] and q.max() <= nd["box_end"][d]


def test_tree_empty_and_single_particle(oracle):
    """No particles: the root alone, a leaf.  One particle: the Ewald criterion still splits
    every non-empty node until its box is small enough, while empty nodes stop at once."""
    e = _random_box(0, 1)
    nodes = oracle.tree_build(*e, 0.7, 1e-3, 128)
    assert len(nodes) == 1 and nodes[0]["leaf"] == 1 and nodes[0]["part_end"] == 0
    s = _random_box(1, 2)
    nodes = oracle.tree_build(*s, 0.7, 1e-3, 128)
    nonempty = nodes[nodes["part_end"] > nodes["part_begin"]]
    # one chain from the root to the leaf holding the particle; every split makes an empty sibling
    assert len(nonempty) == nodes["depth"].max() + 1
    assert len(nodes) == 2 * nodes["depth"].max() + 1
    leaf = nonempty[nonempty["leaf"] == 1]
    assert len(leaf) == 1
    half = (leaf[0]["box_end"] - leaf[0]["box_begin"]).astype(np.float64)
    assert np.all(half >= 0)


def test_tree_coincident_particles(oracle):
    """A bucket of coincident particles fits one leaf; one more cannot be split before depth
    128, where the reference throws and the oracle reports the same failure."""
    def same(n):
        x = np.full(n, 123456789, np.uint32)
        y = np.full(n, 987654321, np.uint32)
        z = np.full(n, 2 ** 31, np.uint32)
        return x, y, z, np.zeros(3 * n, np.float32), np.zeros(n, np.int8)

    nodes = oracle.tree_build(*same(128), 0.7, 1e-3, 128)
    assert nodes["depth"].max() < 127
    with pytest.raises(RuntimeError, match="maximum depth"):
        oracle.tree_build(*same(129), 0.7, 1e-3, 128)
