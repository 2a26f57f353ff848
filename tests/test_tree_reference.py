"""The tree build against the reference's own code (CPU; the device build is compared in
tests/test_gpu_parity.py::test_tree_matches_reference_fixtures).

tests/golden/ref_tree.npz holds the output of the reference's tree_create and particles_sort
(src/tree.cpp:273-601, src/particles.cpp:979-1018) compiled where they lie
(oracle/tree_probe.cpp; tests/golden/make_tree_golden.py): an IEEE build and one with the
reference's own flags (--fast-math -march=native).  This project's CPU restatement (O1) must
give the IEEE build's tree bit for bit -- heap keys, particle ranges, children, centres, radii,
boxes, leaf flags, depths, particle order -- and the native build's keys, ranges, boxes, leaf
flags, depths and order, with its centres and radii within what its contracted arithmetic
changes.  The case with more than a bucket of coincident particles must stop with the
reference's "Maximum depth exceeded".  The same file holds the reference's rung partition
(particles_sort_by_rung with push/pop of the active range, src/particles.cpp:218-235,
1029-1076) over a sequence of operations, which O1 must reproduce exactly.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from tests import oracle_lib

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "ref_tree.npz")
ROOT = os.path.dirname(HERE)
FIELDS = ("key", "part_begin", "part_end", "child_left", "child_right", "pos", "box_begin", "box_end", "leaf", "depth")


def fixture_cases():
    d = np.load(FIX)
    return sorted({k.split("/")[0] for k in d.files} - {"rungs"})


@pytest.fixture(scope="module")
def fix():
    return np.load(FIX)


@pytest.fixture(scope="module")
def oracle():
    return oracle_lib.load()


@pytest.mark.parametrize("case", fixture_cases())
def test_oracle_tree_equals_reference_tree(fix, oracle, case):
    x, y, z = (fix[case + "/in"][k].copy() for k in range(3))
    theta, hsoft, bucket = fix[case + "/params"]
    n = len(x)
    v = np.zeros((n, 3), np.float32)
    r = np.zeros(n, np.int8)
    if bool(fix[case + "/threw"]):
        with pytest.raises(RuntimeError, match="maximum depth exceeded"):
            oracle.tree_build(x, y, z, v, r, float(theta), float(hsoft), int(bucket))
        return
    nodes = oracle.tree_build(x, y, z, v, r, float(theta), float(hsoft), int(bucket))
    assert len(nodes) == len(fix[case + "/key"])
    for f in FIELDS:
        assert np.array_equal(nodes[f], fix[case + "/" + f]), f
    assert np.array_equal(nodes["radius"].view(np.uint32), fix[case + "/radius"].view(np.uint32)), "radius"
    after = fix[case + "/after"]
    assert np.array_equal(x, after[0]) and np.array_equal(y, after[1]) and np.array_equal(z, after[2]), "particle order"
    # the reference built with its own flags: the same tree up to contracted arithmetic in the
    # node geometry (at most 1 ulp in a radius and 64 units of 2^-32 in a centre here)
    assert np.abs(fix[case + "/native_radius_ulps"]).max() <= 1
    assert np.abs(fix[case + "/native_pos_delta"]).max() <= 64


def test_fixture_covers_the_tree_rules(fix):
    """Cases: a clustered box, a lattice, a deep core with a small bucket, one particle (split
    by the Ewald criterion alone), a full bucket of coincident particles and one more (the
    reference's maximum-depth error)."""
    cases = fixture_cases()
    assert {"clustered10", "lattice10", "core1200", "one", "coincident128", "coincident129"} <= set(cases)
    assert bool(fix["coincident129/threw"]) and not bool(fix["coincident128/threw"])
    assert fix["core1200/depth"].max() > fix["lattice10/depth"].max()
    assert len(fix["one/key"]) > 1  # the Ewald criterion splits a single particle's box


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "tree_probe")), reason="reference tree probe not built here")
def test_fixture_equals_a_fresh_run_of_the_reference():
    """Where the probes are built, a fresh recording from the reference's code equals the
    committed fixture (guards the fixture against drift of the generator or the probe)."""
    res = subprocess.run([sys.executable, os.path.join(HERE, "golden", "make_tree_golden.py"), "--check"], capture_output=True, text=True, cwd=ROOT)
    assert res.returncode == 0, res.stdout + res.stderr


def test_oracle_rung_partition_equals_reference(fix, oracle):
    """O1's rung partition and an active-range stack give the reference's range starts after
    every operation and its final particle order, velocities and rungs, bit for bit."""
    x, y, z = (fix["rungs/in_x"][k].copy() for k in range(3))
    v = fix["rungs/in_v"].copy()
    r = fix["rungs/in_rung"].copy()
    begin, stack, got = 0, [], []
    for op in fix["rungs/ops"]:
        if op == "push":
            stack.append(begin)
        elif op == "pop":
            begin = stack.pop()
        else:
            m = int(op)
            begin = 0 if m == 0 else oracle.sort_by_rung(x, y, z, v, r, m, begin)
        got.append(begin)
    assert got == [int(b) for b in fix["rungs/begins"]]
    assert np.array_equal(np.stack([x, y, z]), fix["rungs/x"])
    assert np.array_equal(v, fix["rungs/v"]) and np.array_equal(r, fix["rungs/rung"])
