"""The CPU top of the kick and its work items against the reference's own (CPU).

tests/golden/ref_kick_items.npz holds the work items the reference's kick() (src/kick.cpp:
150-507 with src/gravity.cpp) hands to its GPU workspace when it starts a step over its own
tree (oracle/kick_probe.cpp; tests/golden/make_kick_golden.py): subtree root, incoming
expansion, its centre, direct and Ewald check lists, ordered by first particle.  This
project's CPU oracle (O1) restates that top (ct_or_kick_plan_*); its items feed the reference's
CUDA kick in tests/test_reference_kick.py and the CPU legs of bench.py.  O1 must give the same
items in the same order, the same centres and the same check lists, with two differences that
carry no work: O1 also lists the subtrees without particles as items (the reference skips
them), and it leaves out of its check lists the nodes without particles, which the reference
carries in its lists (they contribute nothing).  The expansions agree to single-precision
rounding (the reference sums its interactions eight at a time in SIMD lanes, O1 one at a time).
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from tests import oracle_lib

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
FIX = os.path.join(HERE, "golden", "ref_kick_items.npz")


def _cases():
    return sorted({k.split("/")[0] for k in np.load(FIX).files})


@pytest.fixture(scope="module")
def fix():
    return np.load(FIX)


@pytest.fixture(scope="module")
def oracle():
    return oracle_lib.load()


@pytest.mark.parametrize("name", _cases())
def test_oracle_work_items_equal_reference(fix, oracle, name):
    """Same items, centres and (non-empty) check lists, bit for bit; expansions within 2e-5
    relative RMS over all items and 5e-4 of each component's largest magnitude (measured: below
    6e-6 and 3e-5)."""
    x, y, z = (fix[name + "/x"][k].copy() for k in range(3))
    theta, hsoft, bucket, _ = fix[name + "/params"]
    n = len(x)
    v = np.zeros((n, 3), np.float32)
    r = np.zeros(n, np.int8)
    nodes = oracle.tree_build(x, y, z, v, r, float(theta), float(hsoft), int(bucket))
    kp = oracle_lib.KickParams(sign=1.0, min_rung=0, a=1.0, t0=1.0, theta=float(theta), h=float(hsoft), eta=0.2, GM=1.0 / n, max_dt=1e30, save_force=0,
                               first_call=1, ascending=1, descending=1, top=1, do_phi=1)
    plan = oracle.plan(kp, nodes, x, y, z, order=7, max_parts=int(fix[name + "/max_parts"]))
    ex = plan.export(nexp=50)
    plan.close()
    nonempty = nodes["part_end"] > nodes["part_begin"]
    # O1 also lists the subtrees without particles below its top as items (no particles, no
    # work); the reference hands them to nobody (kick.cpp:178-181)
    keep = np.nonzero(nonempty[ex["self"]])[0]
    assert np.array_equal(ex["self"][keep], fix[name + "/self"])
    assert np.array_equal(ex["pos"][keep], fix[name + "/pos"])
    for lst, off in (("dlist", "doff"), ("elist", "eoff")):
        ro, rl = fix[name + "/" + off], fix[name + "/" + lst]
        for j, i in enumerate(keep):
            mine = ex[lst][ex[off][i]:ex[off][i + 1]]
            ref = rl[ro[j]:ro[j + 1]]
            assert np.array_equal(mine[nonempty[mine]], ref[nonempty[ref]]), (name, lst, j)
    Lr = fix[name + "/L"].astype(np.float64)
    Lo = ex["L"][keep].astype(np.float64)
    if not np.any(Lr):
        # no interaction above the items (the top's nodes are all near one another)
        assert not np.any(Lo)
        return
    assert np.sqrt(np.sum((Lr - Lo) ** 2) / np.sum(Lr ** 2)) < 2e-5
    # each component against its largest magnitude over the items, with a floor of 1e-9 of the
    # largest component overall: on a lattice, components that cancel by symmetry are rounding
    # noise of ~1e-21 on both sides
    scale = np.max(np.abs(Lr), axis=0)
    assert np.all(np.abs(Lr - Lo) <= 5e-4 * scale + 1e-9 * np.max(np.abs(Lr)))


def test_fixture_covers_the_item_rules(fix):
    """Items of at most a bucket (a B200's 1,184 kick blocks), larger items under a deeper CPU
    top (few blocks), a lattice and clustered boxes."""
    assert int(fix["clustered24_b1184/max_parts"]) == 128
    assert int(fix["clustered24_b8/max_parts"]) > 1000
    assert len(fix["clustered24_b1184/self"]) > 100 and len(fix["lattice16_b64/self"]) > 10
    assert np.any(fix["clustered16_b64/L"]) and np.any(fix["clustered24_b1184/L"])  # far interactions above the items


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "kick_probe")), reason="reference kick probe not built here")
def test_fixture_equals_a_fresh_run_of_the_reference():
    """Where the probe is built, a fresh recording from the reference's code equals the committed
    fixture (guards the fixture against drift of the generator or the probe)."""
    res = subprocess.run([sys.executable, os.path.join(HERE, "golden", "make_kick_golden.py"), "--check"], capture_output=True, text=True, cwd=ROOT)
    assert res.returncode == 0, res.stdout + res.stderr
