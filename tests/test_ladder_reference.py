"""The hierarchical step's ladder against the reference's own kick_step_hierarchical (CPU).

tests/golden/ref_ladder.npz records the reference's kick_step_hierarchical
(src/driver.cpp:382-593) compiled where it lies, over its own tree build and rung partition,
with this project's CPU kick and drift standing in for the GPU calls (oracle/ladder_probe.cpp,
tests/golden/make_ladder_golden.py).  The CPU restatement of the ladder
(oracle_lib.step_hierarchical, which ct_step_hierarchical mirrors on the device and which the
device is compared with step by step in tests/test_gpu_parity_configs.py) must give the same
minimum and maximum rungs, active-range starts and particle states after every step, bit for
bit: the same levels, pushes and pops, kick flags (ascending, descending, top, first call, the
clipped top), drifts per rung and rung sorts.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from tests import oracle_lib
from tests.golden.make_ladder_golden import state_digest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
FIX = os.path.join(HERE, "golden", "ref_ladder.npz")


def reference_ladder():
    """The fixture, or a fresh recording where the probe is built and the fixture was made with
    other oracle sources (its kick and drift stand in for the reference's GPU calls)."""
    from tests.golden import make_ladder_golden as g

    d = dict(np.load(FIX))
    if np.array_equal(d["oracle_digest"], g.oracle_digest()):
        return d
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "ladder_probe")):
        pytest.skip("fixture recorded with other oracle sources and the reference ladder probe is not built here")
    return g.record()


def test_oracle_ladder_equals_reference_ladder():
    d = reference_ladder()
    O = oracle_lib.load()
    x, y, z = (d["in_x"][k].copy() for k in range(3))
    theta, hsoft, bucket, GM, eta, t0 = (float(q) for q in d["params"])
    st = dict(x=x, y=y, z=z, v=d["in_v"].copy(), rung=d["in_rung"].copy(), rung_begin=0, stack=[])
    minrung, max_rung, tau = 0, 0, 0.0
    for s in range(len(d["minrung"])):
        sp = dict(minrung=minrung, minrung0=0, max_rung=max_rung, a=1.0, tau=tau, t0=t0, theta=theta, hsoft=hsoft, bucket=int(bucket), eta=eta, GM=GM,
                  max_dt=1e30, do_phi=1, nocrop=0, drag=0.0, sign=1.0)
        _, minrung, max_rung = oracle_lib.step_hierarchical(O, st, sp)
        tau += t0
        assert (minrung, max_rung, st["rung_begin"]) == (int(d["minrung"][s]), int(d["max_rung"][s]), int(d["rung_begin"][s])), s
        assert np.array_equal(state_digest(st["x"], st["y"], st["z"], st["v"], st["rung"]), d["digest"][s]), "state after step %d" % s
    assert np.array_equal(np.stack([st["x"], st["y"], st["z"]]), d["final_x"])
    assert np.array_equal(st["v"], d["final_v"]) and np.array_equal(st["rung"], d["final_rung"])
    # the case exercises the clipped top (the minimum rung moves up) and several rungs
    assert d["minrung"][0] == 0 and d["minrung"][-1] == 1 and d["max_rung"].max() >= 3


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "ladder_probe")), reason="reference ladder probe not built here")
def test_fixture_equals_a_fresh_run_of_the_reference_ladder():
    res = subprocess.run([sys.executable, os.path.join(HERE, "golden", "make_ladder_golden.py"), "--check"], capture_output=True, text=True, cwd=ROOT)
    assert res.returncode == 0, res.stdout + res.stderr
