"""Record the reference's own hierarchical step as a fixture (tests/golden/ref_ladder.npz).

oracle/ladder_probe.cpp (`make -C oracle ladder`) runs the reference's kick_step_hierarchical
(src/driver.cpp:382-593) compiled where it lies, with its tree build and rung partition, for
STEPS steps on a seeded clustered box; its kick and drift are this project's CPU restatement
(oracle/libct_oracle.so, pinned against the reference's CUDA kernels elsewhere).  The fixture
holds the input state and parameters, after each step the ladder's minimum rung, maximum rung
and active-range start with a SHA-256 digest of the particle state, the final state, and a
digest of the oracle sources it was recorded with (re-record when they change).

    python tests/golden/make_ladder_golden.py            # writes tests/golden/ref_ladder.npz
    python tests/golden/make_ladder_golden.py --check    # compares a fresh recording with it
"""
import argparse
import hashlib
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

OUT = os.path.join(HERE, "ref_ladder.npz")
PROBE = os.path.join(ROOT, "oracle", "_ref", "ladder_probe")
STEPS = 4


def oracle_digest():
    """SHA-256 of the sources of the oracle's kick and drift (the probe's stand-ins for the
    reference's GPU calls): a fixture recorded with other sources no longer applies."""
    h = hashlib.sha256()
    for f in ("cosmictiger_b200/csrc/fmm_p7.h", "cosmictiger_b200/csrc/fmm_common.h", "oracle/ct_oracle.cpp"):
        with open(os.path.join(ROOT, f), "rb") as fh:
            h.update(fh.read())
    return np.frombuffer(h.digest(), np.uint8)


def state_digest(x, y, z, v, r):
    h = hashlib.sha256()
    for a in (x, y, z, v, r):
        h.update(np.ascontiguousarray(a).tobytes())
    return np.frombuffer(h.digest(), np.uint8)


def case():
    """A clustered 12^3 box; t0 set so that the first step spreads the particles over rungs 0-4
    (a few percent of them above rung 2) and the ladder clips its top at the next step."""
    from cosmictiger_b200 import ics

    x, y, z, v, _ = ics.clustered_box(12, nspheres=30, seed=41)
    n = len(x)
    return dict(x=x, y=y, z=z, v=v, rung=np.zeros(n, np.int8), theta=0.55, hsoft=ics.softening(n, 0.02), bucket=128, GM=1.0 / n,
                eta=float(ics.eta_default()), t0=1.5e-3)


def run_probe(c, steps):
    n = len(c["x"])
    with tempfile.TemporaryDirectory() as tmp:
        fin, fout = os.path.join(tmp, "in.bin"), os.path.join(tmp, "out.bin")
        with open(fin, "wb") as f:
            np.array([n], np.int64).tofile(f)
            for k in ("x", "y", "z"):
                np.ascontiguousarray(c[k], np.uint32).tofile(f)
            np.ascontiguousarray(c["v"], np.float32).tofile(f)
            np.ascontiguousarray(c["rung"], np.int8).tofile(f)
        args = [PROBE, fin, fout, str(steps), "%.17g" % c["theta"], "%.17g" % c["hsoft"], str(c["bucket"]), "%.17g" % c["GM"], "%.17g" % c["eta"],
                "%.17g" % c["t0"]]
        res = subprocess.run(args, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError("ladder probe failed (%d): %s" % (res.returncode, res.stderr[-400:]))
        out = []
        with open(fout, "rb") as f:
            for _ in range(steps):
                mr, mx = (int(q) for q in np.fromfile(f, np.int32, 2))
                rb = int(np.fromfile(f, np.int64, 1)[0])
                xs = [np.fromfile(f, np.uint32, n) for _ in range(3)]
                vs = np.fromfile(f, np.float32, 3 * n).reshape(n, 3)
                rs = np.fromfile(f, np.int8, n)
                out.append((mr, mx, rb, xs, vs, rs))
    return out


def record():
    c = case()
    steps = run_probe(c, STEPS)
    data = {"in_x": np.stack([c["x"], c["y"], c["z"]]), "in_v": c["v"], "in_rung": c["rung"],
            "params": np.array([c["theta"], c["hsoft"], c["bucket"], c["GM"], c["eta"], c["t0"]], np.float64)}
    data["minrung"] = np.array([s[0] for s in steps], np.int32)
    data["max_rung"] = np.array([s[1] for s in steps], np.int32)
    data["rung_begin"] = np.array([s[2] for s in steps], np.int64)
    data["digest"] = np.stack([state_digest(*s[3], s[4], s[5]) for s in steps])
    mr, mx, rb, xs, vs, rs = steps[-1]
    data["final_x"] = np.stack(xs)
    data["final_v"] = vs
    data["final_rung"] = rs
    data["oracle_digest"] = oracle_digest()
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
    print("wrote", OUT, os.path.getsize(OUT), "bytes; minrung", data["minrung"], "max_rung", data["max_rung"], "begins", data["rung_begin"])


if __name__ == "__main__":
    main()
