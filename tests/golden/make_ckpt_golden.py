"""Record checkpoints written by the reference's own code as fixtures
(tests/golden/ref_checkpoint.npz).

The reference's write_checkpoint (src/driver.cpp:1143-1173: driver_params, particles_save of
src/particles.cpp:1206-1227, domains_save of src/domain.cpp:87-94) runs for one rank, compiled
where it lies by `make -C oracle ckpt` (oracle/ckpt_probe.cpp, single-threaded HPX stand-in),
on a seeded state: its particles, a driver_params record with every field set, and a rung
ladder built by the reference's particles_sort_by_rung / particles_push_rungs /
particles_pop_rungs from the operations in OPS; the domain section is its one-rank
decomposition (domains_rebound).  For each case the fixture holds the input state, the
operations and the file the reference wrote, byte for byte.

    python tests/golden/make_ckpt_golden.py            # writes tests/golden/ref_checkpoint.npz
    python tests/golden/make_ckpt_golden.py --check    # compares a fresh recording with it

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

OUT = os.path.join(HERE, "ref_checkpoint.npz")
PROBE = os.path.join(ROOT, "oracle", "_ref", "ckpt_probe")
ITER = 7


def cases():
    """(name, params, x, y, z, v, rung, ops)."""
    from cosmictiger_b200 import checkpoint as ck

    out = []
    rng = np.random.default_rng(3)
    n = 257
    x, y, z = (rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32) for _ in range(3))
    v = rng.standard_normal((n, 3)).astype(np.float32)
    r = rng.integers(0, 6, n).astype(np.int8)
    p = ck.default_params(a=0.5, adot=1.25, dummy=0.0, tau=0.3, tau_max=2.0, energy0=-0.75, max_rung=5, iter=ITER, minrung0=1, step=12, bucket_size=128,
                          total_processed=123456789, flops=1.5e12, runtime=3.5, years=1.2e9, itime=99)
    for i, f in enumerate(p["energies"].dtype.names):
        p["energies"][f] = -1.5 + 0.25 * i
    # a three-level ladder in the middle of a step: two saved range starts
    out.append(("ladder257", p, x, y, z, v, r, ["1", "push", "2", "push", "3"]))
    # all particles active, empty stack (the state at the start of a step)
    out.append(("flat257", p, x, y, z, v, r, []))
    # no particles at all
    e = np.zeros(0, np.uint32)
    out.append(("empty", ck.default_params(a=1.0, iter=ITER), e, e, e, np.zeros((0, 3), np.float32), np.zeros(0, np.int8), []))
    return out


def run_probe(params, x, y, z, v, r, ops):
    """The bytes of checkpoint.<ITER>/checkpoint.0.dat as the reference writes them."""
    from cosmictiger_b200 import checkpoint as ck

    with tempfile.TemporaryDirectory() as tmp:
        st = os.path.join(tmp, "state.bin")
        with open(st, "wb") as f:
            f.write(np.asarray(params, ck.DRIVER_PARAMS).tobytes())
            f.write(np.int64(len(x)).tobytes())
            for a in (x, y, z):
                f.write(np.ascontiguousarray(a, np.uint32).tobytes())
            f.write(np.ascontiguousarray(v, np.float32).tobytes())
            f.write(np.ascontiguousarray(r, np.int8).tobytes())
        subprocess.run([PROBE, "write", st, str(ITER)] + list(ops), cwd=tmp, check=True, stdout=subprocess.DEVNULL)
        with open(os.path.join(tmp, "checkpoint.%d" % ITER, "checkpoint.0.dat"), "rb") as f:
            return np.frombuffer(f.read(), np.uint8).copy()


def resave(raw):
    """The reference's read_checkpoint of the file `raw` followed by its write_checkpoint of what
    it loaded (same path): the bytes it writes back."""
    with tempfile.TemporaryDirectory() as tmp:
        d = os.path.join(tmp, "checkpoint.%d" % ITER)
        os.makedirs(d)
        path = os.path.join(d, "checkpoint.0.dat")
        with open(path, "wb") as f:
            f.write(np.asarray(raw, np.uint8).tobytes())
        subprocess.run([PROBE, "resave", str(ITER)], cwd=tmp, check=True, stdout=subprocess.DEVNULL)
        with open(path, "rb") as f:
            return np.frombuffer(f.read(), np.uint8).copy()


def record():
    from cosmictiger_b200 import checkpoint as ck

    d = {}
    for name, p, x, y, z, v, r, ops in cases():
        d[name + "/params"] = np.frombuffer(np.asarray(p, ck.DRIVER_PARAMS).tobytes(), np.uint8).copy()
        d[name + "/x"] = np.stack([x, y, z])
        d[name + "/v"] = v
        d[name + "/rung"] = r
        d[name + "/ops"] = np.array(ops, dtype="U8")
        d[name + "/file"] = run_probe(p, x, y, z, v, r, ops)
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
