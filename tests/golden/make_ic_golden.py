"""Record the reference's own initial conditions and power spectra as fixtures
(tests/golden/ref_ic.npz).

The reference's initialize() (src/initialize.cpp:261-355,436-898: the lattice, the Zel'dovich
displacements of a Gaussian field drawn with GSL's taus generator per k-space row, and the 2LPT
correction) runs with its distributed 3-D transform (src/fft.cpp), particle arrays and growth
factor compiled where they lie by `make -C oracle ic` (oracle/ic_probe.cpp; HPX is the
single-threaded stand-in of oracle/stub/hpx, FFTW's one-line transforms plain discrete Fourier
sums in double precision stored as floats).  For each case below this script writes the
power.init table the reference reads, the cosmology, and the reference's particle positions
(fixed32), velocities and growth factors.  The same probe runs the reference's matter power
spectrum (power_spectrum_compute, src/power.cpp:24-77, binned by src/fft.cpp:172-360, the
density deposited by the kernel of src/power.cu:31-67 run on the host) on seeded particle sets
("power/..." entries: the particles, grid, fold and the reference's k, P and error per bin).

    python tests/golden/make_ic_golden.py            # writes tests/golden/ref_ic.npz
    python tests/golden/make_ic_golden.py --check    # compares a fresh recording with it

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

OUT = os.path.join(HERE, "ref_ic.npz")
PROBE = os.path.join(ROOT, "oracle", "_ref", "ic_probe")


def cases():
    """(name, N, box [Mpc], z0, omega_m, hubble, sigma8, twolpt, k, P): the table is the smooth
    power.init-style spectrum of cosmictiger_b200.ics, cut at a fraction of the grid's Nyquist
    wavenumber, in single precision (the reference reads it with %f)."""
    from cosmictiger_b200 import ics

    out = []
    cos1 = dict(z0=49.0, omega_m=0.3111, hubble=0.6732, sigma8=0.8607)
    k, P = ics.power_law_table(kcut=0.25 * np.pi * 16 / 100.0 / cos1["hubble"])
    out.append(("zeldovich16", 16, 100.0, *cos1.values(), 0, k, P))
    out.append(("twolpt16", 16, 100.0, *cos1.values(), 1, k, P))
    # another box, redshift, cosmology and spectral slope, with the 2LPT correction
    cos2 = dict(z0=9.0, omega_m=0.25, hubble=0.7, sigma8=0.8)
    k, P = ics.power_law_table(index=-2.0, kcut=0.4 * np.pi * 12 / 250.0 / cos2["hubble"])
    out.append(("twolpt12", 12, 250.0, *cos2.values(), 1, k, P))
    return out


def run_probe(N, box, z0, omega_m, hubble, sigma8, twolpt, k, P):
    """The reference's initialize(): (x, y, z) uint32 (3, n), v float32 (3, n), factors float32
    (D1, D2, prefac1, prefac2)."""
    with tempfile.TemporaryDirectory() as tmp:
        table, out = os.path.join(tmp, "table.txt"), os.path.join(tmp, "out.bin")
        with open(table, "w") as f:
            for a, b in zip(k, P):
                f.write("%.9g %.9g\n" % (a, b))
        subprocess.run([PROBE, str(N), repr(box), repr(z0), repr(omega_m), repr(hubble), repr(sigma8), str(int(twolpt)), table, out], cwd=tmp,
                       check=True, stdout=subprocess.DEVNULL)
        raw = open(out, "rb").read()
    n = int(np.frombuffer(raw[:8], np.int64)[0])
    xyz = np.frombuffer(raw[8:8 + 12 * n], np.uint32).reshape(3, n).copy()
    v = np.frombuffer(raw[8 + 12 * n:8 + 24 * n], np.float32).reshape(3, n).copy()
    fac = np.frombuffer(raw[8 + 24 * n:8 + 24 * n + 16], np.float32).copy()
    return xyz, v, fac


def power_cases():
    """(name, x (3, n) uint32, N, fold): n >= N^3 particles, so that the reference deposits the
    density in one box (its sub-box path, for fewer particles than cells per rank, deposits
    particles of neighbouring boxes too and writes up to one cell below and two above each box's
    array, src/power.cpp:44-61 with src/power.cu:41-57)."""
    from cosmictiger_b200 import ics

    rng = np.random.default_rng(5)
    uni = rng.integers(0, 2 ** 32, (3, 16 ** 3), dtype=np.uint64).astype(np.uint32)
    cx, cy, cz, _, _ = ics.clustered_box(16, nspheres=20, seed=31)
    clu = np.stack([cx, cy, cz])
    return [("uniform16_n16_f1", uni, 16, 1), ("uniform16_n16_f2", uni, 16, 2), ("clustered16_n16_f1", clu, 16, 1), ("clustered16_n8_f2", clu, 8, 2)]


POWER_BOX = 100.0  # Mpc; scales k only


def run_power(x, N, fold):
    """The reference's power spectrum of particles x (3, n): k, P, Perr (float32)."""
    with tempfile.TemporaryDirectory() as tmp:
        parts, out = os.path.join(tmp, "parts.bin"), os.path.join(tmp, "ps.bin")
        with open(parts, "wb") as f:
            f.write(np.int64(x.shape[1]).tobytes())
            f.write(np.ascontiguousarray(x, np.uint32).tobytes())
        subprocess.run([PROBE, "power", str(N), str(fold), repr(POWER_BOX), parts, out], cwd=tmp, check=True, stdout=subprocess.DEVNULL)
        raw = open(out, "rb").read()
    m = int(np.frombuffer(raw[:8], np.int64)[0])
    return np.frombuffer(raw[8:8 + 12 * m], np.float32).reshape(3, m).copy()


def record():
    d = {}
    for name, x, N, fold in power_cases():
        d["power/" + name + "/x"] = x
        d["power/" + name + "/params"] = np.array([N, fold, POWER_BOX], np.float64)
        d["power/" + name + "/kpe"] = run_power(x, N, fold)
    for name, N, box, z0, om, hub, s8, twolpt, k, P in cases():
        xyz, v, fac = run_probe(N, box, z0, om, hub, s8, twolpt, k, P)
        d[name + "/params"] = np.array([N, box, z0, om, hub, s8, twolpt], np.float64)
        d[name + "/table"] = np.stack([k, P]).astype(np.float32)
        d[name + "/x"] = xyz
        d[name + "/v"] = v
        d[name + "/factors"] = fac
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
