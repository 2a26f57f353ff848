"""The IC generator's and the power spectrum's oracle against the reference's own initial
conditions and power spectra (CPU; the device generator and power spectrum, ct_initialize and
ct_power_spectrum, are compared with the same oracle in tests/test_gpu_fourier.py).

tests/golden/ref_ic.npz holds the output of the reference's initialize() (src/initialize.cpp:
261-355,436-898) with its 3-D transform (src/fft.cpp) compiled where they lie
(oracle/ic_probe.cpp; tests/golden/make_ic_golden.py): lattice positions displaced by the
Zel'dovich field of a Gaussian field drawn with GSL's taus generator per k-space row, with and
without the 2LPT correction, for two cosmologies and grids.  The numpy restatement
(oracle/fourier_oracle.py, double-precision transforms) must give the same particles: the
reference transforms in single precision and keeps its normalisation and growth factors in
floats, so positions and velocities carry tolerances written below -- relative to the RMS
displacement for the whole field, and relative to the RMS of the 2LPT correction alone for the
difference the correction makes.  The same file holds the reference's power spectrum
(src/power.cpp:24-77, src/fft.cpp:172-360, the density kernel of src/power.cu:31-67) of seeded
Poisson and clustered particle sets at two grids and folds.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import fourier_oracle as F  # noqa: E402

FIX = os.path.join(HERE, "golden", "ref_ic.npz")


@pytest.fixture(scope="module")
def fix():
    return np.load(FIX)


def _case(fix, name):
    N, box, z0, om, hub, s8, twolpt = fix[name + "/params"]
    k, P = fix[name + "/table"]
    return int(N), float(box), float(z0), float(om), float(hub), float(s8), bool(twolpt), k, P


def _oracle(N, box, z0, om, hub, s8, twolpt, k, P):
    # code units of the reference's run: box 1, H0 1
    return F.initialize(N, box, om, z0, hub, s8, 1.0, k, P, twolpt)


def _disp(x, lat, N):
    """Displacement from the lattice in mean spacings (fixed32, wrapped)."""
    return ((x.astype(np.int64) - lat.astype(np.int64) + 2 ** 31) % 2 ** 32 - 2 ** 31) / 2 ** 32 * N


@pytest.mark.parametrize("name", ["zeldovich16", "twolpt16", "twolpt12"])
def test_oracle_equals_reference_initial_conditions(fix, name):
    """Positions within 2e-5 of the RMS displacement and velocities within 2e-5 of their RMS
    (measured: below 6e-6), growth factors and velocity prefactors within 1e-6 (float)."""
    N, box, z0, om, hub, s8, twolpt, k, P = _case(fix, name)
    ox, oy, oz, ov, fac = _oracle(N, box, z0, om, hub, s8, twolpt, k, P)
    rfac = fix[name + "/factors"]
    for i, key in enumerate(("D1", "D2", "prefac1", "prefac2")):
        assert abs(rfac[i] - fac[key]) <= 1e-6 * abs(fac[key]), key
    L = F.lattice(N)
    rx, rv = fix[name + "/x"], fix[name + "/v"]
    for d, mine in enumerate((ox, oy, oz)):
        dr, dm = _disp(rx[d], L[d], N), _disp(mine, L[d], N)
        rms = np.sqrt(np.mean(dr ** 2))
        assert 0.005 < rms < 0.5, rms
        assert np.max(np.abs(dm - dr)) < 2e-5 * rms, (d, np.max(np.abs(dm - dr)) / rms)
        vrms = np.sqrt(np.mean(rv[d].astype(np.float64) ** 2))
        assert np.max(np.abs(ov[:, d] - rv[d])) < 2e-5 * vrms, d


def test_oracle_2lpt_correction_equals_reference(fix):
    """The difference the 2LPT correction makes (twolpt16 minus zeldovich16, same field): within
    3e-4 of its own RMS in positions (fixed32 quantisation of a correction of ~1e-5 of the box
    is ~3e-5 of it) and in velocities (measured: 6e-5 and 2e-5)."""
    N, box, z0, om, hub, s8, _, k, P = _case(fix, "twolpt16")
    o0 = _oracle(N, box, z0, om, hub, s8, False, k, P)
    o1 = _oracle(N, box, z0, om, hub, s8, True, k, P)
    L = F.lattice(N)
    r0x, r1x = fix["zeldovich16/x"], fix["twolpt16/x"]
    r0v, r1v = fix["zeldovich16/v"], fix["twolpt16/v"]
    for d in range(3):
        cr = _disp(r1x[d], L[d], N) - _disp(r0x[d], L[d], N)
        co = _disp(o1[d], L[d], N) - _disp(o0[d], L[d], N)
        rms = np.sqrt(np.mean(co ** 2))
        assert rms > 1e-5, rms  # the correction is there
        assert np.max(np.abs(cr - co)) < 3e-4 * rms, (d, np.max(np.abs(cr - co)) / rms)
        vr = r1v[d].astype(np.float64) - r0v[d]
        vo = o1[3][:, d] - o0[3][:, d]
        assert np.max(np.abs(vr - vo)) < 3e-4 * np.sqrt(np.mean(vo ** 2)), d


def power_names(fix):
    return sorted({k.split("/")[1] for k in fix.files if k.startswith("power/")})


def test_oracle_power_spectrum_equals_reference(fix):
    """Every bin's k within 1e-6, P and its error within 5e-5 relative (the reference deposits
    and transforms in single precision; measured: below 1.3e-5), and the same empty bins."""
    names = power_names(fix)
    assert len(names) == 4
    for name in names:
        x = fix["power/" + name + "/x"]
        N, fold, box = fix["power/" + name + "/params"]
        k, P, E = fix["power/" + name + "/kpe"]
        ok, oP, oE, cnt = F.power_spectrum(x[0], x[1], x[2], int(N), int(fold), float(box))
        assert len(ok) == len(k), name
        assert np.max(np.abs(k - ok) / ok) < 1e-6, name
        assert np.array_equal(P == 0, oP == 0), name
        nz = oP > 0
        assert nz.sum() >= 10, name
        assert np.max(np.abs(P[nz] - oP[nz]) / oP[nz]) < 5e-5, name
        assert np.max(np.abs(E[nz] - oE[nz]) / oE[nz]) < 5e-5, name


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "ic_probe")), reason="reference IC probe not built here")
def test_fixture_equals_a_fresh_run_of_the_reference():
    """Where the probe is built, a fresh recording from the reference's code equals the committed
    fixture (guards the fixture against drift of the generator or the probe)."""
    res = subprocess.run([sys.executable, os.path.join(HERE, "golden", "make_ic_golden.py"), "--check"], capture_output=True, text=True, cwd=ROOT)
    assert res.returncode == 0, res.stdout + res.stderr
