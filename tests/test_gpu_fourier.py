"""The IC generator (ct_initialize) and the power spectrum (ct_power_spectrum) on the device
against the numpy restatement of the reference's (oracle/fourier_oracle.py): same random field
(GSL taus per k-space row), same kernels and bins; single-precision cuFFT against double-precision
numpy, so the comparisons carry tolerances written below."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import fourier_oracle as F  # noqa: E402

from cosmictiger_b200 import ics  # noqa: E402

pytestmark = pytest.mark.gpu

COSMO = dict(omega_m=0.3111, z0=49.0, hubble=0.6732, sigma8=0.8607, H0=1.0)


@pytest.fixture(scope="module")
def ctx():
    import cosmictiger_b200 as ct

    c = ct.Context(order=7)
    yield c
    c.close()


def _table(N, box, frac):
    # power cut off at frac of the grid's Nyquist wavenumber (k in h / Mpc)
    return ics.power_law_table(kcut=frac * np.pi * N / box / COSMO["hubble"])


def _disp(x, lattice, N):
    d = (x.astype(np.int64) - lattice.astype(np.int64) + 2 ** 31) % 2 ** 32 - 2 ** 31
    return d / 2 ** 32 * N  # mean spacings


@pytest.mark.parametrize("twolpt", [False, True])
def test_initialize_matches_oracle(ctx, twolpt):
    """Positions and velocities of 32^3 particles agree with the double-precision restatement
    to 1e-4 of the RMS displacement (float transforms), and the growth factors to 1e-5."""
    N, box = 32, 100.0
    k, P = _table(N, box, 0.25)
    b = ctx.box(N ** 3)
    r = b.initialize(N, box, k, P, twolpt=twolpt, **COSMO)
    out = b.download()
    b.close()
    ox, oy, oz, ov, fac = F.initialize(N, box, COSMO["omega_m"], COSMO["z0"], COSMO["hubble"], COSMO["sigma8"], COSMO["H0"], k, P, twolpt)
    for key in ("D1", "D2", "prefac1", "prefac2", "norm"):
        assert abs(r[key] - fac[key]) <= 1e-5 * abs(fac[key]), key
    L = F.lattice(N)
    for d, (mine, ref) in enumerate(zip((out["x"], out["y"], out["z"]), (ox, oy, oz))):
        dm, dr = _disp(mine, L[d], N), _disp(ref, L[d], N)
        rms = np.sqrt(np.mean(dr ** 2))
        assert 0.005 < rms < 0.5, rms
        assert np.max(np.abs(dm - dr)) < 1e-4 * rms, d
        vrms = np.sqrt(np.mean(ov[:, d] ** 2))
        assert np.max(np.abs(out["v"][:, d] - ov[:, d])) < 1e-4 * vrms, d
    assert np.all(out["rung"] == 0)


@pytest.mark.parametrize("fold", [1, 2])
def test_power_spectrum_matches_oracle(ctx, fold):
    """Shells, mean power and the reference's error estimate of a clustered 32^3 box."""
    N, box = 32, 50.0
    x, y, z, v, r = ics.clustered_box(N, nspheres=30, seed=5)
    b = ctx.box(len(x))
    b.upload(x, y, z, v, r)
    k, P, E = b.power_spectrum(N, box, fold)
    b.close()
    ok_, oP, oE, cnt = F.power_spectrum(x, y, z, N, fold, box)
    assert len(k) == len(oP) == max(N // 8, 64)
    assert np.allclose(k, ok_, rtol=1e-6)
    has = cnt > 1
    assert has.sum() > 10
    assert np.allclose(P[has], oP[has], rtol=2e-3, atol=1e-6 * oP.max())
    assert np.allclose(E[has], oE[has], rtol=2e-2, atol=1e-5 * oE.max())
    assert np.all(P[cnt == 0] == 0)


def test_power_spectrum_recovers_the_input_spectrum(ctx):
    """Zel'dovich ICs of 128^3 particles: below a quarter of the Nyquist wavenumber the measured
    mean |delta_k|^2 is N^6 D1^2 P(k) / V (unnormalised transform), shell by shell within the
    scatter of the shell's mode count, on average within 7%."""
    N, box = 128, 200.0
    k, P = _table(N, box, 0.5)
    b = ctx.box(N ** 3)
    r = b.initialize(N, box, k, P, twolpt=False, **COSMO)
    kc, Pm, _ = b.power_spectrum(N, box, 1)
    b.close()
    Pn, lkmin, dlk, _, _ = F.power_table(k, P, COSMO["hubble"], COSMO["sigma8"])
    kgrid = kc * box / (2 * np.pi)
    sel = (kgrid > 3) & (kgrid < N / 8) & (Pm > 0)
    expect = N ** 6 * r["D1"] ** 2 * F.interp_power(Pn, lkmin, dlk, kc[sel]) / box ** 3
    ratio = Pm[sel] / expect
    print("measured / expected power per shell:", np.round(ratio, 3))
    assert sel.sum() >= 10
    assert np.all(np.abs(ratio - 1) < 0.35)
    assert abs(np.mean(ratio) - 1) < 0.07


def test_initialize_rejects_bad_input(ctx):
    import cosmictiger_b200 as ct

    k, P = _table(16, 100.0, 0.25)
    b = ctx.box(1000)
    with pytest.raises(ct.GravityError):
        b.initialize(16, 100.0, k, P, **COSMO)  # 1000 particles is not 16^3
    b.close()
    b = ctx.box(16 ** 3)
    with pytest.raises(ct.GravityError):
        b.initialize(16, 100.0, k[:400], P[:400], **COSMO)  # table stops below the grid's k
    with pytest.raises(ct.GravityError):
        b.power_spectrum(15, 100.0)  # odd grid
    b.close()
