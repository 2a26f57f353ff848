"""Lightcone capture in the drift (src/drift.cu:36-154) and its HEALPix pixels
(src/healpix.cu:55-171): properties of the CPU oracle's restatement.  The CUDA path is checked
against the reference's own drift kernel and against this oracle in test_gpu_lightcone.py."""
import numpy as np
import pytest

from cosmictiger_b200 import ics


def _unit_vectors(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.standard_normal((n, 3))
    return v / np.linalg.norm(v, axis=1)[:, None]


def test_healpix_known_pixels(oracle):
    """nside 1: the 12 base faces, 0-3 north, 4-7 equatorial (face 4 centred on phi = 0), 8-11 south."""
    hp = oracle.healpix_nest
    assert hp(1, 1, 0, 0) == 4
    assert hp(1, 0, 1, 0) == 5
    assert hp(1, -1, 0, 0) == 6
    assert hp(1, 0, -1, 0) == 7
    assert hp(1, 0, 0, 1) == 0
    assert hp(1, 0, 0, -1) == 8
    s = np.sqrt(0.5)
    # mid-latitude north/south between the faces: phi = pi/4 lies inside face 0 / 8
    assert hp(1, s * 0.3, s * 0.3, 0.95) == 0
    assert hp(1, s * 0.3, s * 0.3, -0.95) == 8
    # scale invariance: only the direction matters
    assert hp(64, 0.3, -0.2, 0.5) == hp(64, 3.0, -2.0, 5.0)


def test_healpix_nested_hierarchy(oracle):
    """A nested pixel at nside 2k lies inside pixel p // 4 at nside k."""
    for x, y, z in _unit_vectors(400, 5):
        p = oracle.healpix_nest(8192, x, y, z)
        k = 4096
        while k >= 1:
            q = oracle.healpix_nest(k, x, y, z)
            assert q == p // 4, (x, y, z, k)
            p = q
            k //= 2


def test_healpix_equal_area(oracle):
    """Isotropic directions fill the 12 nside^2 pixels evenly (HEALPix pixels have equal area)."""
    nside = 4
    npix = 12 * nside * nside
    v = _unit_vectors(60000, 7)
    counts = np.bincount([oracle.healpix_nest(nside, *u) for u in v], minlength=npix)
    assert counts.shape == (npix,) and counts.min() > 0
    expect = len(v) / npix
    chi2 = float(np.sum((counts - expect) ** 2 / expect))
    # chi-square with 191 degrees of freedom: mean 191, sd 19.5
    assert chi2 < 191 + 6 * 19.5, chi2


def _state(n=12, seed=9, vscale=1.0):
    x, y, z, v, r = ics.clustered_box(n, nspheres=8, seed=seed)
    v = (v * vscale).astype(np.float32)
    rng = np.random.default_rng(seed)
    r = rng.integers(0, 3, len(x)).astype(np.int8)
    return x, y, z, v, r


@pytest.mark.parametrize("tau0,dt,tau_max", [(0.45, 0.02, 1.3), (0.05, 0.1, 1.0), (1.2, 0.03, 2.1)])
def test_lightcone_oracle_crossings_on_the_cone(oracle, tau0, dt, tau_max):
    """Each entry lies inside the unit sphere at a distance r with tau0 + t + r = k tau_max for a
    crossing time t within the drift (0 <= t <= dt, up to rounding), and its pixel is the
    pixel of its position."""
    x, y, z, v, r = _state(vscale=10.0)
    ent = oracle.drift_lc(x.copy(), y.copy(), z.copy(), v.copy(), r, 1, 1.0, dt, tau0, tau0 + dt, tau_max, 16)
    assert len(ent) > 100
    q = np.stack([ent["x"], ent["y"], ent["z"]], axis=1).astype(np.float64) / 2 ** 31
    rr = np.linalg.norm(q, axis=1)
    assert np.all(rr <= 1.0 + 1e-9)
    k = np.floor((tau0 + dt + rr) / tau_max + 1e-9)
    lag = k * tau_max - tau0 - rr  # crossing time t
    assert np.all(lag > -1e-6) and np.all(lag < dt + 1e-6), (lag.min(), lag.max())
    pix = np.array([oracle.healpix_nest(16, *p) for p in q])
    # positions are truncated to 2^-31: a pixel can only differ right at a boundary
    assert np.mean(pix == ent["pix"]) > 0.999


def test_lightcone_oracle_same_drift_as_plain(oracle):
    """Capturing the light cone does not change the drift: positions and (dragged) velocities
    equal the plain drift's."""
    x, y, z, v, r = _state()
    a = [q.copy() for q in (x, y, z, v)]
    b = [q.copy() for q in (x, y, z, v)]
    oracle.drift(*a, r, 2, 0.8, 0.04, drag=0.3)
    ent = oracle.drift_lc(*b, r, 2, 0.8, 0.04, 0.5, 0.54, 1.4, 8, drag=0.3)
    assert len(ent) > 0
    for p, q in zip(a, b):
        assert np.array_equal(p, q)
    # no capture when tau_max - tau1 >= 1 (src/drift.cu:38)
    c = [q.copy() for q in (x, y, z, v)]
    assert len(oracle.drift_lc(*c, r, 2, 0.8, 0.04, 0.1, 0.14, 1.2, 8)) == 0


def _pix2vec_nest(nside, p):
    """Centre of nested pixel p (the inverse construction of Gorski et al. 2005): face and
    in-face (ix, iy) from the bits, ring and longitude index from the face's base ring and
    longitude, then z and phi of the ring position."""
    jrll = [2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4]
    jpll = [1, 3, 5, 7, 0, 2, 4, 6, 1, 3, 5, 7]
    face, ipf = divmod(p, nside * nside)
    ix = iy = 0
    for b in range(16):
        ix |= ((ipf >> (2 * b)) & 1) << b
        iy |= ((ipf >> (2 * b + 1)) & 1) << b
    jr = jrll[face] * nside - ix - iy - 1
    if jr < nside:
        nr, z, kshift = jr, 1 - jr * jr / (3.0 * nside * nside), 0
    elif jr > 3 * nside:
        nr = 4 * nside - jr
        z, kshift = -1 + nr * nr / (3.0 * nside * nside), 0
    else:
        nr, z, kshift = nside, (2 * nside - jr) * 2.0 / (3.0 * nside), (jr - nside) & 1
    jp = (jpll[face] * nr + ix - iy + 1 + kshift) // 2
    if jp > 4 * nside:
        jp -= 4 * nside
    if jp < 1:
        jp += 4 * nside
    phi = (jp - (kshift + 1) * 0.5) * (np.pi / 2 / nr)
    st = np.sqrt(max(0.0, 1 - z * z))
    return st * np.cos(phi), st * np.sin(phi), z


@pytest.mark.parametrize("nside", [1, 2, 4, 8, 16])
def test_healpix_pixel_centres_round_trip(oracle, nside):
    """Every pixel's centre, from the independent inverse construction, lies in that pixel."""
    for p in range(12 * nside * nside):
        assert oracle.healpix_nest(nside, *_pix2vec_nest(nside, p)) == p, (nside, p)
