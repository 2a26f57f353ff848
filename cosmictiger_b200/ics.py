"""Seeded synthetic initial conditions for the gravity step.

The reference reads its initial conditions from a Boltzmann-code power spectrum through a
distributed FFT (src/initialize.cpp:261-355); none of that is on the gravity path.  The
workloads here are seeded stand-ins with the shapes the benchmark configurations name:

* ``zeldovich_lattice``: an n^3 lattice at i/n (src/initialize.cpp:650-700 places particles
  the same way) displaced by the Zel'dovich field of a Gaussian random field with
  P(k) ~ k^index, cut at the lattice Nyquist frequency, scaled to a given RMS displacement
  in units of the mean spacing; velocities = displacement * vel_factor.
* ``plummer_spheres``: particles in Plummer spheres with uniform centres and power-law
  masses.
* ``clustered_box``: the 70% lattice / 30% Plummer mix.

Positions are returned as 32-bit fixed point (the reference's fixed32, cosmictiger/fixed.hpp:36,
truncation of 2^32 x) in three uint32 arrays, velocities as float32 (N, 3) (AoS, as the
reference stores particles_v), rungs as int8 zeros.
"""
import numpy as np


def to_fixed32(x):
    """Wrap into [0, 1) and convert to fixed32 by truncation of 2^32 x."""
    x = np.asarray(x, dtype=np.float64)
    x = x - np.floor(x)
    i = np.floor(x * 4294967296.0)
    i = np.where(i >= 4294967296.0, 0.0, i)
    return i.astype(np.uint64).astype(np.uint32)


def fixed32_to_double(i):
    return i.astype(np.float64) * (1.0 / 4294967296.0)


def _displacement_field(n, index, rng):
    """Zel'dovich displacement (3, n, n, n) of a Gaussian field with P(k) ~ k^index, |k| < k_Nyquist."""
    k1 = np.fft.fftfreq(n, d=1.0 / n)
    kz = np.fft.rfftfreq(n, d=1.0 / n)
    KX, KY, KZ = np.meshgrid(k1, k1, kz, indexing="ij")
    k2 = KX ** 2 + KY ** 2 + KZ ** 2
    k = np.sqrt(k2)
    nyq = n / 2
    amp = np.zeros_like(k)
    mask = (k > 0) & (k < nyq)
    amp[mask] = k[mask] ** (index / 2.0)
    delta = (rng.standard_normal(k.shape) + 1j * rng.standard_normal(k.shape)) * amp
    out = np.empty((3, n, n, n), dtype=np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = np.where(k2 > 0, 1.0 / k2, 0.0)
    for d, K in enumerate((KX, KY, KZ)):
        psi_k = 1j * K * inv * delta
        out[d] = np.fft.irfftn(psi_k, s=(n, n, n), axes=(0, 1, 2))
    return out


def zeldovich_lattice(n, index=-2.0, rms_spacing=0.25, seed=1, vel_factor=1.0, count=None):
    """n^3 (or the first `count`) lattice particles with a Zel'dovich displacement."""
    rng = np.random.default_rng(seed)
    psi = _displacement_field(n, index, rng)
    rms = np.sqrt(np.mean(np.sum(psi ** 2, axis=0)))
    if rms > 0:
        psi *= (rms_spacing / n) / rms
    i, j, k = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    base = np.stack([i, j, k]).astype(np.float64) / n
    pos = (base + psi).reshape(3, -1)
    vel = (psi * vel_factor).reshape(3, -1).T.astype(np.float32)
    if count is not None:
        sel = rng.permutation(pos.shape[1])[:count]
        sel.sort()
        pos = pos[:, sel]
        vel = vel[sel]
    x, y, z = (to_fixed32(p) for p in pos)
    return x, y, z, np.ascontiguousarray(vel), np.zeros(len(x), np.int8)


def plummer_spheres(npart, nspheres=20000, mmin=1e2, mmax=1e5, slope=-1.9, a0=0.002, seed=2, rmax_a=10.0):
    """npart particles split over Plummer spheres with dN/dM ~ M^slope on [mmin, mmax],
    scale radius a0 (M/1e3)^(1/3), centres uniform in the unit box, truncated at rmax_a * a."""
    rng = np.random.default_rng(seed)
    nspheres = max(1, min(nspheres, npart))
    # power-law masses by inverse transform, then rescaled to the particle budget
    u = rng.random(nspheres)
    g = slope + 1.0
    m = (mmin ** g + u * (mmax ** g - mmin ** g)) ** (1.0 / g)
    counts = np.maximum(np.floor(m / m.sum() * npart).astype(np.int64), 1)
    while counts.sum() > npart:
        counts[np.argmax(counts)] -= counts.sum() - npart
    counts[np.argmax(counts)] += npart - counts.sum()
    centres = rng.random((nspheres, 3))
    a = a0 * (m / 1e3) ** (1.0 / 3.0)
    owner = np.repeat(np.arange(nspheres), counts)
    # Plummer radius inversion: r = a / sqrt(U^(-2/3) - 1), truncated
    cmax = (rmax_a ** 3) / (1.0 + rmax_a ** 2) ** 1.5
    U = rng.random(npart) * cmax
    r = a[owner] / np.sqrt(U ** (-2.0 / 3.0) - 1.0)
    v = rng.standard_normal((npart, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    pos = centres[owner] + v * r[:, None]
    x, y, z = (to_fixed32(p) for p in pos.T)
    vel = np.zeros((npart, 3), np.float32)
    return x, y, z, vel, np.zeros(npart, np.int8)


def clustered_box(n, lattice_frac=0.7, index=-1.5, rms_spacing=0.5, nspheres=20000, seed=3):
    """The 70% Zel'dovich lattice / 30% Plummer-sphere mix of n^3 particles."""
    N = n ** 3
    nl = int(round(lattice_frac * N))
    lx, ly, lz, lv, _ = zeldovich_lattice(n, index=index, rms_spacing=rms_spacing, seed=seed, count=nl)
    px, py, pz, pv, _ = plummer_spheres(N - nl, nspheres=nspheres, seed=seed + 1)
    x = np.concatenate([lx, px])
    y = np.concatenate([ly, py])
    z = np.concatenate([lz, pz])
    v = np.concatenate([lv, pv])
    return x, y, z, np.ascontiguousarray(v), np.zeros(N, np.int8)


def softening(n_total, hsoft_spacing):
    """Kernel support h of the reference: hsoft (in mean spacings) * self_phi * N^(-1/3)
    (src/options.cpp:165,217)."""
    return hsoft_spacing * (693.0 / 256.0) * n_total ** (-1.0 / 3.0)


def eta_default(eta=0.25):
    """eta / sqrt(self_phi) (src/options.cpp:166)."""
    return eta / np.sqrt(693.0 / 256.0)


def read_power_init(path):
    """The rows of a power.init file (two columns: k in h/Mpc, P in (Mpc/h)^3; the format
    read_power_spectrum reads, src/initialize.cpp:870-898), as float32 arrays."""
    rows = np.loadtxt(path, dtype=np.float64, ndmin=2)
    return rows[:, 0].astype(np.float32), rows[:, 1].astype(np.float32)


def power_law_table(kmin=1e-4, kmax=100.0, n=1024, index=-1.5, k0=0.1, bend=2.0, kcut=None):
    """A smooth synthetic power.init-style table (k in h/Mpc, log-uniform): P = k / (1 + (k/k0)^bend)^((1 - index)/bend),
    rising as k at large scales and falling as k^index at small ones; kcut multiplies it by
    exp(-(k/kcut)^2) (power far below the grid scale)."""
    k = np.exp(np.linspace(np.log(kmin), np.log(kmax), n))
    P = 2e4 * (k / k0) / (1.0 + (k / k0) ** bend) ** ((1.0 - index) / bend)
    if kcut is not None:
        P = P * np.exp(-(k / kcut) ** 2) + 1e-30
    return k.astype(np.float32), P.astype(np.float32)
