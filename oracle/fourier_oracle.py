"""Test infrastructure only: a numpy restatement of the reference's initial-condition generator
(src/initialize.cpp:261-355,436-898) and matter power spectrum (src/power.cpp:33-77,
src/power.cu:32-85, src/fft.cpp:172-360), the checker of the CUDA path (ct_initialize,
ct_power_spectrum).  Transforms are numpy's FFTs in double precision; the random field uses the
same per-row generator (GSL's "taus", L'Ecuyer 1996, restated below), so that both sides draw
the same numbers.  Pinned against the reference's own initialize() and power_spectrum_compute()
run on the host (oracle/ic_probe.cpp; fixtures tests/golden/ref_ic.npz, tests/test_ic_reference.py).
Only tests/ import this module.
"""
import numpy as np

CLOUD_MIN, CLOUD_MAX = -2, 3
M32 = np.uint64(0xFFFFFFFF)


# ---------------------------------------------------------------- GSL "taus", one per row
class Taus:
    """Vectorised taus generators (one per seed), as gsl_rng_taus seeds and steps them."""

    def __init__(self, seeds):
        s = np.asarray(seeds, np.uint64) & M32
        s = np.where(s == 0, np.uint64(1), s)
        self.s1 = (np.uint64(69069) * s) & M32
        self.s2 = (np.uint64(69069) * self.s1) & M32
        self.s3 = (np.uint64(69069) * self.s2) & M32
        for _ in range(6):
            self.next()

    def next(self):
        s1, s2, s3 = self.s1, self.s2, self.s3
        s1 = (((s1 & np.uint64(4294967294)) << np.uint64(12)) & M32) ^ ((((s1 << np.uint64(13)) & M32) ^ s1) >> np.uint64(19))
        s2 = (((s2 & np.uint64(4294967288)) << np.uint64(4)) & M32) ^ ((((s2 << np.uint64(2)) & M32) ^ s2) >> np.uint64(25))
        s3 = (((s3 & np.uint64(4294967280)) << np.uint64(17)) & M32) ^ ((((s3 << np.uint64(3)) & M32) ^ s3) >> np.uint64(11))
        self.s1, self.s2, self.s3 = s1, s2, s3
        return s1 ^ s2 ^ s3

    def uniform_pos(self):
        v = self.next()
        while np.any(v == 0):
            # only the generators that returned 0 draw again
            z = v == 0
            w = self.next()
            v = np.where(z, w, v)
        return v.astype(np.float64) / 4294967296.0


# ---------------------------------------------------------------- cloud kernel
def cloud_weight(x):
    x = np.abs(np.asarray(x, np.float64))
    x2, x3 = x * x, x ** 3
    x4, x5 = x2 * x2, x3 * x2
    w = np.where(x < 1, (33 - 30 * x2 + 15 * x4 - 5 * x5) / 60,
                 np.where(x < 2, (51 + 75 * x - 210 * x2 + 150 * x3 - 45 * x4 + 5 * x5) / 120,
                          (243 - 405 * x + 270 * x2 - 90 * x3 + 15 * x4 - x5) / 120))
    return np.where(x > 3, 0.0, w)


def sinc(x):
    x = np.asarray(x, np.float64)
    out = np.ones_like(x)
    nz = x != 0
    out[nz] = np.sin(x[nz]) / x[nz]
    return out


def cloud_filter(kh):
    s = sinc(0.5 * np.asarray(kh, np.float64))
    return 1.0 / (s * s * s) ** 2


# ---------------------------------------------------------------- power table
def power_table(table_k, table_p, hubble, sigma8):
    """(P in Mpc^3, logkmin, dlogk, logkmax, norm) as read_power_spectrum + normalize take the
    table (initialize.cpp:141-172,853-880), in double."""
    k = np.asarray(table_k, np.float64) * hubble
    P = np.asarray(table_p, np.float64) / hubble ** 3
    logkmin, logkmax = np.log(k.min()), np.log(k.max())
    dlogk = (logkmax - logkmin) / (len(P) - 1)

    def interp(kk):
        return interp_power(P, logkmin, dlogk, kk)

    R = 8.0 / hubble
    c0 = 9.0 / (2 * np.pi ** 2) / R ** 6

    def integrand(x):
        kk = np.exp(x)
        t = np.sin(kk * R) - kk * R * np.cos(kk * R)
        return c0 * interp(kk) * t * t * kk ** -3

    N = 8192
    lmax = logkmax - 2.5 * dlogk
    lmin = logkmin + 1.5 * dlogk
    d = (lmax - lmin) / N
    xs = lmin + d * np.arange(N + 1)
    w = np.where(np.arange(N + 1) % 2 == 1, 4.0, 2.0)
    w[0] = w[-1] = 1.0
    s = np.sum(w * integrand(xs)) * d / 3.0
    norm = sigma8 ** 2 / s
    return P * norm, logkmin, dlogk, logkmax, norm


def interp_power(P, logkmin, dlogk, k):
    k0 = (np.log(np.asarray(k, np.float64)) - logkmin) / dlogk
    i0 = np.clip(k0.astype(np.int64) - 1, 0, len(P) - 4)
    x = k0 - (i0 + 1)
    y0, y1, y2, y3 = (np.log(P[i0 + q]) for q in range(4))
    k1 = (y2 - y0) * 0.5
    k2 = (y3 - y1) * 0.5
    c = -2 * k1 - k2 - 3 * y1 + 3 * y2
    d = k1 + k2 + 2 * y1 - 2 * y2
    return np.exp(y1 + k1 * x + c * x * x + d * x ** 3)


# ---------------------------------------------------------------- fields
def modes(N, box, dim1, dim2, P, logkmin, dlogk):
    """The half-complex field Y[I0, I1, I2] of twolpt_generate (initialize.cpp:436-540)."""
    NZ = N // 2 + 1
    I0, I1 = np.meshgrid(np.arange(N), np.arange(N), indexing="ij")
    I0, I1 = I0.ravel(), I1.ravel()
    sgnd = lambda I: np.where(I < N // 2, I, I - N)
    i, j = sgnd(I0), sgnd(I1)
    kf = 2 * np.pi / box
    kx, ky = kf * i, kf * j
    factor = box ** -1.5 * N ** 3
    Y = np.zeros((N * N, NZ), np.complex128)

    def value(kz, x, y):
        k2 = kx * kx + ky * ky + kz * kz
        K0 = np.sqrt(k2)
        rn = np.exp(1j * 2 * np.pi * y) * np.sqrt(-np.log(np.abs(x)))
        Kc = [-1j * kx, -1j * ky, -1j * kz, np.ones_like(kx)]
        with np.errstate(divide="ignore", invalid="ignore"):
            return rn * np.sqrt(interp_power(P, logkmin, dlogk, np.where(K0 > 0, K0, 1.0))) * factor * Kc[dim1] * Kc[dim2] / k2

    def filt(kz):
        return cloud_filter(kx * box / N) * cloud_filter(ky * box / N) * cloud_filter(np.full_like(kx, kz) * box / N)

    g = Taus(((I0.astype(np.int64) * N + I1) * 1234 + 42) & 0xFFFFFFFF)
    for _ in range(8):
        g.uniform_pos()
    for I2 in range(1, NZ):
        k = I2 if I2 < N // 2 else I2 - N
        x = g.uniform_pos()
        y = g.uniform_pos()
        Y[:, I2] = value(kf * k, x, y) * filt(kf * k)
    J0 = np.where(I0 > N // 2, N - I0, I0)
    J1 = np.where(I1 > N // 2, N - I1, I1)
    g = Taus(((J0.astype(np.int64) * N + J1) * 1234 + 42) & 0xFFFFFFFF)
    for _ in range(8):
        g.uniform_pos()
    x = g.uniform_pos()
    y = g.uniform_pos()
    v = value(0.0, x, y)
    sgn = (-1.0 if dim1 != 3 else 1.0) * (-1.0 if dim2 != 3 else 1.0)
    flip = (I0 > N // 2) | ((I0 == 0) & (I1 > N // 2))
    v = np.where(flip, np.conj(v) * sgn, v)
    v = np.where(i * i + j * j > 0, v, 0.0)
    Y[:, 0] = v * filt(0.0)
    return Y.reshape(N, N, NZ)


def inverse(Y, N):
    """The reference's normalised inverse transform (1/N per axis)."""
    return np.fft.irfftn(Y, s=(N, N, N), axes=(0, 1, 2))


def lattice(N):
    I = np.arange(N, dtype=np.float64) / N
    f = np.floor(I * 4294967296.0).astype(np.uint64).astype(np.uint32)
    X = np.broadcast_to(f[:, None, None], (N, N, N)).ravel().copy()
    Yc = np.broadcast_to(f[None, :, None], (N, N, N)).ravel().copy()
    Z = np.broadcast_to(f[None, None, :], (N, N, N)).ravel().copy()
    return X, Yc, Z, f


def interpolate_at_lattice(R, N, f):
    """Cloud-kernel interpolation of R at the lattice points (zeldovich_end's sum), by axes."""
    x0 = f.astype(np.float64) / 4294967296.0
    i1 = (x0 * N).astype(np.int64)
    t = x0 * N - i1
    out = R
    for axis in range(3):
        acc = np.zeros_like(out)
        for jj in range(CLOUD_MIN, CLOUD_MAX + 1):
            w = cloud_weight((-jj + t).astype(np.float32))
            idx = (i1 + jj) % N
            sl = np.take(out, idx, axis=axis)
            shape = [1, 1, 1]
            shape[axis] = N
            acc += sl * w.reshape(shape)
        out = acc
    return out.ravel()


def growth_factor(omega_m, a):
    ol = 1.0 - omega_m
    a3 = a ** 3
    den = 1.0 / (omega_m + a3 * ol)
    Om, Ol = omega_m * den, a3 * ol * den
    return a * 2.5 * Om / (Om ** (4.0 / 7.0) - Ol + (1.0 + 0.5 * Om) * (1.0 + 0.014285714 * Ol))


def initialize(N, box, omega_m, z0, hubble, sigma8, H0, table_k, table_p, twolpt):
    """Positions (uint32), velocities (float64, (n, 3)) and the factors of initialize()."""
    P, logkmin, dlogk, _, norm = power_table(table_k, table_p, hubble, sigma8)
    a0 = 1.0 / (z0 + 1.0)
    D1 = growth_factor(omega_m, a0) / growth_factor(omega_m, 1.0)
    Om = omega_m / (omega_m + a0 ** 3 * (1 - omega_m))
    H = H0 * np.sqrt(omega_m / a0 ** 3 + 1 - omega_m)
    prefac1 = Om ** (5 / 9) * H * a0 * a0
    D2 = -3 * D1 * D1 / 7
    prefac2 = 2 * Om ** (6 / 11) * H * a0 * a0
    X, Yc, Z, f = lattice(N)
    pos = [X.astype(np.float64) / 4294967296.0, Yc.astype(np.float64) / 4294967296.0, Z.astype(np.float64) / 4294967296.0]
    vel = np.zeros((N ** 3, 3))

    def displace(R, dim, D, pre):
        dx = interpolate_at_lattice(R, N, f) * (-D / box)
        x = pos[dim] + dx
        pos[dim] = np.where(x >= 1.0, x - 1.0, np.where(x < 0.0, x + 1.0, x))
        vel[:, dim] += pre * dx

    for dim in range(3):
        displace(inverse(modes(N, box, dim, 3, P, logkmin, dlogk), N), dim, D1, prefac1)
    if twolpt:
        delta2 = np.zeros((N, N, N))
        part = None
        pairs = [(1, 1), (2, 2), (0, 0), (2, 2), (0, 0), (1, 1), (0, 1), (0, 2), (1, 2)]
        for ph, (d1, d2) in enumerate(pairs):
            r = inverse(modes(N, box, d1, d2, P, logkmin, dlogk), N)
            if ph > 6:
                delta2 -= r * r
            elif ph % 2 == 0:
                part = r
            else:
                delta2 += part * r
        S = np.fft.rfftn(delta2)
        I = np.arange(N)
        sg = np.where(I < N // 2, I, I - N)
        kf = 2 * np.pi / box
        kx = (kf * sg)[:, None, None]
        ky = (kf * sg)[None, :, None]
        kz = (kf * sg[: N // 2 + 1])[None, None, :]
        k2 = kx * kx + ky * ky + kz * kz
        filt = cloud_filter(kx * box / N) * cloud_filter(ky * box / N) * cloud_filter(kz * box / N)
        for dim, K in enumerate((kx, ky, kz)):
            with np.errstate(divide="ignore", invalid="ignore"):
                Yd = np.where(k2 > 0, -1j * K * S / k2 * filt, 0.0)
            displace(inverse(Yd, N), dim, -D2, prefac2)
    xs = [np.floor(p * 4294967296.0).astype(np.uint64).astype(np.uint32) for p in pos]
    return xs[0], xs[1], xs[2], vel, {"D1": D1, "D2": D2, "prefac1": prefac1, "prefac2": prefac2, "norm": norm}


# ---------------------------------------------------------------- power spectrum
def kbins(N):
    Ns = max(N / 8.0, 64.0)
    lmin, lmax = np.log(0.999999), np.log(N / 2.0)
    dl = (lmax - lmin) / Ns
    return np.array([np.exp(lmin + dl * i) for i in range(int(Ns) + 1)], np.float32)


def density(x, y, z, N, fold):
    rho = np.full(N ** 3, -1.0)
    pos = [np.fmod(np.float32(fold) * (q.astype(np.float32) * np.float32(2.0 ** -32)), np.float32(1.0)) for q in (x, y, z)]
    cells = [(p * np.float32(N)).astype(np.int64) for p in pos]
    frac = [p * np.float32(N) - c.astype(np.float32) for p, c in zip(pos, cells)]
    w = [[cloud_weight((fr - np.float32(q)).astype(np.float32)) for q in range(CLOUD_MIN, CLOUD_MAX + 1)] for fr in frac]
    for a in range(6):
        ia = (cells[0] + a + CLOUD_MIN) % N
        for b in range(6):
            ib = (cells[1] + b + CLOUD_MIN) % N
            wab = w[0][a] * w[1][b]
            for c in range(6):
                ic = (cells[2] + c + CLOUD_MIN) % N
                np.add.at(rho, (ia * N + ib) * N + ic, wab * w[2][c])
    return rho.reshape(N, N, N)


def power_spectrum(x, y, z, N, fold, box):
    """(k, P, Perr) of fft3d_power_spectrum with power_spectrum_compute / compute2."""
    kb = kbins(N)
    nb = len(kb) - 1
    Y = np.fft.rfftn(density(x, y, z, N, fold))
    I = np.arange(N)
    sg = np.where(I < N // 2, I, I - N).astype(np.float64)
    i = sg[:, None, None]
    j = sg[None, :, None]
    k = sg[: N // 2 + 1][None, None, :]
    c1 = cloud_filter(2 * np.pi * i / N) * cloud_filter(2 * np.pi * j / N) * cloud_filter(2 * np.pi * k / N)
    Y = Y * c1
    kk = np.sqrt(i * i + j * j + k * k)
    kk = np.broadcast_to(kk, Y.shape).ravel()
    ok = (kk > 0) & (kk < kb[-1])
    b = np.searchsorted(kb.astype(np.float64), kk, side="right") - 1
    pw = (np.abs(Y) ** 2).ravel()
    cnt = np.bincount(b[ok], minlength=nb)[:nb].astype(np.float64)
    psum = np.bincount(b[ok], weights=pw[ok], minlength=nb)[:nb]
    with np.errstate(divide="ignore", invalid="ignore"):
        P = np.where(cnt > 0, psum / cnt, 0.0)
    c2 = (1.0 / (sinc(np.pi * i / N) * sinc(np.pi * j / N) * sinc(np.pi * k / N))) ** 3
    pw2 = (np.abs(Y * c2) ** 2).ravel()
    dev = np.bincount(b[ok], weights=(pw2[ok] - P[b[ok]]) ** 2, minlength=nb)[:nb]
    with np.errstate(divide="ignore", invalid="ignore"):
        err = np.where(cnt > 1, np.sqrt(dev) / np.sqrt(cnt - 1) / np.sqrt(cnt), 0.0)
    P = np.where(cnt == 1, 0.0, P)
    kc = np.sqrt(kb[:-1].astype(np.float64) * kb[1:]) * (2 * np.pi / box) * fold
    return kc, P, err, cnt
