"""The Fourier oracle (oracle/fourier_oracle.py: the reference's IC generator and power
spectrum restated in numpy) against known answers and exact properties.  The CUDA path
(ct_initialize, ct_power_spectrum) is compared with this oracle in test_gpu_fourier.py."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import fourier_oracle as F  # noqa: E402

from cosmictiger_b200 import ics  # noqa: E402


def test_taus_known_answer():
    """GSL's taus generator, seed 1: the 10000th output is 2733957125 (the known-answer value of
    GSL's generator test for taus), here for a vector of identical generators."""
    g = F.Taus([1, 1, 1])
    for _ in range(10000):
        v = g.next()
    assert v.tolist() == [2733957125] * 3
    # seed 0 means seed 1; uniform_pos lies in (0, 1)
    a, b = F.Taus([0]), F.Taus([1])
    assert a.next()[0] == b.next()[0]
    u = F.Taus(np.arange(1000)).uniform_pos()
    assert np.all((u > 0) & (u < 1))


def test_cloud_kernel_partition_of_unity():
    """The six weights of any offset add to 1 (a uniform lattice has no density contrast)."""
    for t in np.linspace(0, 1, 17):
        w = sum(float(F.cloud_weight(t - q)) for q in range(F.CLOUD_MIN, F.CLOUD_MAX + 1))
        assert abs(w - 1.0) < 1e-12, t


@pytest.mark.parametrize("dims", [(0, 3), (2, 3), (0, 1), (1, 1)])
def test_modes_hermitian_kz0_plane(dims):
    """The kz = 0 plane takes the mirrored row's generator and the conjugate on its lower half,
    so Y(-kx, -ky, 0) = conj(Y(kx, ky, 0)) away from the Nyquist rows."""
    k, P = ics.power_law_table()
    Pn, lkmin, dlk, _, _ = F.power_table(k, P, 0.6732, 0.8607)
    N = 16
    Y = F.modes(N, 100.0, dims[0], dims[1], Pn, lkmin, dlk)
    for I0 in range(N):
        for I1 in range(N):
            if I0 == N // 2 or I1 == N // 2 or (I0 == 0 and I1 == 0):
                continue
            assert Y[I0, I1, 0] == np.conj(Y[(-I0) % N, (-I1) % N, 0])
    assert Y[0, 0, 0] == 0


def test_power_spectrum_of_lattice_and_plane_wave():
    """A particle per cell on the grid's lattice has no power; a lattice displaced by one
    sinusoidal mode along x puts its power in the shell of that wavenumber."""
    N = 16
    X, Y, Z, f = F.lattice(N)
    _, P, _, cnt = F.power_spectrum(X, Y, Z, N, 1, 100.0)
    assert np.abs(P).max() < 1e-12
    m = 3
    q = X.astype(np.float64) / 2 ** 32
    x = q + 0.01 / N * np.sin(2 * np.pi * m * q)
    Xd = np.floor((x % 1.0) * 2 ** 32).astype(np.uint64).astype(np.uint32)
    kc, P, _, cnt = F.power_spectrum(Xd, Y, Z, N, 1, 100.0)
    kb = F.kbins(N)
    peak = int(np.searchsorted(kb, m, side="right") - 1)
    assert int(np.argmax(P)) == peak and P[peak] > 1e3 * np.sort(P)[-2]


def test_displacements_first_order_dominate_with_a_cut_spectrum():
    """With power far below the grid scale, 2LPT changes the Zel'dovich displacements by a
    small correction of order D2 / D1."""
    N, box = 16, 100.0
    k, P = ics.power_law_table(kcut=0.25 * np.pi * N / box / 0.6732)
    a = F.initialize(N, box, 0.3111, 49.0, 0.6732, 0.8607, 1.0, k, P, False)
    b = F.initialize(N, box, 0.3111, 49.0, 0.6732, 0.8607, 1.0, k, P, True)
    L = F.lattice(N)[0].astype(np.int64)

    def disp(x):
        d = (x.astype(np.int64) - L + 2 ** 31) % 2 ** 32 - 2 ** 31
        return d / 2 ** 32 * N

    d1, d2 = disp(a[0]), disp(b[0])
    assert 0.005 < np.sqrt(np.mean(d1 ** 2)) < 0.5
    assert np.sqrt(np.mean((d2 - d1) ** 2)) < 0.05 * np.sqrt(np.mean(d1 ** 2))


def test_sigma8_normalisation_by_independent_quadrature():
    """The normalised table's top-hat variance at R = 8/h Mpc, integrated by adaptive quadrature
    over the same k range, is sigma8^2 (the restated Simpson sum, initialize.cpp:141-172)."""
    from scipy import integrate

    k, P = ics.power_law_table()
    h, s8 = 0.6732, 0.8607
    Pn, lkmin, dlk, lkmax, _ = F.power_table(k, P, h, s8)
    R = 8.0 / h

    def f(lk):
        kk = np.exp(lk)
        x = kk * R
        W = 3 * (np.sin(x) - x * np.cos(x)) / x ** 3
        return kk ** 3 * F.interp_power(Pn, lkmin, dlk, np.array([kk]))[0] * W * W / (2 * np.pi ** 2)

    val, _ = integrate.quad(f, lkmin + 1.5 * dlk, lkmax - 2.5 * dlk, limit=2000)
    assert abs(np.sqrt(val) / s8 - 1) < 1e-6


@pytest.mark.parametrize("kh", [0.3, 1.0, 2.0, 3.0])
def test_cloud_kernel_window_is_sinc6(kh):
    """The continuous Fourier transform of the quintic cloud kernel is sinc(k/2)^6, the window
    whose inverse (cloud_filter) the IC generator and the power spectrum apply."""
    from scipy import integrate

    ft, _ = integrate.quad(lambda x: F.cloud_weight(np.array([x]))[0] * np.cos(kh * x), -3, 3, limit=200)
    assert abs(ft - np.sinc(kh / 2 / np.pi) ** 6) < 1e-8
    assert abs(F.cloud_filter(np.array([kh]))[0] * ft - 1) < 1e-7


@pytest.mark.parametrize("a", [0.02, 0.1, 0.3, 0.6])
def test_growth_factor_fit_against_exact_growth(a):
    """The growth factor's fitting formula (cosmos_growth_factor, cosmology.cpp:80-87), normalised
    to a = 1, follows the exact flat-LCDM linear growth D(a) ~ H(a) int da / (a H)^3 within 0.3%."""
    from scipy import integrate

    om = 0.3111

    def exact(x):
        E = lambda u: np.sqrt(om / u ** 3 + 1 - om)  # noqa: E731
        val, _ = integrate.quad(lambda u: 1.0 / (u * E(u)) ** 3, 0, x)
        return 2.5 * om * E(x) * val

    fit = F.growth_factor(om, a) / F.growth_factor(om, 1.0)
    assert abs(fit / (exact(a) / exact(1.0)) - 1) < 3e-3


def _ref_functions():
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_functions.json")
    import json

    with open(path) as f:
        return json.load(f)


def test_cloud_kernel_and_window_match_the_reference():
    """cloud_weight and cloud_filter (cosmictiger/fft.hpp:116-134) against the reference's own
    functions at fixed points (tests/golden/ref_functions.json, written by oracle/func_probe.cu
    built from the reference's headers).  The reference evaluates the kernel in float: the
    restatement in double agrees to float rounding of terms up to 243/120; the window (double
    in both) agrees exactly."""
    d = _ref_functions()
    cw = np.array(d["cloud_weight"])
    assert len(cw) == 81
    assert np.abs(F.cloud_weight(cw[:, 0].astype(np.float32)) - cw[:, 1]).max() < 4e-6
    cf = np.array(d["cloud_filter"])
    assert len(cf) == 41
    assert np.array_equal(F.cloud_filter(cf[:, 0]), cf[:, 1])


def test_growth_factor_matches_the_reference():
    """cosmos_growth_factor (src/cosmology.cpp:80-87), compiled from the reference's source,
    against the restatement for three matter densities and five scale factors (a passed as
    float, as the reference's signature takes it)."""
    g = np.array(_ref_functions()["growth_factor"])
    assert len(g) == 15
    ours = np.array([F.growth_factor(om, float(np.float32(a))) for om, a, _ in g])
    assert np.abs(ours / g[:, 2] - 1).max() < 1e-7
