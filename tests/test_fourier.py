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
