"""FMM operators of this project vs golden vectors recorded from the reference's own operators.

The golden files (tests/golden/ops_p{7,5}.npz, written by tests/golden/make_golden.py) hold
the outputs of the reference's generated operators (cosmictiger/fmm_kernels.hpp) compiled
from its sources.  Here the oracle's host build of this project's generated operators is
compared against them; the CUDA build of the same headers is compared against the oracle
by the GPU tests.
"""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def golden(order):
    return np.load(os.path.join(HERE, "golden", "ops_p%d.npz" % order))


def relmax(a, b):
    """Max-norm error relative to the max-norm of the expected vector."""
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-37))


@pytest.mark.parametrize("order", [7, 5])
def test_greens_m2l_l2l_p2m_m2m(oracle, order):
    g = golden(order)
    X, Xs = g["X"], g["Xs"]
    NE = order * order + 1
    NM = (order - 1) ** 2 + 1
    for i in range(len(X)):
        D = np.zeros(NE, np.float32)
        oracle.op("greens", order, X[i], D)
        assert relmax(D, g["greens"][i]) < 1e-5, ("greens", i)
        for phi in (0, 1):
            L = g["Lin"][i].copy()
            oracle.op("m2l", order, g["M"][i], g["greens"][i], L, flag=phi)
            assert relmax(L, g["m2l_phi%d" % phi][i]) < 1e-5, ("m2l", i, phi)
            L2 = np.zeros(5, np.float32)
            oracle.op("m2l2", order, g["M"][i], g["greens"][i], L2, flag=phi)
            assert relmax(L2[:4], g["m2l2_phi%d" % phi][i][:4]) < 1e-5, ("m2l2", i, phi)
            Lo = np.zeros(NE, np.float32)
            oracle.op("l2l", order, g["Lin"][i], Xs[i], Lo, flag=phi)
            assert relmax(Lo, g["l2l_phi%d" % phi][i]) < 1e-5, ("l2l", i, phi)
            Lp = np.zeros(5, np.float32)
            oracle.op("l2p", order, g["Lin"][i], Xs[i], Lp, flag=phi)
            assert relmax(Lp[:4], g["l2p_phi%d" % phi][i][:4]) < 1e-5, ("l2p", i, phi)
        M = np.zeros(NM, np.float32)
        oracle.op("p2m", order, Xs[i], M)
        assert relmax(M, g["p2m"][i]) < 1e-5, ("p2m", i)
        Mo = np.zeros(NM)
        oracle.op("m2m_d", order, g["Md"][i], Xs[i].astype(np.float64), Mo)
        # the reference's generated double code carries 10-digit literals
        assert relmax(Mo, g["m2m"][i]) < 1e-8, ("m2m", i)


@pytest.mark.parametrize("order", [7, 5])
def test_ewald_greens(oracle, order):
    """Ewald Green's function: matches the reference where its n=0-image recursion is
    accurate (|x| >= 0.02), and matches this operator's own FP64 evaluation everywhere."""
    g = golden(order)
    X = g["X"]
    NE = order * order + 1
    checked = 0
    for i in range(len(X)):
        D = np.zeros(NE, np.float32)
        oracle.op("ewald_greens", order, X[i], D)
        Dd = np.zeros(NE)
        oracle.op("ewald_greens_d", order, X[i].astype(np.float64), Dd)
        assert relmax(D.astype(np.float64), Dd) < 3e-6, ("fp32 vs fp64", i)
        if np.linalg.norm(X[i]) >= 0.02:
            assert relmax(D, g["ewald"][i]) < 5e-6, ("vs reference", i)
            checked += 1
    assert checked >= len(X) // 4


@pytest.mark.parametrize("order", [7, 5])
def test_ewald_tables(oracle, order):
    g = golden(order)
    NE = order * order + 1
    nfull = order * (order + 1) * (order + 2) // 6
    real = np.zeros((178, 3), np.float32)
    four = np.zeros((92, 3), np.float32)
    fexp = np.zeros((92, NE), np.float32)
    d0 = np.zeros(nfull, np.float32)
    oracle.op("ewald_tables", order, real, four, fexp, d0)
    assert set(map(tuple, real)) == set(map(tuple, g["ewald_real"]))
    # the images within 2.3 box lengths of the unit cell lead the table (the kick's Green's
    # function reads only those), each part by |n|^2 descending as the reference orders them
    cell = np.sqrt((np.maximum(np.abs(real) - 0.5, 0.0) ** 2).sum(1))
    ng = 116
    assert (cell[:ng] < 2.3).all() and (cell[ng:] >= 2.3).all()
    for part in (real[:ng], real[ng:]):
        n2 = (part ** 2).sum(1)
        assert (np.diff(n2) <= 0).all()
    assert set(map(tuple, four)) == set(map(tuple, g["ewald_four"]))
    # one vector of each +h/-h pair first (first nonzero component positive), then the negatives
    half = four[:46]
    assert set(map(tuple, -half)) == set(map(tuple, four[46:]))
    first = np.array([v[np.nonzero(v)[0][0]] for v in half])
    assert (first > 0).all()
    ref = {tuple(g["ewald_four"][i]): g["ewald_four_exp"][i] for i in range(92)}
    for i in range(92):
        assert relmax(fexp[i], ref[tuple(four[i])]) < 1e-6
    # D0 limit tensor: this project stores +limit in its own full order; the reference stores -limit
    exps_mine = full_exponents(order)
    mine = {tuple(e): d0[k] for k, e in enumerate(exps_mine)}
    for k, e in enumerate(g["ewald_D0_exps"]):
        assert abs(mine[tuple(e)] + g["ewald_D0_ref_negated"][k]) <= 1e-6 * abs(g["ewald_D0_ref_negated"][k]) + 1e-37


def full_exponents(P):
    out = []
    for N in range(P):
        for a in range(N, -1, -1):
            for b in range(N - a, -1, -1):
                out.append((a, b, N - a - b))
    return out


@pytest.mark.parametrize("order", [7, 5])
def test_generated_operator_headers_are_current(order):
    """The committed operator headers (csrc/fmm_p{7,5}.h, compiled into both the library and the
    oracle) are exactly what csrc/gen_fmm.py generates, so an edit of the generator cannot
    leave the two behind each other."""
    import importlib.util

    csrc = os.path.join(os.path.dirname(HERE), "cosmictiger_b200", "csrc")
    spec = importlib.util.spec_from_file_location("gen_fmm", os.path.join(csrc, "gen_fmm.py"))
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    with open(os.path.join(csrc, "fmm_p%d.h" % order)) as f:
        assert f.read() == gen.gen_header(order)


@pytest.mark.parametrize("order", [7, 5])
def test_operator_goldens_equal_a_fresh_recording(order):
    """Where the reference's operators are built (oracle/_ref/libctref_p{7,5}.so, from
    `make -C oracle ref`), recording the golden vectors again gives the committed files exactly."""
    import importlib.util

    root = os.path.dirname(HERE)
    if not os.path.exists(os.path.join(root, "oracle", "_ref", "libctref_p%d.so" % order)):
        pytest.skip("reference operators not built")
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "golden", "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    fresh = mg.vectors(order)
    g = golden(order)
    assert sorted(fresh) == sorted(g.files)
    for k in g.files:
        a, b = fresh[k], g[k]
        if k.startswith("l2p_"):
            # the reference's L2P writes four of its five outputs (potential and force); the
            # fifth is whatever the harness's stack held, so only the four are compared, here
            # as in the parity test above
            a, b = a[:, :4], b[:, :4]
        assert np.array_equal(a, b), k
