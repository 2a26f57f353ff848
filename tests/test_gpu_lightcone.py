"""The drift's lightcone capture on the device against the reference's OWN drift kernel
(src/drift.cu cuda_drift_kernel with do_lc, compiled from its sources for sm_100a:
oracle/_ref/libctref_gpu.so) and against the CPU oracle's restatement."""
import numpy as np
import pytest

from cosmictiger_b200 import ics

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import cosmictiger_b200 as ct

    c = ct.Context(order=7)
    yield c
    c.close()


@pytest.fixture(scope="module")
def ref():
    from tests import reference_gpu_lib

    if not reference_gpu_lib.available():
        pytest.fail("oracle/_ref/libctref_gpu.so is not built (make -C oracle refgpu)")
    return reference_gpu_lib.ReferenceGPU()


def _state(n=24, seed=21, vscale=1.0, nrung=3):
    x, y, z, v, r = ics.clustered_box(n, nspheres=12, seed=seed)
    rng = np.random.default_rng(seed)
    return x, y, z, (v * vscale).astype(np.float32), rng.integers(0, nrung, len(x)).astype(np.int8)


def _sorted(e):
    return np.sort(e, order=["pix", "x", "y", "z", "vx", "vy", "vz"])


def _drift(ctx, st, level, a, dt, tau0, tau1, tau_max, nside, drag=0.0, reserve=None):
    x, y, z, v, r = st
    box = ctx.box(len(x))
    box.upload(x, y, z, v, r)
    if reserve is not None:
        box.lightcone_reserve(reserve)
    n = box.drift_lightcone(level, a, dt, tau0, tau1, tau_max, nside, drag)
    ent = box.lightcone()
    out = box.download()
    box.close()
    assert n == len(ent)
    return out, ent


CASES = [
    # level, a, dt, tau0, tau_max, nside, vscale, create_glass
    (0, 1.0, 0.02, 0.45, 1.3, 16, 1.0, False),
    (1, 0.7, 0.05, 0.05, 1.0, 1, 10.0, False),
    (2, 0.9, 0.03, 1.2, 2.1, 8192, 5.0, True),
    (0, 0.5, 0.1, 0.3, 1.25, 256, 20.0, True),
]


@pytest.mark.parametrize("level,a,dt,tau0,tau_max,nside,vscale,glass", CASES)
def test_lightcone_matches_reference_cuda_drift(ctx, ref, level, a, dt, tau0, tau_max, nside, vscale, glass):
    """Same entries (as a set: the order within a drift is the kernel's), positions and
    velocities as the reference's drift with its lightcone on, bit for bit."""
    st = _state(vscale=vscale)
    tau1 = tau0 + dt
    drag = np.pi if glass else 0.0  # the reference's drift takes pi with create_glass (drift.cu:183)
    out, ent = _drift(ctx, st, level, a, dt, tau0, tau1, tau_max, nside, drag)
    rx, ry, rz, rv, rent = ref.drift_lc(*st, level, a, dt, tau0, tau1, tau_max, nside, create_glass=glass)
    print("lightcone vs reference CUDA drift: %d entries, %d particles of rung %d" % (len(rent), int(np.sum(st[4] == level)), level))
    assert len(rent) > 50
    assert len(ent) == len(rent)
    a_, b_ = _sorted(ent), _sorted(rent)
    for f in ("x", "y", "z", "pix"):
        assert np.array_equal(a_[f], b_[f]), f
    for f in ("vx", "vy", "vz"):
        assert np.array_equal(a_[f].view(np.uint32), b_[f].view(np.uint32)), f
    assert np.array_equal(out["x"], rx) and np.array_equal(out["y"], ry) and np.array_equal(out["z"], rz)
    assert np.array_equal(out["v"].view(np.uint32), rv.view(np.uint32))


def test_lightcone_matches_oracle(ctx, oracle):
    """The CPU restatement (no FMA contraction) agrees up to the last bits of FP64 rounding:
    same count, positions within 2 units of 2^-31, pixels equal but at pixel boundaries."""
    st = _state(vscale=10.0)
    out, ent = _drift(ctx, st, 1, 0.8, 0.05, 0.3, 0.35, 1.2, 64)
    x, y, z, v, r = (q.copy() for q in st)
    oent = oracle.drift_lc(x, y, z, v, r, 1, 0.8, 0.05, 0.3, 0.35, 1.2, 64)
    assert len(ent) == len(oent) and len(ent) > 50
    a_, b_ = _sorted(ent), _sorted(oent)
    for f in ("x", "y", "z"):
        assert np.max(np.abs(a_[f].astype(np.int64) - b_[f].astype(np.int64))) <= 2, f
    assert np.mean(a_["pix"] == b_["pix"]) > 0.999
    assert np.array_equal(out["x"], x) and np.array_equal(out["y"], y) and np.array_equal(out["z"], z)


def test_lightcone_buffer_growth_drops_nothing(ctx):
    """An entry buffer far too small grows to the candidates' need before any entry is written;
    entries and positions equal a run with room to spare, and entries accumulate over drifts."""
    st = _state(vscale=10.0)
    args = (0, 1.0, 0.05, 0.4, 0.45, 1.3, 32)
    o1, e1 = _drift(ctx, st, *args, reserve=4)
    o2, e2 = _drift(ctx, st, *args, reserve=1 << 20)
    assert len(e1) == len(e2) > 100
    assert np.array_equal(_sorted(e1), _sorted(e2))
    for f in ("x", "y", "z", "v"):
        assert np.array_equal(o1[f], o2[f]), f
    # two drifts append; download without clearing keeps them
    x, y, z, v, r = st
    box = ctx.box(len(x))
    box.upload(x, y, z, v, r)
    n1 = box.drift_lightcone(0, 1.0, 0.05, 0.4, 0.45, 1.3, 32)
    n2 = box.drift_lightcone(0, 1.0, 0.05, 0.45, 0.5, 1.3, 32)
    kept = box.lightcone(clear=False)
    assert len(kept) == n1 + n2 and len(box.lightcone()) == n1 + n2 and len(box.lightcone()) == 0
    box.close()


def test_lightcone_drift_equals_plain_drift(ctx):
    """With the capture on, particles move exactly as ct_drift moves them; with tau_max - tau1 >= 1
    nothing is captured."""
    st = _state()
    x, y, z, v, r = st
    box = ctx.box(len(x))
    box.upload(x, y, z, v, r)
    box.drift(1, 0.8, 0.04, 0.3)
    plain = box.download()
    box.close()
    out, ent = _drift(ctx, st, 1, 0.8, 0.04, 0.5, 0.54, 1.4, 8, drag=0.3)
    assert len(ent) > 0
    for f in ("x", "y", "z", "v"):
        assert np.array_equal(out[f], plain[f]), f
    out2, ent2 = _drift(ctx, st, 1, 0.8, 0.04, 0.1, 0.14, 1.2, 8, drag=0.3)
    assert len(ent2) == 0
    for f in ("x", "y", "z", "v"):
        assert np.array_equal(out2[f], plain[f]), f


def test_lightcone_many_candidates_first_drift(ctx, oracle):
    """128^3 particles: the first drift's candidates overflow the initial candidate room, the
    pass is redone after the list grows, and the entries still agree with the oracle's."""
    x, y, z, v, _ = ics.zeldovich_lattice(128, index=-2.0, rms_spacing=0.25, seed=8)
    v = (v * 10.0).astype(np.float32)
    r = np.zeros(len(x), np.int8)
    st = (x, y, z, v, r)
    out, ent = _drift(ctx, st, 0, 1.0, 0.01, 0.62, 0.63, 1.5, 128)
    xs, ys, zs, vs = (q.copy() for q in (x, y, z, v))
    oent = oracle.drift_lc(xs, ys, zs, vs, r, 0, 1.0, 0.01, 0.62, 0.63, 1.5, 128)
    print("lightcone 128^3: %d entries" % len(ent))
    assert len(ent) > 70000
    assert len(ent) == len(oent)
    a_, b_ = _sorted(ent), _sorted(oent)
    for f in ("x", "y", "z"):
        assert np.max(np.abs(a_[f].astype(np.int64) - b_[f].astype(np.int64))) <= 2, f
    assert np.mean(a_["pix"] == b_["pix"]) > 0.999
    assert np.array_equal(out["x"], xs) and np.array_equal(out["y"], ys) and np.array_equal(out["z"], zs)
