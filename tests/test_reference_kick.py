"""This project's kick and drift against the reference's OWN CUDA kernels, run on the same GPU.

The reference's device code (src/kick.cu cuda_kick_kernel with src/gravity.cu, src/drift.cu
cuda_drift_kernel) is compiled from its sources for sm_100a (oracle/_ref/libctref_gpu.so,
`make -C oracle refgpu`) and driven through a host harness: the reference kernel walks the
whole tree from one root work item, on the particles and the tree that this project's
tree build produced (the tree build itself is bit-exact against the oracle's restatement of
tree_create).  On clustered boxes forces, potentials and velocities must agree within 1e-5
relative RMS; on a near-uniform lattice, where the reference's Ewald operator has an error
floor, this kick must be at least as accurate against the FP64 direct Ewald sum; the drift
must agree bit for bit.

The inputs keep the reference kernel's device asserts (which trap) out of reach: every rung
starts at 0 and a kick raises a rung by at most one (kick.cu:136-140, MAX_RUNG = 16); leaves
satisfy the Ewald criterion by the tree_create leaf rule; sizes are small (one warp walks
the whole tree).
"""
import numpy as np
import pytest

from cosmictiger_b200 import ics
from tests import reference_gpu_lib as rg

pytestmark = pytest.mark.gpu

KICK_RMS_TOL = 1e-5


def rel_rms(a, b):
    return float(np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)))


@pytest.fixture(scope="module")
def ref():
    if not rg.available():
        pytest.fail("oracle/_ref/libctref_gpu.so is not built (make -C oracle refgpu)")
    return rg.ReferenceGPU()


@pytest.fixture(scope="module")
def ctx():
    import cosmictiger_b200 as ct

    c = ct.Context(order=7)
    yield c
    c.close()


def kick_both(ctx, ref, x, y, z, v, r, theta, direct=False):
    """Tree build here, then this project's kick and the reference's kernel on the same
    tree-ordered particles and tree; optionally the FP64 direct Ewald sum at every particle."""
    import cosmictiger_b200 as ct

    N = len(x)
    h = ics.softening(N, 0.02)
    eta = ics.eta_default()
    box = ctx.box(N)
    box.upload(x, y, z, v, r)
    box.tree_create(theta, h, 128)
    before = box.download()  # tree order, the input of both kicks
    nodes = box.tree()
    kr = box.kick(ct.KickParams.make(theta=theta, h=h, GM=1.0 / N, eta=eta, t0=1.0 / 64, first_call=True, save_force=True))
    out = box.download(forces=True)
    rp = rg.RefKickParams(sign=1.0, min_rung=0, a=1.0, t0=1.0 / 64, theta=theta, h=h, eta=eta, GM=1.0 / N, max_dt=1e30, save_force=1, first_call=1,
                          ascending=1, descending=1, top=1, do_phi=1)
    ro = ref.kick(before, nodes, rp)
    gd = None
    if direct:
        dg = box.direct_ewald(before["x"], before["y"], before["z"], h)
        gd = np.stack(dg[:3], 1) / N
    box.close()
    return kr, out, ro, gd


def forces(d):
    return np.stack([d["gx"], d["gy"], d["gz"]], 1).astype(np.float64)


@pytest.mark.parametrize("n,theta,seed", [(16, 0.55, 2), (16, 0.3, 2), (24, 0.55, 5)])
def test_kick_matches_reference_cuda_kick(ctx, ref, n, theta, seed):
    """Clustered boxes: forces, potentials and kicked velocities within 1e-5 relative RMS of
    the reference's own kick, the same rungs and kick-return sums."""
    x, y, z, v, r = ics.clustered_box(n, nspheres=20, seed=seed)
    kr, out, ro, _ = kick_both(ctx, ref, x, y, z, v, r, theta)
    ferr = rel_rms(forces(out), forces(ro))
    perr = rel_rms(out["pot"].astype(np.float64), ro["pot"].astype(np.float64))
    verr = rel_rms(out["v"].astype(np.float64), ro["v"].astype(np.float64))
    rdiff = float(np.mean(out["rung"] != ro["rung"]))
    print("vs reference CUDA kick, clustered n=%d theta=%g: force rel rms %.3g, potential rel rms %.3g, velocity rel rms %.3g, rungs differing %.2g"
          % (n, theta, ferr, perr, verr, rdiff))
    assert ferr < KICK_RMS_TOL, ferr
    assert perr < KICK_RMS_TOL, perr
    assert verr < KICK_RMS_TOL, verr
    assert rdiff < 1e-3
    assert kr.max_rung == ro["max_rung"]
    assert abs(kr.kin - ro["kin"]) <= 1e-5 * abs(ro["kin"])


@pytest.mark.parametrize("theta", [0.7, 0.25])
def test_lattice_kick_at_least_as_accurate_as_reference(ctx, ref, theta):
    """Near-uniform lattice: net forces are small residuals of large periodic sums, so the
    reference's Ewald operator for the n = 0 image (a downward recursion that loses accuracy
    at small separations, fmm_kernels.hpp:333-356) leaves an error floor that this project's
    convergent series does not have.  Against the FP64 direct Ewald sum this kick must be at
    least as accurate as the reference's, and the two may differ only by the reference's own
    error; at theta = 0.25 the floor shows (the reference stays near 3e-3)."""
    x, y, z, v, r = ics.zeldovich_lattice(16, index=-2.0, rms_spacing=0.25, seed=1)
    kr, out, ro, gd = kick_both(ctx, ref, x, y, z, v, r, theta, direct=True)
    e_ours = rel_rms(forces(out), gd)
    e_ref = rel_rms(forces(ro), gd)
    gap = rel_rms(forces(out), forces(ro))
    print("lattice 16^3 theta=%g: force error vs FP64 Ewald %.3g (here) / %.3g (reference kick); difference %.3g" % (theta, e_ours, e_ref, gap))
    assert e_ours <= 1.02 * e_ref
    assert gap <= e_ref
    if theta < 0.3:
        assert e_ours < 0.2 * e_ref
    assert float(np.mean(out["rung"] != ro["rung"])) < 1e-3


def test_drift_matches_reference_cuda_drift(ctx, ref):
    rng = np.random.default_rng(17)
    N = 40000
    x, y, z = (rng.integers(0, 2 ** 32, N, dtype=np.uint64).astype(np.uint32) for _ in range(3))
    v = (rng.standard_normal((N, 3)) * 0.3).astype(np.float32)
    r = rng.integers(0, 3, N).astype(np.int8)
    for level, a, dt in ((0, 1.0, 0.01), (1, 0.7, 0.013), (2, 0.31, 0.002)):
        box = ctx.box(N)
        box.upload(x, y, z, v, r)
        box.drift(level, a, dt)
        out = box.download()
        rx, ry, rz = ref.drift(x, y, z, v, r, level, a, dt)
        moved = float(np.mean(out["x"] != x))
        print("vs reference CUDA drift, rung %d: %.3f of the particles moved" % (level, moved))
        assert moved > 0.2
        assert np.array_equal(out["x"], rx) and np.array_equal(out["y"], ry) and np.array_equal(out["z"], rz)
        box.close()


def test_kick_matches_reference_production_work_items(ctx, ref, oracle):
    """The reference's kick in its production form: the CPU top of the walk (the oracle's
    restatement, kick.cpp:150-507 with kick.cu's list rules) hands the subtrees of at most
    max_parts particles (kick.cpp:173-177) to cuda_execute_kicks as work items ordered by first
    particle (kick_workspace.cpp:308-310); the reference's kernel then walks them on its
    resident grid.  Same tree and particles as this project's kick: forces, potentials and
    velocities within 1e-5 relative RMS, and the same rungs."""
    import cosmictiger_b200 as ct
    from tests import oracle_lib

    x, y, z, v, r = ics.clustered_box(48, nspheres=int(round(20000 * (48 / 256) ** 3)), seed=7)
    N = len(x)
    theta = 0.55
    h = ics.softening(N, 0.02)
    eta = ics.eta_default()
    nodes = oracle.tree_build(x, y, z, v, r, theta, h, 128)
    box = ctx.box(N)
    box.upload(x, y, z, v, r)
    box.tree_create(theta, h, 128)
    before = box.download()
    assert np.array_equal(before["x"], x)  # already in tree order
    t0 = 1.0 / 64
    kr = box.kick(ct.KickParams.make(theta=theta, h=h, GM=1.0 / N, eta=eta, t0=t0, first_call=True, save_force=True))
    out = box.download(forces=True)
    box.close()
    okp = oracle_lib.KickParams(sign=1.0, min_rung=0, a=1.0, t0=t0, theta=theta, h=h, eta=eta, GM=1.0 / N, max_dt=1e30, save_force=1, first_call=1,
                                ascending=1, descending=1, top=1, do_phi=1)
    plan = oracle.plan(okp, nodes, x, y, z, max_parts=ref.max_parts(N))
    items = plan.export()
    plan.close()
    assert len(items["self"]) > 100
    rp = rg.RefKickParams(sign=1.0, min_rung=0, a=1.0, t0=t0, theta=theta, h=h, eta=eta, GM=1.0 / N, max_dt=1e30, save_force=1, first_call=1,
                          ascending=1, descending=1, top=1, do_phi=1)
    ro = ref.kick_items(before, nodes, rp, items, repeats=1)
    ferr = rel_rms(forces(out), forces(ro))
    perr = rel_rms(out["pot"].astype(np.float64), ro["pot"].astype(np.float64))
    verr = rel_rms(out["v"].astype(np.float64), ro["v"].astype(np.float64))
    rdiff = int(np.sum(out["rung"] != ro["rung"]))
    print("vs reference CUDA kick on %d work items (clustered 48^3): force rel rms %.3g, potential %.3g, velocity %.3g, rungs differing %d, %.2f ms"
          % (len(items["self"]), ferr, perr, verr, rdiff, ro["ms"][0]))
    assert ferr < KICK_RMS_TOL and perr < KICK_RMS_TOL and verr < KICK_RMS_TOL
    assert rdiff <= 2
    assert kr.max_rung == ro["max_rung"]
