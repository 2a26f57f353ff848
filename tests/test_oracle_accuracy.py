"""The CPU oracle's tree and kick (O1) against its own FP64 direct Ewald sum (O3 restated on the
host): a physics check of the restatement independent of the reference.  The force error falls
with the opening angle and with the expansion order, and is 1e-4 or less at theta 0.55, order 7."""
import numpy as np

from cosmictiger_b200 import ics


def _force_error(oracle, order, theta, state):
    from tests import oracle_lib

    x, y, z, v, r = (q.copy() for q in state)
    N = len(x)
    h = ics.softening(N, 0.02)
    nodes = oracle.tree_build(x, y, z, v, r, theta, h, 128, order=order)
    kp = oracle_lib.KickParams(sign=1.0, min_rung=0, a=1.0, t0=1.0, theta=theta, h=h, eta=ics.eta_default(), GM=1.0 / N, max_dt=1e30,
                               save_force=1, first_call=1, ascending=1, descending=1, top=1, do_phi=1)
    (gx, gy, gz, _), _, _ = oracle.kick(kp, nodes, x, y, z, v, r, order=order)
    sel = np.arange(0, N, 7)
    d = oracle.direct_ewald(x, y, z, x[sel], y[sel], z[sel], h)
    gd = np.stack(d[:3], 1) / N
    gt = np.stack([gx[sel], gy[sel], gz[sel]], 1).astype(np.float64)
    return float(np.sqrt(np.sum((gt - gd) ** 2) / np.sum(gd ** 2)))


def test_oracle_kick_accuracy_against_fp64_ewald(oracle):
    state = ics.clustered_box(14, nspheres=15, seed=7)
    err = {(o, t): _force_error(oracle, o, t, state) for o in (5, 7) for t in (0.3, 0.55, 0.8)}
    print({k: "%.2e" % e for k, e in err.items()})
    for o in (5, 7):
        assert err[(o, 0.3)] < err[(o, 0.55)] < err[(o, 0.8)], o
    for t in (0.3, 0.55, 0.8):
        assert err[(7, t)] < err[(5, t)], t
    assert err[(7, 0.55)] < 1e-4
