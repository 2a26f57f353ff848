"""The benchmark's reference arm (the CPU oracle timed on the host) keeps the JSON line the
benchmark contract asks for, and the power.init reader round-trips a table."""
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--n", "32", "--steps", "1", "--warmup", "0"],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling", "dtype", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["value"] > 0 and d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] in ("port", "reference") and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert "workload" in d["config"]


def test_read_power_init_round_trip(tmp_path):
    from cosmictiger_b200 import ics

    k, P = ics.power_law_table(n=64, kcut=5.0)
    path = tmp_path / "power.init"
    with open(path, "w") as f:
        for a, b in zip(k, P):
            f.write("%.9e %.9e\n" % (a, b))
    k2, P2 = ics.read_power_init(str(path))
    assert k2.dtype == np.float32 and P2.dtype == np.float32
    assert np.allclose(k2, k, rtol=1e-7) and np.allclose(P2, P, rtol=1e-7)
    # log-uniform in k, as the reference's reader assumes
    d = np.diff(np.log(k2.astype(np.float64)))
    assert np.allclose(d, d[0], rtol=1e-4)


def test_reference_arm_under_torchrun_two_ranks():
    """Launched as the multi-GPU bench is (torch.distributed.run, two ranks on one node): rank 0
    alone runs the CPU reference arm and prints the one JSON line; the other rank exits 0
    without work."""
    import socket

    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr", "127.0.0.1",
           "--master-port", str(port), os.path.join(ROOT, "bench.py"), "--impl", "reference", "--grid", "32", "--steps", "1", "--warmup", "0"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.lstrip().startswith("{")]
    assert len(lines) == 1, out.stdout[-2000:]
    d = json.loads(lines[0].strip())
    assert d["impl"] == "reference" and d["value"] > 0
