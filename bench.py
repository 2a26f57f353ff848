#!/usr/bin/env python3
"""Gravity-step benchmark: particle-steps/s of tree build + kick + drift on one B200.

Workload (default): the clustered 256^3 box -- 70% of 16.8M particles on a Zel'dovich-displaced
lattice (P(k) ~ k^-1.5, 0.5 mean-spacing RMS), 30% in 20,000 Plummer spheres with power-law
masses -- at theta = 0.55, expansion order 7, softening 1/50 of the mean spacing, Ewald on.
A step (--mode multistep, the default) is one hierarchical step of kick_step_hierarchical:
the rung ladder of sorts, tree builds over the active particles, kicks and drifts, so that
value counts particle-steps of the whole box per device second.  --mode single kicks every
particle each step (one tree build, one kick, one drift).  Inputs are seeded synthetic
stand-ins generated here (no dataset is involved).

  value   particle-steps/s with particles resident in HBM (device-timed, CUDA events)
  e2e     the same through the public API with host buffers: every step uploads the
          particles from pinned host memory and downloads positions, velocities and rungs
  roofline  k_p2p (the particle-particle kernel, the largest share of the step) on the
          all-particles step against the measured FP32 FMA peak, 21 flops per pair (the
          reference's per-interaction count), timed by CUDA events on the library's stream
  cpu_baseline  the CPU oracle (this project's restatement of the reference's algorithm; the
          reference's own CPU kick cannot run) on a bounded sample of the same workload

--impl reference times that CPU implementation alone on all host cores.
Multi-GPU (--gpus N under torchrun): independent boxes per rank (weak scaling, no collective
on the data path); value = all ranks' particle-steps / max rank time.
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", "--grid", dest="n", type=int, default=256, help="particles = n^3 (spell it --grid under torch.distributed.run, which takes --n for its own --nnodes/--nproc-per-node)")
    ap.add_argument("--theta", type=float, default=0.55)
    ap.add_argument("--workload", default="clustered", choices=["clustered", "lattice"])
    ap.add_argument("--mode", default="multistep", choices=["multistep", "single"],
                    help="multistep: hierarchical rung ladder (kick_step_hierarchical); single: all particles every step")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-ref-gpu", action="store_true", help="skip the reference's own CUDA kick on the same box")
    ap.add_argument("--no-tune", action="store_true", help="keep the default launch shape instead of autotuning it first")
    ap.add_argument("--accuracy-sinks", type=int, default=10000, help="FP64 direct-Ewald check on this many seeded sinks (0: skip)")
    ap.add_argument("--ensemble-boxes", type=int, default=512, help="boxes of the batched-vs-plain ensemble comparison (0: skip)")
    ap.add_argument("--ensemble-nmin", type=int, default=16)
    ap.add_argument("--ensemble-nmax", type=int, default=128)
    ap.add_argument("--ensemble-steps", type=int, default=20)
    ap.add_argument("--study", default="none", choices=["none", "precision", "ensemble", "serving", "lightcone", "fourier", "autotune"],
                    help="instead of the benchmark line: precision (theta x order x summation, force error vs FP64 Ewald and "
                         "particle-steps/s), ensemble (512 boxes of 16^3..128^3, batched vs box by box, 20 steps) or serving "
                         "(Poisson arrivals of 32^3..256^3 requests, rate sweep, p50/p99 latency vs sequential runs) or lightcone "
                         "(drift with the lightcone capture vs plain drift) or fourier (IC generator and power spectrum on an n^3 grid)")
    ap.add_argument("--study-seed", type=int, default=11)
    ap.add_argument("--serving-lanes", type=int, default=2, help="serving study: device contexts (streams), each driven by its own host thread")
    ap.add_argument("--serving-requests", type=int, default=48, help="serving study: requests per arrival rate")
    ap.add_argument("--serving-big-total", type=int, default=1, help="serving study: large requests (above 2^20 particles) active at once over "
                    "all lanes (0: one per lane)")
    return ap.parse_args()


def make_ensemble(nbox, nmin, nmax, seed):
    """nbox boxes of n_i^3 particles, n_i log-uniform in [nmin, nmax] (seeded), each with its
    own Zel'dovich field: spectral index uniform in [-2.5, -1], RMS displacement uniform in
    0.1-0.6 mean spacings."""
    from cosmictiger_b200 import ics

    rng = np.random.default_rng(seed)
    ns = np.rint(np.exp(rng.uniform(np.log(nmin), np.log(nmax), nbox))).astype(int)
    idx = rng.uniform(-2.5, -1.0, nbox)
    rms = rng.uniform(0.1, 0.6, nbox)
    jobs = [(int(n), float(i), float(r), int(seed * 1000 + k)) for k, (n, i, r) in enumerate(zip(ns, idx, rms))]
    # every box has its own seed, so the threads' order does not change the result; numpy's
    # FFTs release the interpreter lock, so the host's cores share the generation
    from concurrent.futures import ThreadPoolExecutor

    with ThreadPoolExecutor(max(1, min(16, os.cpu_count() or 1))) as ex:
        return list(ex.map(lambda j: ics.zeldovich_lattice(j[0], index=j[1], rms_spacing=j[2], seed=j[3]), jobs))


def ensemble_compare(ct, torch, ctx, args, theta, lib_stream):
    """Aggregate particle-steps/s of an ensemble run as one batched ensemble vs the plain
    single-box path launched box by box; per-box latency percentiles of the plain path."""
    from cosmictiger_b200 import ics

    sets = make_ensemble(args.ensemble_boxes, args.ensemble_nmin, args.ensemble_nmax, seed=4)
    counts = [len(s[0]) for s in sets]
    N = int(np.sum(counts))
    h = ics.softening(float(np.mean(counts)), 0.02)
    eta = ics.eta_default()
    t0 = 1.0 / 64
    hs = np.array([ics.softening(n, 0.02) for n in counts], np.float32)
    gms = np.array([1.0 / n for n in counts], np.float32)
    # the launch shape tuned for this workload (the first 128 boxes of the set, batched; 12
    # candidates, timing only), used by both paths and put back afterwards
    prev_shape = ctx.tuning()
    shape = None
    if not args.no_tune:
        from cosmictiger_b200 import autotune

        nt = min(len(sets), 128)
        tc = counts[:nt]
        tcat = [np.concatenate([s[k] for s in sets[:nt]]) for k in range(5)]

        def factory():
            e = ctx.ensemble(tc)
            e.upload(*tcat)
            e.set_box_params(hs[:nt], gms[:nt])
            return e

        try:
            tr = autotune.tune(ctx, tcat, theta=theta, h=float(hs[:nt].max()), buckets=(128,), max_force_rms=None, repeats=1, box_factory=factory,
                               forces=False)
            shape = {"chosen": {k: tr["best"][k] for k in ("p2p_stage", "warps_per_tile", "tile_width")}, "ms_kick_chosen": tr["best"]["ms"],
                     "ms_kick_default": tr["reference"]["ms"], "candidates": len(tr["rows"]), "tuned_on": "the first %d boxes, batched" % nt}
        except Exception as e:  # reported; both paths then run at the context's shape
            ctx.set_tuning(prev_shape["p2p_stage"], prev_shape["warps_per_tile"], prev_shape["tile_width"])
            shape = {"failed": str(e), **prev_shape}
        del tcat
    ens = ctx.ensemble(counts)
    ens.upload(*[np.concatenate([s[k] for s in sets]) for k in range(5)])
    ens.set_box_params(hs, gms)

    def ens_step(first):
        ens.tree_create(theta, float(hs.max()), 128)
        ens.kick(ct.KickParams.make(theta=theta, h=float(hs.max()), GM=1.0 / N, eta=eta, t0=t0, first_call=first, save_force=False))
        ens.drift(0, 1.0, t0)

    plain = []
    for s in sets:
        bx = ctx.box(len(s[0]))
        bx.upload(*s)
        plain.append(bx)

    def plain_step(first, lat=None):
        for k, bx in enumerate(plain):
            t = time.perf_counter()
            bx.tree_create(theta, float(hs.max()), 128)
            bx.kick(ct.KickParams.make(theta=theta, h=float(hs[k]), GM=float(gms[k]), eta=eta, t0=t0, first_call=first, save_force=False))
            bx.drift(0, 1.0, t0)
            if lat is not None:
                ctx.synchronize()
                lat.append((time.perf_counter() - t) * 1e3)

    for i in range(2):
        ens_step(i == 0)
        plain_step(i == 0)
    ctx.synchronize()
    K = args.ensemble_steps
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(lib_stream)
    for i in range(K):
        ens_step(False)
    e1.record(lib_stream)
    ctx.synchronize()
    torch.cuda.synchronize()
    ms_b = e0.elapsed_time(e1)
    cb = ens.counters()
    breakdown = {k: cb[k] for k in ("ms_tree", "ms_walk", "ms_m2l", "ms_leaf", "ms_leafkick", "cc_ewald", "cc_direct", "cp_pairs", "pp_pairs", "nodes")
                 if k in cb}
    e0.record(lib_stream)
    for i in range(K):
        plain_step(False)
    e1.record(lib_stream)
    ctx.synchronize()
    torch.cuda.synchronize()
    ms_p = e0.elapsed_time(e1)
    lat = []
    plain_step(False, lat)
    for bx in plain:
        bx.close()
    ens.close()
    ctx.set_tuning(prev_shape["p2p_stage"], prev_shape["warps_per_tile"], prev_shape["tile_width"])
    vb = N * K / (ms_b / 1e3)
    vp = N * K / (ms_p / 1e3)
    return {"boxes": len(counts), "particles": N, "n_range": [args.ensemble_nmin, args.ensemble_nmax], "steps": K,
            "launch_shape": shape if shape else prev_shape,
            "batched_particle_steps_s": vb, "plain_particle_steps_s": vp, "speedup": vb / vp,
            "batched_ms_per_step": ms_b / K, "batched_last_kick": breakdown, "plain_box_ms_p50": float(np.percentile(lat, 50)), "plain_box_ms_p99": float(np.percentile(lat, 99))}


def make_ics(args, seed):
    from cosmictiger_b200 import ics

    if args.workload == "clustered":
        nsph = max(1, int(round(20000 * (args.n / 256.0) ** 3)))
        return ics.clustered_box(args.n, nspheres=nsph, seed=seed)
    return ics.zeldovich_lattice(args.n, index=-2.0, rms_spacing=0.25, seed=seed)


def workload_name(args):
    steps = "4-rung hierarchical steps" if args.mode == "multistep" else "all particles per step"
    if args.workload == "clustered":
        return "clustered %d^3 (70%% Zel'dovich k^-1.5 / 30%% Plummer), theta %.2f, order 7, Ewald, %s" % (args.n, args.theta, steps)
    return "lattice %d^3 Zel'dovich k^-2, theta %.2f, order 7, Ewald, all particles per step" % (args.n, args.theta)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [s.strip() for s in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if p[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return
    if args.study != "none":
        if rank == 0:
            run_study(args)
        return
    import torch

    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    import cosmictiger_b200 as ct
    from cosmictiger_b200 import ics

    x, y, z, v, r = make_ics(args, seed=3 + 101 * rank)
    N = len(x)
    theta = args.theta
    h = ics.softening(N, 0.02)
    GM = 1.0 / N
    eta = ics.eta_default()
    t0 = 1.0 / 64
    ctx = ct.Context(device=local, order=7)
    tuning = None
    if not args.no_tune:
        # the kick's launch shape (P2P cell-list size, warps per sink tile, sink tile width)
        # tuned on this workload at the benchmark's leaf size; results change only by rounding
        from cosmictiger_b200 import autotune

        tr = autotune.tune(ctx, (x, y, z, v, r), theta=args.theta, h=ics.softening(N, 0.02), buckets=(128,), max_force_rms=1e-5, repeats=1)
        tuning = {"chosen": {k: tr["best"][k] for k in ("p2p_stage", "warps_per_tile", "tile_width")}, "ms_kick_chosen": tr["best"]["ms"],
                  "ms_kick_default": tr["reference"]["ms"], "candidates": len(tr["rows"]), "by": "cosmictiger_b200.autotune.tune (device time of "
                  "one all-particles tree build + kick per candidate)"}
    box = ctx.box(N)
    box.upload(x, y, z, v, r)

    def step(first):
        box.tree_create(theta, h, 128)
        kp = ct.KickParams.make(theta=theta, h=h, GM=GM, eta=eta, t0=t0, first_call=first, save_force=False)
        kr = box.kick(kp)
        box.drift(0, 1.0, t0)
        return kr

    ms = None
    cpu_seed = ((x, y, z, v, r), None, t0)
    if args.mode == "multistep":
        # choose t0 so that the rung rule dt = eta sqrt(a h / |g|) (kick.cu:133-136) spreads the
        # particles over rungs 0-3: 1% of them want rung >= 3
        box.tree_create(theta, h, 128)
        box.kick(ct.KickParams.make(theta=theta, h=h, GM=GM, eta=eta, t0=1.0, save_force=True, descending=False, ascending=False))
        g = box.download(forces=True)
        gm = np.sqrt(g["gx"].astype(np.float64) ** 2 + g["gy"] ** 2 + g["gz"] ** 2)
        dts = eta * np.sqrt(h / np.maximum(gm, 1e-30))
        ms = {"t0": float(8.0 * np.percentile(dts, 1))}
        # the CPU legs start from these particles (tree order) with rungs set by these forces
        cpu_seed = ((g["x"], g["y"], g["z"], g["v"], g["rung"]), np.stack([g["gx"], g["gy"], g["gz"]], 1), ms["t0"])
        del g, gm, dts
        box.upload(x, y, z, v, r)
        box.sort_by_rung(0)
        ms["state"] = dict(minrung=0, max_rung=0, tau=0.0)

        def mstep():
            s = ms["state"]
            sp = ct.StepParams(minrung=s["minrung"], minrung0=0, max_rung=s["max_rung"], a=1.0, tau=s["tau"], t0=ms["t0"], theta=theta, hsoft=h,
                               bucket=128, eta=eta, GM=GM, max_dt=1e30, do_phi=1, nocrop=0, drag=0.0, sign=1.0)
            res = box.step_hierarchical(sp)
            s["minrung"], s["max_rung"], s["tau"] = res.minrung, res.max_rung, s["tau"] + ms["t0"]
            return res

        for i in range(args.warmup):
            mstep()
    else:
        # warm-up (the first is the reference's first call: no ascending half kick)
        for i in range(args.warmup):
            step(i == 0)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    # events on the library's own stream
    lib_stream = torch.cuda.ExternalStream(ctx.lib.ct_stream(ctx.h))
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    launches0 = ctx.launches()
    t_start = time.perf_counter()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(lib_stream)
    leaf_ms, leafkick_ms = [], []
    walk_ms, m2l_ms, tree_ms = [], [], []
    counters = None
    kicked = 0.0
    for i in range(args.steps):
        if ms is not None:
            res = mstep()
            kicked += res.particles_kicked
        else:
            step(False)
            kicked += N
        c = box.counters()
        leaf_ms.append(c["ms_leaf"])
        leafkick_ms.append(c["ms_leafkick"])
        walk_ms.append(c["ms_walk"])
        m2l_ms.append(c["ms_m2l"])
        tree_ms.append(c["ms_tree"])
        counters = c
    ev1.record(lib_stream)
    ctx.synchronize()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t_start
    launches = ctx.launches() - launches0
    clocks = sampler.stop()
    ms_dev = ev0.elapsed_time(ev1)
    ms_step = ms_dev / args.steps
    t_max = ms_dev
    if pg:
        tt = torch.tensor([ms_dev], device="cuda")
        pg.all_reduce(tt, op=pg.ReduceOp.MAX)
        t_max = float(tt.item())
    value = N * world * args.steps / (t_max / 1e3)
    multistep = None
    if ms is not None:
        rc = box.rung_counts()
        multistep = {"t0": ms["t0"], "rung_counts": [int(q) for q in rc[:8]], "active_kicks_per_step": kicked / args.steps,
                     "active_kicks_s": kicked * world / (t_max / 1e3), "minrung": ms["state"]["minrung"], "max_rung": ms["state"]["max_rung"]}

    # ---- e2e through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        cur = box.download()
        def pinned_set(src=None):
            xyz = [torch.empty(N, dtype=torch.int32).pin_memory().numpy().view(np.uint32) for _ in range(3)]
            vv = torch.empty((N, 3), dtype=torch.float32).pin_memory().numpy()
            rr = torch.empty(N, dtype=torch.int8).pin_memory().numpy()
            if src is not None:
                for a, k in zip(xyz, ("x", "y", "z")):
                    np.copyto(a, src[k])
                np.copyto(vv, src["v"])
                np.copyto(rr, src["rung"])
            return xyz + [vv, rr]

        # two pinned host sets used in turn: each step uploads the particles from one and
        # downloads its result into the other, which the next step uploads
        bufs = [pinned_set(cur), pinned_set()]

        def e2e_step(first):
            src, dst = bufs[0], bufs[1]
            box.upload(*src)
            if ms is not None:
                mstep()
            else:
                step(first)
            p = lambda a: ctypes.c_void_p(a.ctypes.data)  # noqa: E731
            ctx.check(ctx.lib.ct_box_download(ctx.h, box.id, *[p(a) for a in dst], None, None, None, None), "download")
            bufs.reverse()

        e2e_step(True)
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(lib_stream)
        ke = args.steps
        for i in range(ke):
            e2e_step(False)
        e1.record(lib_stream)
        torch.cuda.synchronize()
        ms_e = e0.elapsed_time(e1)
        if pg:
            tt = torch.tensor([ms_e], device="cuda")
            pg.all_reduce(tt, op=pg.ReduceOp.MAX)
            ms_e = float(tt.item())
        e2e = {"value": N * world * ke / (ms_e / 1e3), "unit": "particle-steps/s", "h2d_bytes_per_step": int(N * (12 + 12 + 1)),
               "d2h_bytes_per_step": int(N * (12 + 12 + 1))}
    if multistep is not None:
        # the all-particles step on the same box, for reference and for the leaf roofline
        box.upload(x, y, z, v, r)
        box.sort_by_rung(0)
        for i in range(2):
            step(i == 0)
        ctx.synchronize()
        e0s = torch.cuda.Event(enable_timing=True)
        e1s = torch.cuda.Event(enable_timing=True)
        e0s.record(lib_stream)
        ks = max(2, min(args.steps, 3))
        leaf_ms, leafkick_ms, walk_ms, m2l_ms, tree_ms = [], [], [], [], []
        for i in range(ks):
            step(False)
            c = box.counters()
            leaf_ms.append(c["ms_leaf"])
            leafkick_ms.append(c["ms_leafkick"])
            walk_ms.append(c["ms_walk"])
            m2l_ms.append(c["ms_m2l"])
            tree_ms.append(c["ms_tree"])
            counters = c
        e1s.record(lib_stream)
        ctx.synchronize()
        torch.cuda.synchronize()
        multistep["single_rung_particle_steps_s"] = N * ks / (e0s.elapsed_time(e1s) / 1e3)
        multistep["single_rung_ms_per_step"] = e0s.elapsed_time(e1s) / ks
    # ---- roofline of the leaf kernel (reference flop convention)
    L = ctx.lib
    pk = ctypes.c_double(0)
    ctx.check(L.ct_fp32_peak(ctx.h, ctypes.byref(pk)), "ct_fp32_peak")
    peak_tf = pk.value
    c = counters
    # k_p2p: 21 flops per particle pair (the reference's count, gravity.hpp), per launch
    p2p_flops = 21.0 * c["pp_pairs"]
    p2p_s = float(np.mean(leaf_ms)) / 1e3
    achieved = p2p_flops / p2p_s / 1e12
    traffic = read_traffic()
    roofline = {"bound": "fp32_fma", "kernel": "k_p2p (particle-particle forces, all-particles step)", "achieved": achieved, "peak": peak_tf,
                "unit": "TFLOP/s", "frac": achieved / peak_tf if peak_tf else None, "traffic": traffic,
                "flops_per_launch": p2p_flops, "ms_per_launch": p2p_s * 1e3,
                "peak_source": "measured on this GPU by ct_fp32_peak (FFMA chains, 2 flops per FMA); the measured peaks file has no FP32 entry"}
    extra = {"ms_tree": float(np.mean(tree_ms)), "ms_walk": float(np.mean(walk_ms)), "ms_m2l": float(np.mean(m2l_ms)), "ms_p2p": float(np.mean(leaf_ms)),
             "ms_leafkick": float(np.mean(leafkick_ms)),
             "pp_pairs": c["pp_pairs"], "cc_direct": c["cc_direct"], "cc_ewald": c["cc_ewald"], "pc_pairs": c["pc_pairs"], "cp_pairs": c["cp_pairs"],
             "nodes": c["nodes"], "leaves": c["leaves"], "flops_per_step": c["flops"], "wall_s": wall}
    ens_res = None
    if args.ensemble_boxes > 0:
        ens_res = ensemble_compare(ct, torch, ctx, args, theta, lib_stream)
    acc = None
    if args.accuracy_sinks:
        # every rank checks its own box (rank 0 reports), so that no rank waits at the barrier
        # below for another's check
        def steps_fn(th):
            box.upload(x, y, z, v, r)
            box.sort_by_rung(0)
            return timed_steps(torch, ctx, box, th, h, N, 2, lib_stream)

        acc = accuracy(box, args.accuracy_sinks, h, N, theta, steps_fn=steps_fn if world == 1 else None)
    cpu = None
    c1 = None
    if not args.no_cpu and rank == 0 and world == 1:
        cpu = cpu_baseline(args, *cpu_seed)
        try:
            c1 = {"workload": "lattice 64^3 Zel'dovich k^-2, 0.25 spacing RMS, theta 0.7, order 7, Ewald, one all-particles step (tree, kick, drift)",
                  "gpu": gpu_c1(ct, torch, ctx, lib_stream), "cpu_full": cpu_c1_full()}
            c1["e2e_speedup"] = c1["cpu_full"]["seconds"] * 1e3 / c1["gpu"]["e2e_ms"]
        except Exception as e:  # reported, never required
            c1 = {"failed": str(e)}
    ref_gpu = None
    if not args.no_ref_gpu and rank == 0 and world == 1:
        try:
            ref_gpu = reference_gpu_compare(ct, torch, ctx, lib_stream, args)
        except Exception as e:  # reported, never required
            ref_gpu = {"failed": str(e)}
    if pg:
        pg.barrier()
    if rank == 0:
        line = {
            "metric": "particle-steps/s at <=1e-3 rms force err; ensemble-batched vs plain; p50/p99 ms",
            "value": value,
            "unit": "particle-steps/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_step,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 (fixed32 positions, f64 tree geometry)",
            "data": "synthetic (seeded generator)",
            "config": {"workload": workload_name(args), "particles_per_gpu": N, "theta": theta, "order": 7, "bucket": 128,
                       "launch_shape": tuning if tuning else ctx.tuning(),
                       "parallelism": "independent boxes per GPU" if world > 1 else "single box",
                       "l2": "inputs larger than L2 (%.0f MB of particle state)" % (N * 41 / 1e6)},
            "e2e": e2e,
            "gpu_launches": launches,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "clocks": clocks,
            "breakdown": extra,
        }
        if acc:
            line["force_error"] = acc
        if ens_res:
            line["ensemble"] = ens_res
        if multistep:
            line["multistep"] = multistep
        if c1:
            line["c1_unsampled"] = c1
        if ref_gpu:
            line["ref_gpu"] = ref_gpu
        print(json.dumps(line), flush=True)
    box.close()
    ctx.close()
    if pg:
        pg.destroy_process_group()


def read_traffic():
    """DRAM bytes per launch of k_p2p from the committed ncu summary, if present."""
    p = os.path.join(ROOT, "profiles", "k_p2p_clustered192.txt")
    if not os.path.exists(p):
        return None
    try:
        for ln in open(p):
            if ln.startswith("dram_bytes_per_launch_full_size="):
                return float(ln.split("=", 1)[1])
    except Exception:
        return None
    return None


def _errors(gt, gd):
    err = np.linalg.norm(gt - gd, axis=1) / np.linalg.norm(gd, axis=1)
    mag = np.abs(np.linalg.norm(gt, axis=1) - np.linalg.norm(gd, axis=1)) / np.linalg.norm(gd, axis=1)
    return {"rms": float(np.sqrt(np.sum((gt - gd) ** 2) / np.sum(gd ** 2))), "rms_per_particle": float(np.sqrt(np.mean(err ** 2))),
            "p99_per_particle": float(np.percentile(err, 99)), "mag_p50": float(np.percentile(mag, 50)), "mag_p99": float(np.percentile(mag, 99))}


SINK_MARK = 1000.0


def mark_sinks(v, sel):
    """A copy of the velocities with the chosen sinks' x velocity set to -(1000 + k): a kick
    without its half steps (ascending and descending off) leaves velocities as they are, so the
    sinks can be found again in any tree order by one scan (find_sinks) instead of a sort."""
    vm = np.array(v, np.float32, copy=True)
    vm[sel, 0] = -(SINK_MARK + np.arange(len(sel), dtype=np.float32))
    return vm


def find_sinks(out, nsink):
    """Rows of the marked sinks in a downloaded state, in the order they were marked."""
    vx = out["v"][:, 0]
    rows = np.nonzero(vx <= -SINK_MARK)[0]
    k = np.rint(-vx[rows] - SINK_MARK).astype(np.int64)
    if len(rows) != nsink or not np.array_equal(np.sort(k), np.arange(nsink)):
        raise RuntimeError("marked sinks lost (%d of %d found)" % (len(rows), nsink))
    idx = np.empty(nsink, np.int64)
    idx[k] = rows
    return idx


def accuracy(box, nsink, h, N, theta, gate_thetas=(0.5, 0.45, 0.4, 0.35), steps_fn=None):
    """Force error of the kick vs the FP64 direct Ewald sum on nsink seeded sinks at the run's
    theta, and the force-error gate: the same sinks (marked, found again in every tree order)
    at smaller theta, each with the particle-steps/s of the all-particles step
    (steps_fn(theta) -> ms), until one passes 1e-3 per-particle RMS."""
    import cosmictiger_b200 as ct

    rng = np.random.default_rng(4321 + 42)
    base = box.download()  # every kick below starts from these positions (timing steps move them)
    sel = np.sort(rng.choice(N, size=min(nsink, N), replace=False))
    vm = mark_sinks(base["v"], sel)

    def kick_at(th):
        box.upload(base["x"], base["y"], base["z"], vm, base["rung"])
        box.sort_by_rung(0)
        box.tree_create(th, h, 128)
        box.kick(ct.KickParams.make(theta=th, h=h, GM=1.0 / N, eta=0.25 / np.sqrt(693 / 256.0), save_force=True, descending=False, ascending=False))
        out = box.download(forces=True)
        idx = find_sinks(out, len(sel))
        return np.stack([out["gx"][idx], out["gy"][idx], out["gz"][idx]], 1).astype(np.float64)

    dg = box.direct_ewald(base["x"][sel], base["y"][sel], base["z"][sel], h)
    gd = np.stack(dg[:3], 1) / N
    gt = kick_at(theta)
    res = {"sinks": int(len(sel)), **_errors(gt, gd),
           "definition": "vs FP64 direct Ewald on seeded sinks: rms = sqrt(sum|dg|^2 / sum|g|^2) (the global norm, dominated by the largest "
                         "forces); per_particle = |dg|/|g| per sink, its rms and 99th percentile (every sink weighted alike, as the "
                         "reference's force test reads its sinks one by one, analytic.cpp:78-89); mag = ||g|-|g_ref||/|g_ref| (that test's "
                         "own measure)"}
    rows = [{"theta": theta, **{k: res[k] for k in ("rms", "rms_per_particle", "p99_per_particle")}}]
    if steps_fn:
        rows[0]["ms_all_particles_step"] = steps_fn(theta)
        rows[0]["particle_steps_s"] = N / (rows[0]["ms_all_particles_step"] / 1e3)
    for th in gate_thetas:
        if rows[-1]["rms_per_particle"] <= 1e-3:
            break
        e = _errors(kick_at(th), gd)
        row = {"theta": th, **{q: e[q] for q in ("rms", "rms_per_particle", "p99_per_particle")}}
        if steps_fn:
            row["ms_all_particles_step"] = steps_fn(th)
            row["particle_steps_s"] = N / (row["ms_all_particles_step"] / 1e3)
        rows.append(row)
    passing = [r for r in rows if r["rms_per_particle"] <= 1e-3]
    res["gate"] = {"order": 7, "rows": rows, "threshold": 1e-3,
                   "passes_global_rms": rows[0]["theta"] if rows[0]["rms"] <= 1e-3 else None,
                   "passes_per_particle_rms": passing[0]["theta"] if passing else None}
    return res


def cpu_start_state(args, state, g, t0):
    """Starting state of the CPU legs: the workload's particles (in the order `g` belongs to)
    with the rungs the rung rule gives for the forces g (N, 3) at step t0, the active range and
    rung stack those rungs leave (tests/oracle_lib.rung_state_from_forces), and the step
    parameters of the benchmark's hierarchical step.  With g None (--mode single) every particle
    stays on rung 0 and a step kicks all of them."""
    from cosmictiger_b200 import ics
    from tests import oracle_lib

    O = oracle_lib.load(build=False)
    x, y, z, v, r = state
    N = len(x)
    h = ics.softening(N, 0.02)
    st = {"x": x.copy(), "y": y.copy(), "z": z.copy(), "v": v.copy(), "rung": np.zeros(N, np.int8), "rung_begin": 0, "stack": []}
    minrung, max_rung = 0, 0
    if g is not None:
        minrung, max_rung = oracle_lib.rung_state_from_forces(O, st, g, t0, ics.eta_default(), h)
    sp = dict(minrung=minrung, minrung0=0, max_rung=max_rung, a=1.0, tau=t0, t0=t0, theta=args.theta, hsoft=h, bucket=128, eta=ics.eta_default(),
              GM=1.0 / N, max_dt=1e30, do_phi=1, nocrop=0 if g is not None else 1, drag=0.0, sign=1.0)
    return st, sp


def cpu_estimates(args, st0, sp0, frac, repeats, seed):
    """Estimated CPU seconds of one step from (st0, sp0), `repeats` times with independent
    samples (tests/oracle_lib.estimate_step_hierarchical on all host threads)."""
    import copy

    from tests import oracle_lib

    O = oracle_lib.load(build=False)
    out = []
    for k in range(repeats):
        st = copy.deepcopy(st0)
        sec, est = oracle_lib.estimate_step_hierarchical(O, st, dict(sp0), frac, seed=seed + 7919 * k)
        out.append((sec, est))
    return out


def cpu_summary(args, N, runs, frac, wall_s, forces="the device's"):
    secs = np.array([r[0] for r in runs])
    est = runs[-1][1]
    vals = N / secs
    return {"value": float(N / secs.mean()), "unit": "particle-steps/s", "cores": int(est["threads"]), "kind": "port",
            "repeats": len(runs), "spread": {"min": float(vals.min()), "max": float(vals.max()), "rel_std": float(vals.std() / vals.mean()) if len(vals) > 1 else 0.0},
            "est_s_per_step": float(secs.mean()), "wall_s": wall_s,
            "sample": "%s: one hierarchical step (the same ladder of rung sorts, tree builds over the active particles, kicks and drifts as the "
                      "device step; %d kicks, %.2e active kicks) per repeat; tree builds (%d threads), the top of each walk, sorts and drifts run in "
                      "full; of %d work items below the top, %d were walked (chosen with probability proportional to a cost proxy, %.0f%% of it "
                      "covered) and the walk of all items estimated from them (Horvitz-Thompson total, thread schedule simulated); starting rungs from %s forces by the rung rule"
                      % (workload_name(args), est["kicks"], est["active"], est["threads"], est["items"], est["sampled_items"], 100 * frac, forces)}


def cpu_baseline(args, state, g, t0):
    import time as _t

    try:
        t = _t.perf_counter()
        st0, sp0 = cpu_start_state(args, state, g, t0)
        runs = cpu_estimates(args, st0, sp0, frac=0.03, repeats=3, seed=12345)
        return cpu_summary(args, len(state[0]), runs, 0.03, _t.perf_counter() - t)
    except Exception as e:  # the baseline is reported, never required
        return {"value": None, "unit": "particle-steps/s", "cores": os.cpu_count(), "kind": "port", "sample": "failed: %s" % e}


def cpu_c1_full():
    """The CPU oracle on the lattice workload (64^3 Zel'dovich k^-2 lattice, 0.25 spacing RMS,
    theta 0.7, one all-particles step: tree build, kick, drift) in full on all host threads, no
    sample and no extrapolation."""
    from cosmictiger_b200 import ics
    from tests import oracle_lib

    O = oracle_lib.load(build=False)
    x, y, z, v, r = ics.zeldovich_lattice(64, index=-2.0, rms_spacing=0.25, seed=3)
    N = len(x)
    h = ics.softening(N, 0.02)
    t = time.perf_counter()
    nodes = O.tree_build(x, y, z, v, r, 0.7, h, 128)
    kp = oracle_lib.KickParams(sign=1.0, min_rung=0, a=1.0, t0=1.0 / 64, theta=0.7, h=h, eta=ics.eta_default(), GM=1.0 / N, max_dt=1e30,
                               save_force=0, first_call=1, ascending=1, descending=1, top=1, do_phi=1)
    O.kick(kp, nodes, x, y, z, v, r, save_force=False)
    O.drift(x, y, z, v, r, 0, 1.0, 1.0 / 64)
    return {"seconds": time.perf_counter() - t, "particles": N, "cores": os.cpu_count()}


def gpu_c1(ct, torch, ctx, lib_stream):
    """The same lattice step on the device: device time (CUDA events) and end to end (host
    buffers in and out) for one all-particles step after one warm-up."""
    from cosmictiger_b200 import ics

    x, y, z, v, r = ics.zeldovich_lattice(64, index=-2.0, rms_spacing=0.25, seed=3)
    N = len(x)
    h = ics.softening(N, 0.02)
    box = ctx.box(N)

    def step():
        box.upload(x, y, z, v, r)
        box.tree_create(0.7, h, 128)
        box.kick(ct.KickParams.make(theta=0.7, h=h, GM=1.0 / N, eta=ics.eta_default(), t0=1.0 / 64, first_call=True, save_force=False))
        box.drift(0, 1.0, 1.0 / 64)
        return box.download()

    step()
    ctx.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    t = time.perf_counter()
    e0.record(lib_stream)
    step()
    e1.record(lib_stream)
    ctx.synchronize()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t
    box.close()
    return {"device_ms": e0.elapsed_time(e1), "e2e_ms": wall * 1e3, "particles": N}


def reference_gpu_compare(ct, torch, ctx, lib_stream, args):
    """The reference's own CUDA kick (src/kick.cu cuda_kick_kernel, compiled from its sources
    for sm_100a, oracle/_ref/libctref_gpu.so) in its production form on the benchmark box: the
    CPU top of the walk (the oracle's restatement) hands subtrees of at most max_parts particles
    (kick.cpp:173-177) to cuda_execute_kicks as work items.  The same tree (the oracle's,
    bit-identical to this project's) and particles; every particle kicked once (first call,
    single rung).  Milliseconds of the second of two calls each (CUDA events; the reference's
    around cuda_execute_kicks, this project's around ct_kick), and the force difference."""
    from cosmictiger_b200 import ics
    from tests import oracle_lib
    from tests import reference_gpu_lib as rg

    if not rg.available():
        return {"unavailable": "oracle/_ref/libctref_gpu.so not built (it is compiled from the reference's sources where they are present)"}
    O = oracle_lib.load(build=False)
    ref = rg.ReferenceGPU(heap_bytes=16 << 30)
    x, y, z, v, r = make_ics(args, seed=3)
    N = len(x)
    h = ics.softening(N, 0.02)
    eta = ics.eta_default()
    theta = args.theta
    t0 = 1.0 / 64
    t = time.perf_counter()
    nodes = O.tree_build(x, y, z, v, r, theta, h, 128)
    t_tree = time.perf_counter() - t
    okp = oracle_lib.KickParams(sign=1.0, min_rung=0, a=1.0, t0=t0, theta=theta, h=h, eta=eta, GM=1.0 / N, max_dt=1e30, save_force=1, first_call=1,
                                ascending=1, descending=1, top=1, do_phi=1)
    mp = ref.max_parts(N)
    plan = O.plan(okp, nodes, x, y, z, max_parts=mp)
    items = plan.export()
    top_s = plan.top_seconds
    plan.close()
    rp = rg.RefKickParams(sign=1.0, min_rung=0, a=1.0, t0=t0, theta=theta, h=h, eta=eta, GM=1.0 / N, max_dt=1e30, save_force=1, first_call=1,
                          ascending=1, descending=1, top=1, do_phi=1)
    state = {"x": x, "y": y, "z": z, "v": v, "rung": r}
    ro = ref.kick_items(state, nodes, rp, items, repeats=2)
    box = ctx.box(N)
    box.upload(x, y, z, v, r)
    box.tree_create(theta, h, 128)
    kp = ct.KickParams.make(theta=theta, h=h, GM=1.0 / N, eta=eta, t0=t0, first_call=True, save_force=True)
    ms = []
    for i in range(2):
        ctx.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(lib_stream)
        box.kick(kp)
        e1.record(lib_stream)
        ctx.synchronize()
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    out = box.download(forces=True)
    box.close()
    g1 = np.stack([out["gx"], out["gy"], out["gz"]], 1).astype(np.float64)
    g0 = np.stack([ro["gx"], ro["gy"], ro["gz"]], 1).astype(np.float64)
    ferr = float(np.sqrt(np.sum((g1 - g0) ** 2) / np.sum(g0 ** 2)))
    perr = float(np.sqrt(np.sum((out["pot"].astype(np.float64) - ro["pot"]) ** 2) / np.sum(ro["pot"].astype(np.float64) ** 2)))
    return {"what": "all-particles kick of the benchmark box (same tree and particles): the reference's cuda_kick_kernel on production work items "
                    "vs this project's kick (walk, interaction kernels, leaf kick)",
            "workload": workload_name(args).replace("4-rung hierarchical steps", "one all-particles kick"), "particles": N,
            "reference_ms": ro["ms"][-1], "this_ms": ms[-1], "speedup": ro["ms"][-1] / ms[-1], "reference_ms_calls": ro["ms"], "this_ms_calls": ms,
            "work_items": int(len(items["self"])), "max_parts": mp, "reference_blocks": ref.kick_block_count(),
            "cpu_top_s": top_s, "cpu_tree_s": t_tree, "force_rel_rms": ferr, "potential_rel_rms": perr}


def run_reference(args):
    """The reference arm: the CPU implementation of the path (the oracle port; the reference's
    own CPU kick aborts in P2P, src/gravity.cpp:257-258) on all host threads, timing the same
    step as the device arm.  The forces that set the starting rungs come from one full CPU kick
    (untimed set-up); every warm-up and timed step is then one estimated hierarchical step from
    that state with an independent sample."""
    from cosmictiger_b200 import ics
    from tests import oracle_lib

    t_all = time.perf_counter()
    state = make_ics(args, seed=3)
    x, y, z, v, r = (a.copy() for a in state)
    N = len(x)
    h = ics.softening(N, 0.02)
    O = oracle_lib.load(build=False)
    g, t0 = None, 1.0 / 64
    t_setup = time.perf_counter()
    if args.mode == "multistep":
        nodes = O.tree_build(x, y, z, v, r, args.theta, h, 128)
        kp = oracle_lib.KickParams(sign=1.0, min_rung=0, a=1.0, t0=1.0, theta=args.theta, h=h, eta=ics.eta_default(), GM=1.0 / N, max_dt=1e30,
                                   save_force=1, first_call=1, ascending=0, descending=0, top=1, do_phi=1)
        (gx, gy, gz, _), _, _ = O.kick(kp, nodes, x, y, z, v.copy(), r.copy())
        g = np.stack([gx, gy, gz], 1)
        dts = ics.eta_default() * np.sqrt(h / np.maximum(np.linalg.norm(g.astype(np.float64), axis=1), 1e-30))
        t0 = float(8.0 * np.percentile(dts, 1))
    t_setup = time.perf_counter() - t_setup
    st0, sp0 = cpu_start_state(args, (x, y, z, v, r), g, t0)
    # each step's sample sized so that warm-up and timed steps together stay within a few minutes
    frac = float(np.clip(0.03 * 12.0 / max(1, args.steps + args.warmup), 0.005, 0.03))
    cpu_estimates(args, st0, sp0, frac=0.002, repeats=args.warmup, seed=999)
    t = time.perf_counter()
    runs = cpu_estimates(args, st0, sp0, frac=frac, repeats=args.steps, seed=4242)
    wall = time.perf_counter() - t
    summ = cpu_summary(args, N, runs, frac, wall, forces="a full CPU kick's")
    v = summ["value"]
    line = {"impl": "reference", "metric": "particle-steps/s at <=1e-3 rms force err; ensemble-batched vs plain; p50/p99 ms", "value": v,
            "unit": "particle-steps/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * N / v,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator)",
            "config": {"workload": workload_name(args), "particles_per_gpu": N, "theta": args.theta, "order": 7, "bucket": 128, "parallelism": "host threads"},
            "cpu_baseline": {k: summ[k] for k in ("value", "unit", "cores", "kind", "sample", "repeats", "spread")},
            "e2e": {"value": v, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "extrapolated": {"what": "ms_per_step is the estimated full CPU step; each timed step walks a sampled %.1f%% (by cost proxy) of the "
                                     "work items and runs tree builds, walk tops, sorts and drifts in full" % (100 * frac),
                             "measured_ms_per_step": 1e3 * wall / max(1, args.steps), "setup_full_kick_s": t_setup,
                             "run_s": time.perf_counter() - t_all}}
    print(json.dumps(line), flush=True)


def force_errors(box, state, theta, h, N, sel, gd):
    """Kick every particle of `state` (its sinks `sel` marked) with save_force, then compare the
    sinks with the FP64 direct Ewald forces gd (same definitions as the benchmark line's
    force_error)."""
    import cosmictiger_b200 as ct
    from cosmictiger_b200 import ics

    x, y, z, v, r = state
    box.upload(x, y, z, mark_sinks(v, sel), r)
    box.sort_by_rung(0)
    box.tree_create(theta, h, 128)
    box.kick(ct.KickParams.make(theta=theta, h=h, GM=1.0 / N, eta=ics.eta_default(), save_force=True, descending=False, ascending=False))
    out = box.download(forces=True)
    idx = find_sinks(out, len(sel))
    gt = np.stack([out["gx"][idx], out["gy"][idx], out["gz"][idx]], 1).astype(np.float64)
    del out
    err = np.linalg.norm(gt - gd, axis=1) / np.linalg.norm(gd, axis=1)
    return {"rms": float(np.sqrt(np.sum((gt - gd) ** 2) / np.sum(gd ** 2))), "rms_per_particle": float(np.sqrt(np.mean(err ** 2))),
            "p99_per_particle": float(np.percentile(err, 99))}


def timed_steps(torch, ctx, box, theta, h, N, steps, lib_stream):
    """Device time of `steps` all-particle steps (tree build, kick, drift) after one warm-up."""
    import cosmictiger_b200 as ct
    from cosmictiger_b200 import ics

    def step(first):
        box.tree_create(theta, h, 128)
        box.kick(ct.KickParams.make(theta=theta, h=h, GM=1.0 / N, eta=ics.eta_default(), t0=1.0 / 64, first_call=first, save_force=False))
        box.drift(0, 1.0, 1.0 / 64)

    step(True)
    ctx.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(lib_stream)
    for i in range(steps):
        step(False)
    e1.record(lib_stream)
    ctx.synchronize()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def study_precision(args, torch):
    """Precision study (the clustered generator with a varied seed): theta in {0.4, 0.55, 0.7} x
    expansion order in {5, 7} x compensated / plain FP32 P2P sums; force error against the
    FP64 direct Ewald sum on seeded sinks and particle-steps/s of the all-particles step."""
    import cosmictiger_b200 as ct
    from cosmictiger_b200 import ics

    state = make_ics(args, seed=args.study_seed)
    N = len(state[0])
    h = ics.softening(N, 0.02)
    nsink = args.accuracy_sinks if args.accuracy_sinks > 0 else 1000
    sel = np.sort(np.random.default_rng(4321).choice(N, size=min(nsink, N), replace=False))
    rows = []
    gd = None
    for order in (5, 7):
        ctx = ct.Context(order=order)
        lib_stream = torch.cuda.ExternalStream(ctx.lib.ct_stream(ctx.h))
        box = ctx.box(N)
        if gd is None:
            # the FP64 direct Ewald forces on the sinks, once (positions are the same in every run)
            box.upload(*state)
            dg = box.direct_ewald(state[0][sel], state[1][sel], state[2][sel], h)
            gd = np.stack(dg[:3], 1) / N
        for theta in (0.4, 0.55, 0.7):
            for comp in (True, False):
                ctx.set_compensated(comp)
                box.upload(*state)
                box.sort_by_rung(0)
                ms = timed_steps(torch, ctx, box, theta, h, N, 2, lib_stream)
                err = force_errors(box, state, theta, h, N, sel, gd)
                row = {"order": order, "theta": theta, "summation": "compensated" if comp else "plain", "ms_per_step": ms,
                       "particle_steps_s": N / (ms / 1e3), **err}
                rows.append(row)
                print(json.dumps(row), flush=True)
        box.close()
        ctx.close()
    return {"study": "precision", "workload": workload_name(args).replace("4-rung hierarchical steps", "all particles per step") + ", seed %d" % args.study_seed,
            "particles": N, "sinks": nsink, "rows": rows}


def study_ensemble(args, torch):
    """512 independent boxes, n_i log-uniform in [16, 128], own Zel'dovich fields, theta 0.55,
    20 steps (the --ensemble-* defaults, or the sizes given): one batched ensemble vs the plain
    single-box path launched box by box, without the benchmark line around it."""
    import cosmictiger_b200 as ct

    ctx = ct.Context(order=7)
    lib_stream = torch.cuda.ExternalStream(ctx.lib.ct_stream(ctx.h))
    res = ensemble_compare(ct, torch, ctx, args, args.theta, lib_stream)
    ctx.close()
    return {"study": "ensemble", **res}


def study_serving(args, torch):
    """Continuous batching: open-loop Poisson arrivals of requests for boxes of n^3 particles, n
    log-uniform in [32, 256], 1-16 steps each, admission by a 150 GB device-memory budget; a sweep
    of arrival rates up to and above saturation, each against the same requests served one at a
    time in arrival order.  The server runs --serving-lanes lanes (contexts with their own
    streams, each driven by its own host thread)."""
    import cosmictiger_b200 as ct
    from cosmictiger_b200 import serving

    lanes = [ct.Context(order=7) for _ in range(max(1, args.serving_lanes))]
    ctx = lanes[0]
    count = args.serving_requests
    states = {}
    out = []
    for rate in (1.0, 2.0, 4.0, 8.0, 16.0):
        reqs = serving.poisson_requests(count, rate=rate, nmin=32, nmax=256, smin=1, smax=16, seed=args.study_seed)
        for r in reqs:
            if r.rid not in states:
                states[r.rid] = serving.request_state(r)
        srv = serving.Server(lanes, theta=args.theta, hbm_budget=150e9, big_total=args.serving_big_total or None)
        done = srv.run(reqs, states)
        s_b = serving.summarize(done)
        seq = serving.poisson_requests(count, rate=rate, nmin=32, nmax=256, smin=1, smax=16, seed=args.study_seed)
        s_p = serving.summarize(serving.run_sequential(ctx, seq, states, theta=args.theta))
        row = {"rate_per_s": rate, "requests": count, "lanes": len(lanes), "big_total": args.serving_big_total or None, "batched": s_b, "sequential": s_p, "ticks": srv.ticks,
               "throughput_ratio": s_b["particle_steps_s"] / s_p["particle_steps_s"], "p99_ratio": s_b["p99_ms"] / s_p["p99_ms"]}
        out.append(row)
        print(json.dumps(row), flush=True)
    for c in lanes:
        c.close()
    return {"study": "serving", "n_range": [32, 256], "steps_range": [1, 16], "hbm_budget_gb": 150, "lanes": len(lanes), "rows": out}


def study_lightcone(args, torch):
    """Drift with the lightcone capture (cuda_drift with do_lc) on the benchmark box, every
    particle on rung 0: plain drift vs drift + capture per call (CUDA events on the library's
    stream; the capture's call includes its read-back of the entry count), entries per drift,
    and the HBM rate of the capture against the measured copy bandwidth (algorithmic bytes:
    37 per particle (positions and velocities read, rung read, positions written) + 28 per
    entry).  The observer's cone sweeps a shell at distance about tau_max - tau (tau_max 1.6,
    drifts of dt 0.005 from tau 0.7, so the shell sits near radius 0.9)."""
    import cosmictiger_b200 as ct
    from tests import oracle_lib

    state = make_ics(args, seed=args.study_seed)
    x, y, z, v, _ = state
    N = len(x)
    r0 = np.zeros(N, np.int8)
    ctx = ct.Context(order=7)
    lib_stream = torch.cuda.ExternalStream(ctx.lib.ct_stream(ctx.h))
    box = ctx.box(N)
    box.upload(x, y, z, v, r0)
    dt, tau_max, K = 0.005, 1.6, 10
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)

    def timed(fn):
        ms = []
        for i in range(3 + K):
            ctx.synchronize()
            e0.record(lib_stream)
            fn(i)
            e1.record(lib_stream)
            ctx.synchronize()
            torch.cuda.synchronize()
            # the entries are handed over after every drift (the reference flushes its lists
            # to the lightcone store each drift); here they are only dropped, untimed
            box.lightcone_clear()
            if i >= 3:
                ms.append(e0.elapsed_time(e1))
        return float(np.median(ms))

    ms_plain = timed(lambda i: box.drift(0, 1.0, dt))
    rows = []
    hbm = peaks_hbm()
    for nside in (64, 4096):
        counts = []

        def lc(i):
            tau0 = 0.7 + dt * i
            counts.append(box.drift_lightcone(0, 1.0, dt, tau0, tau0 + dt, tau_max, nside))

        ms = timed(lc)
        ent = float(np.mean(counts[3:]))
        gbs = (37.0 * N + 28.0 * ent) / (ms / 1e3) / 1e9
        rows.append({"nside": nside, "ms_per_drift": ms, "entries_per_drift": ent, "particles_s": N / (ms / 1e3), "achieved_gbs": gbs,
                     "hbm_peak_gbs": hbm, "frac": gbs / hbm if hbm else None})
        print(json.dumps(rows[-1]), flush=True)
    box.close()
    ctx.close()
    # the CPU oracle (one thread) on the first 2^20 particles
    O = oracle_lib.load(build=False)
    m = min(N, 1 << 20)
    xs, ys, zs, vs = (np.ascontiguousarray(q[:m]).copy() for q in (x, y, z, v))
    t = time.perf_counter()
    ent = O.drift_lc(xs, ys, zs, vs, r0[:m].copy(), 0, 1.0, dt, 0.7, 0.7 + dt, tau_max, 64)
    cpu_s = time.perf_counter() - t
    return {"study": "lightcone", "workload": workload_name(args).replace("4-rung hierarchical steps", "drift of every particle") + ", seed %d" % args.study_seed,
            "particles": N, "dt": dt, "tau_max": tau_max, "plain_drift_ms": ms_plain, "plain_particles_s": N / (ms_plain / 1e3), "rows": rows,
            "cpu_baseline": {"value": m / cpu_s, "unit": "particles/s", "cores": 1, "kind": "port", "sample": "%d particles, %d entries" % (m, len(ent))}}


def study_fourier(args, torch):
    """The IC generator and the power spectrum on an n^3 grid (default 256^3, box 500 Mpc, a
    synthetic power.init-style table cut off at half the grid's Nyquist wavenumber): device time
    per call (CUDA events on the library's stream around ct_initialize / ct_power_spectrum,
    median of 5 after 2 warm-ups), particles per second, and the numpy restatement on 64^3 as
    the CPU baseline (double-precision transforms, one process)."""
    import cosmictiger_b200 as ct
    from cosmictiger_b200 import ics

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import fourier_oracle as F

    N, box = args.n, 500.0
    cosmo = dict(omega_m=0.3111, z0=49.0, hubble=0.6732, sigma8=0.8607, H0=1.0)
    k, P = ics.power_law_table(kcut=0.5 * np.pi * N / box / cosmo["hubble"])
    ctx = ct.Context(order=7)
    lib_stream = torch.cuda.ExternalStream(ctx.lib.ct_stream(ctx.h))
    b = ctx.box(N ** 3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)

    def timed(fn):
        ms = []
        for i in range(7):
            ctx.synchronize()
            e0.record(lib_stream)
            fn()
            e1.record(lib_stream)
            ctx.synchronize()
            torch.cuda.synchronize()
            if i >= 2:
                ms.append(e0.elapsed_time(e1))
        return float(np.median(ms))

    rows = {}
    for tw in (False, True):
        ms = timed(lambda: b.initialize(N, box, k, P, twolpt=tw, **cosmo))
        rows["initialize_2lpt" if tw else "initialize_zeldovich"] = {"ms": ms, "particles_s": N ** 3 / (ms / 1e3)}
    ms = timed(lambda: b.power_spectrum(N, box, 1))
    rows["power_spectrum"] = {"ms": ms, "particles_s": N ** 3 / (ms / 1e3)}
    b.close()
    ctx.close()
    for key, r in rows.items():
        print(json.dumps({key: r}), flush=True)
    m = 64
    km, Pm = ics.power_law_table(kcut=0.5 * np.pi * m / box / cosmo["hubble"])
    t = time.perf_counter()
    x, y, z, _, _ = F.initialize(m, box, cosmo["omega_m"], cosmo["z0"], cosmo["hubble"], cosmo["sigma8"], cosmo["H0"], km, Pm, True)
    t_ic = time.perf_counter() - t
    t = time.perf_counter()
    F.power_spectrum(x, y, z, m, 1, box)
    t_ps = time.perf_counter() - t
    return {"study": "fourier", "grid": N, "particles": N ** 3, "box_mpc": box, "rows": rows,
            "cpu_baseline": {"initialize_2lpt_particles_s": m ** 3 / t_ic, "power_spectrum_particles_s": m ** 3 / t_ps, "unit": "particles/s",
                             "cores": 1, "kind": "port", "sample": "numpy restatement on %d^3" % m}}


def study_autotune(args, torch):
    """The autotuner's joint search (leaf size x launch shape) on the benchmark box (clustered,
    n^3, theta 0.55) and on a batched ensemble of the C4 kind (boxes of 16^3..128^3); every
    candidate's device time and force difference from the default (leaf 128, shape 128/1/32)."""
    import cosmictiger_b200 as ct
    from cosmictiger_b200 import autotune, ics

    out = {}
    ctx = ct.Context(order=7)
    state = make_ics(args, seed=3)
    N = len(state[0])
    res = autotune.tune(ctx, state, theta=args.theta, h=ics.softening(N, 0.02), buckets=(64, 96, 128, 160, 192), max_force_rms=None, repeats=2)
    out["single_box"] = {"workload": workload_name(args).replace("4-rung hierarchical steps", "all-particles kick"), **res}
    print(json.dumps({"single_box_best": res["best"], "reference": res["reference"]}), flush=True)
    nb = args.ensemble_boxes if args.ensemble_boxes != 512 else 128
    sets = make_ensemble(nb, 16, 128, seed=4)
    counts = [len(s[0]) for s in sets]
    cat = [np.concatenate([s[k] for s in sets]) for k in range(5)]
    hs = np.array([ics.softening(n, 0.02) for n in counts], np.float32)
    gms = np.array([1.0 / n for n in counts], np.float32)

    def factory():
        e = ctx.ensemble(counts)
        e.upload(*cat)
        e.set_box_params(hs, gms)
        return e

    res2 = autotune.tune(ctx, cat, theta=args.theta, h=float(hs.max()), buckets=(64, 96, 128, 160, 192), max_force_rms=None, repeats=2,
                         box_factory=factory)
    out["ensemble"] = {"boxes": nb, "particles": int(sum(counts)), "n_range": [16, 128], **res2}
    print(json.dumps({"ensemble_best": res2["best"], "reference": res2["reference"]}), flush=True)
    ctx.close()
    return {"study": "autotune", **out}


def peaks_hbm():
    try:
        with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"])
    except (OSError, KeyError, ValueError):
        return None


def run_study(args):
    import torch

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    fn = {"precision": study_precision, "ensemble": study_ensemble, "serving": study_serving, "lightcone": study_lightcone, "fourier": study_fourier,
          "autotune": study_autotune}[args.study]
    t = time.perf_counter()
    res = fn(args, torch)
    res["wall_s"] = time.perf_counter() - t
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
