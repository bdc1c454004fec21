"""Benchmark of the multi-block D2Q9 BGK step (MLUPS, % HBM roofline).

Workload: the 3-level cylinder at Re=100, 4096x1024 coarse cells, level-1 box
[768,1280]x[384,640], level-2 box [896,1152]x[448,576], D=32 at (960,512),
U0=0.04 (6,986,527 cell updates per coarse step), FP32 storage of f - w.
A step is one coarse time step of evolution() over all levels.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torchrun, one process per GPU, each GPU advancing its own
independent case (weak scaling, no data-path collective).  Rank 0 prints one
JSON line.  --impl reference times the reference program's own CUDA build
(oracle/_ref/ref_c2: its kernels compiled unmodified, FP64) on the same
workload; when that binary is absent it times the FP64 C oracle on the host.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "multi-block-lbm-gpu_b200"))

METRIC = "multi-block D2Q9 MLUPS & % HBM roofline; time-to-Cd (±0.5%) vs plain FP32"
WORKLOAD = "3-level cylinder Re=100, 4096x1024 coarse, L1 box 512x256, L2 box 256x128 coarse, D=32"
BYTES_PER_UPDATE = {"f32": 72, "f32u": 72, "f16s": 36, "f16c": 36, "f64": 144}


def peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def dram_traffic_per_launch(prec):
    """dram__bytes_read.sum + dram__bytes_write.sum of one level-0 block-step
    launch, from the committed ncu summary (None when absent)."""
    path = os.path.join(REPO, "profiles", f"block_step_L0_config2_{prec}.md")
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_launch_full:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


class Clocks:
    """nvidia-smi sampling (200 ms) while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                v = [x.strip() for x in line.split(",")]
                if len(v) >= 9 and v[1].isdigit():
                    rows.append(v)
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [int(r[1]) for r in rows]
        loaded = [int(r[1]) for r in rows if float(r[3]) > 300] or sm
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for n, val in zip(names, r[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": int(rows[0][2]), "reasons": sorted(reasons),
                "samples": len(rows)}


def cpu_baseline(budget_s=12.0):
    """The FP64 C oracle (OpenMP over all host cores) on the same workload,
    bounded to about budget_s seconds of coarse steps."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import mblbm
    import oracle

    g = mblbm.config2_geometry()
    oracle.set_threads(os.cpu_count())
    o = oracle.Oracle(g)
    o.init()
    o.evolution(1)
    t0 = time.perf_counter()
    n = 0
    while True:
        o.evolution(1)
        n += 1
        if time.perf_counter() - t0 > budget_s or n >= 400:
            break
    dt = time.perf_counter() - t0
    upd = mblbm.updates_per_coarse_step(g)
    o.close()
    return {"value": round(upd * n / dt / 1e6, 2), "unit": "MLUPS", "cores": os.cpu_count(), "kind": "port",
            "sample": f"{n} coarse steps of the same workload after 1 warm-up step ({dt:.1f} s), FP64 C oracle, OpenMP"}


# Cell updates of one coarse step of WORKLOAD: level 0 has 4,079,875 cells in
# 4 blocks (1 sub-step), level 1 401,676 cells in 4 blocks (2 sub-steps),
# level 2 525,825 cells in 1 block (4 sub-steps).  The product arm counts it
# from its geometry (mblbm.updates_per_coarse_step); the reference binary
# prints it from its own AREA table (sum over blocks of nx*ny*m).
UPDATES_PER_STEP = 6986527
L2_NOTE = "working set larger than L2 (5.1M cells: 370 MB of FP32 state buffers, 740 MB in FP64); no flush"


def bench_config(world):
    """The `config` object of both arms (the compute precision is `dtype`)."""
    return {"workload": WORKLOAD, "cell_updates_per_step": UPDATES_PER_STEP, "l2": L2_NOTE,
            "parallelism": f"{world} independent cases, one per GPU"}


def level0_in_step(sim, stream):
    """(kernel, mean ms, algorithmic bytes) of level 0's interior block-step
    launches inside one replayed plan of `period` coarse steps, from the
    CUPTI kernel records of torch.profiler (outside any timed region); None
    when the profiler records no such kernel."""
    import torch
    from torch.profiler import ProfilerActivity, profile

    n = 13  # one plan of 6 steps twice, then single steps
    sim.prepare(n)
    torch.cuda.synchronize()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        sim.evolution(n, stream)
        torch.cuda.synchronize()
    durs = {}
    for e in prof.events():
        nm = e.name
        interior = "block_step_q<" in nm or ("block_step_p<" in nm and ", true>" in nm) or \
            ("block_step_r<" in nm and ", true>" in nm) or "block_step_tb<" in nm
        if e.device_type == torch.autograd.DeviceType.CUDA and interior:
            durs.setdefault(e.name.split("(")[0], []).append((e.time_range.end - e.time_range.start) / 1e3)
    if not durs:
        return None
    name, d = max(durs.items(), key=lambda kv: len(kv[1]))
    geo = sim.geo
    # the interior (distance >= 2 from the block edges) of the level-0 blocks
    cells = sum((geo.Areas[a].nx - 4) * (geo.Areas[a].ny - 4) for a in range(geo.layout.ASP[0], geo.layout.ASP[1]))
    return name, float(sum(d) / len(d)), float(BYTES_PER_UPDATE[sim.precision]) * cells


def step_timeline(sim, stream, n=48):
    """CUPTI kernel records (torch.profiler) of an n-step call after 30 warm-up
    steps: every launch of the two coarse steps that start at the 21st
    level-0 interior launch, as (start us from that launch, duration us,
    kernel), and the period and duration of the interior launches around it."""
    import torch
    from torch.profiler import ProfilerActivity, profile

    sim.evolution(30, stream)
    sim.prepare(n)
    torch.cuda.synchronize()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        sim.evolution(n, stream)
        torch.cuda.synchronize()
    ev = sorted((e.time_range.start, e.time_range.end, e.name.split("(")[0].replace("void mblbm::dev::", ""))
                for e in prof.events() if e.device_type == torch.autograd.DeviceType.CUDA)
    ints = [e for e in ev if ("block_step_p<" in e[2] and ", true>" in e[2]) or "block_step_q<" in e[2]
            or ("block_step_r<" in e[2] and ", true>" in e[2]) or "block_step_tb<" in e[2] or "block_step_o<" in e[2]]
    if len(ints) < 24:
        return None
    t0, t1 = ints[20][0], ints[22][0]
    return {"launches": [(round(a - t0, 1), round(b - a, 1), nm) for a, b, nm in ev if t0 - 5 <= a < t1 + 5],
            "interior_period_us": [round(ints[i + 1][0] - ints[i][0], 1) for i in range(18, 23)],
            "interior_us": [round(e[1] - e[0], 1) for e in ints[18:23]]}


def run_reference(args):
    """The reference's own CUDA build (oracle/_ref/ref_c2) on WORKLOAD.  Loads
    nothing of this repository's library: the update count comes from the
    reference binary itself."""
    exe = os.path.join(REPO, "oracle", "_ref", "ref_c2")
    base = {"metric": METRIC, "unit": "MLUPS", "impl": "reference", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "data": "synthetic",
            "config": bench_config(1)}
    js, why = None, "reference build absent (oracle/_ref/ref_c2)"
    if os.path.exists(exe):
        wd = tempfile.mkdtemp()
        try:
            r = subprocess.run([exe, "bench", str(args.steps), str(args.warmup)], cwd=wd, capture_output=True,
                               text=True, timeout=1800)
        except subprocess.TimeoutExpired:
            r, why = None, "reference build did not finish within 1800 s"
        if r is not None:
            lines = r.stdout.strip().splitlines()
            try:
                js = json.loads(lines[-1]) if r.returncode == 0 and lines else None
            except ValueError:
                js = None
            if js is None:
                err = (r.stderr.strip().splitlines() or ["no output"])[-1]
                why = f"reference build failed (exit {r.returncode}): {err[:200]}"
    if js is not None:
        upd = int(js["cell_updates_per_step"])
        if upd != UPDATES_PER_STEP:
            raise RuntimeError(f"reference build counts {upd} cell updates per step, expected {UPDATES_PER_STEP}")
        v = upd / js["ms_per_step"] / 1e3
        ve = upd / js["ms_per_step_diag"] / 1e3
        base.update(value=round(v, 2), ms_per_step=js["ms_per_step"], dtype="f64",
                    e2e={"value": round(ve, 2), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                         "what": "the reference's shipped loop: evolution + error_L2 + getDrag_block every step"},
                    cpu_baseline={"value": round(v, 2), "unit": "MLUPS", "cores": 1, "kind": "reference",
                                  "sample": f"reference CUDA build (kernels and host code unmodified, FP64, nvcc -arch=sm_100a) "
                                            f"on cuda:0, {args.steps} timed coarse steps after {args.warmup}"})
    else:  # the FP64 C oracle on the host cores stands in for the reference build
        cb = cpu_baseline()
        base.update(value=cb["value"], ms_per_step=round(UPDATES_PER_STEP / cb["value"] / 1e3, 4), dtype="f64",
                    cpu_baseline=cb, note=why,
                    e2e={"value": cb["value"], "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
    print(json.dumps(base), flush=True)


def run_batch(args):
    """The batched workload: 256 independent cases drawn by mblbm.batch_case
    (seeded per case), grouped by level count into two batches, each
    autotuned, then K coarse steps of both timed together with CUDA events.
    Under torchrun the cases are sharded over the ranks by cost (cell updates
    per coarse step, mblbm.ranks.balance); ranks exchange nothing while they
    step, only the slowest rank's time and the total updates."""
    import torch
    import mblbm
    from mblbm import ranks

    rank, world, local = ranks.env()
    torch.cuda.set_device(local)
    dist = ranks.init("nccl") if world > 1 else None
    stream = torch.cuda.Stream()
    t_setup = time.perf_counter()
    drawn = [mblbm.batch_case(i) for i in range(args.cases)]
    costs = [mblbm.updates_per_coarse_step(g) for g, _ in drawn]
    mine = ranks.balance(costs, rank, world)
    groups = {2: [], 3: []}
    for i in mine:
        g, prm = drawn[i]
        sim = mblbm.MultiBlockLBM(g, args.precision)
        sim.init(stream)
        groups[prm["levels"]].append(sim)
    batches = [mblbm.Batch(v) for v in groups.values() if v]
    tune = [b.autotune(steps=6, stream=stream) for b in batches]
    upd = sum(b.stats()["updates_per_step"] for b in batches)
    for b in batches:
        b.evolution(args.warmup, stream)
        b.prepare(args.steps)  # plans and graphs of the timed call, compiled outside the timed region
    torch.cuda.synchronize()
    t_setup = time.perf_counter() - t_setup

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        barrier()
        e0.record(stream)
        for b in batches:
            b.evolution(args.steps, stream)
        e1.record(stream)
        barrier()
    ms = e0.elapsed_time(e1)
    kernels = sum(b.stats()["kernels_last_call"] for b in batches)
    cds = [b.drag(stream)[0] for b in batches]
    # per-case Cd against the single-case solver: a few cases of each batch
    # stepped alone from rest for as many coarse steps as the batch took
    check = []
    for b, sims in zip(batches, [v for v in groups.values() if v]):
        done = b.stats()["steps_done"]
        cd_b = b.drag(stream)[0]
        for q in sorted({0, len(sims) // 2, len(sims) - 1})[: args.cd_check]:
            one = mblbm.MultiBlockLBM(sims[q].geo, args.precision)
            one.init(stream)
            one.evolution(done, stream)
            cd1 = one.getDrag_block(stream)[2]
            check.append(abs(float(cd_b[q]) / cd1 - 1.0) if cd1 != 0 else abs(float(cd_b[q])))
            one.close()
    cd_lo = min(float(c.min()) for c in cds) if cds else float("inf")
    cd_hi = max(float(c.max()) for c in cds) if cds else float("-inf")
    ms, = ranks.reduce([ms], "max", dist, device="cuda")
    tot_upd, tot_kernels = ranks.reduce([upd, kernels], "sum", dist, device="cuda")
    if rank == 0:
        peak, src = peaks()
        bpu = BYTES_PER_UPDATE[args.precision]
        achieved = tot_upd * args.steps * bpu / (ms * 1e-3) / 1e9
        line = {"metric": METRIC, "value": round(tot_upd * args.steps / (ms * 1e-3) / 1e6, 1), "unit": "MLUPS",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 5),
                "higher_is_better": True, "scaling": "strong" if world > 1 else "weak", "vs_baseline": None,
                "dtype": args.precision, "data": "synthetic",
                "config": {"workload": f"batched: {args.cases} cases, D~U[10,40], aspect~U[1,3], angle~U[0,pi), "
                                       "Re~U[20,200], domain 20Dx8D, U0=0.04, 2 or 3 levels, splitmix64 seed 20250+case",
                           "batches_rank0": {f"{len(v)} cases of {lv} levels": t for (lv, v), t in
                                             zip([(lv, v) for lv, v in groups.items() if v], tune)},
                           "cell_updates_per_step": int(tot_upd), "setup_s": round(t_setup, 1),
                           "parallelism": f"{args.cases} cases sharded by cost over {world} GPU(s)"},
                "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                             "frac": round(achieved / peak, 4), "traffic": None, "peak_source": src,
                             "kernel": "whole batched step (all launches)", "bytes_per_update": bpu},
                "gpu_launches": int(tot_kernels), "clocks": clk.summary(),
                "cd_range_rank0": [round(cd_lo, 4), round(cd_hi, 4)],
                "cd_vs_single_case_rank0": {"cases": len(check), "max_rel_diff": max(check) if check else None}}
        print(json.dumps(line), flush=True)
    for b in batches:
        b.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_timetocd(args):
    """Convergence of Cd on the 2-level case (400x160 coarse, Re=40, steady):
    the FP64 value after --steps coarse steps is the converged reference; for
    FP32 and FP16 storage, the first step after which Cd stays within 0.5 %
    of it, and the device time to get there (diagnostics every step)."""
    import torch
    import mblbm

    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    geo = mblbm.config1_geometry()
    upd = mblbm.updates_per_coarse_step(geo)
    out = {}
    series = {}
    for prec in ("f64", "f32", "f16s", "f16c"):
        sim = mblbm.MultiBlockLBM(geo, prec)
        sim.init(stream)
        if args.bc == "channel":  # free-slip top and bottom, half-way bounce-back on the cylinder
            mblbm.channel_walls(sim, geo)
        sim.init(stream)
        sim.prepare_diag(args.steps)  # plans, graphs and result buffers of the timed call
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        cd, cl, l2 = sim.evolution_diag(args.steps, stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        series[prec] = (cd, ms)
        sim.close()
    ref = float(series["f64"][0][-1])
    for prec, (cd, ms) in series.items():
        n = mblbm.settle_step(cd, ref)
        out[prec] = {"cd_final": round(float(cd[-1]), 6), "rel_to_f64": float(cd[-1] / ref - 1.0),
                     "steps_to_cd": n, "ms_to_cd": round(ms * n / args.steps, 2),
                     "ms_per_step_with_diag": round(ms / args.steps, 5)}
    line = {"metric": "time to Cd within 0.5% of the converged FP64 value", "unit": "ms", "higher_is_better": False,
            "value": out["f32"]["ms_to_cd"], "n_gpus": 1, "steps": args.steps, "warmup": 12, "data": "synthetic",
            "config": {"workload": "2-level cylinder Re=40, 400x160 coarse, fine box [60,140]x[40,120], D=20, U0=0.05",
                       "boundaries": ("free-slip top and bottom, half-way bounce-back cylinder" if args.bc == "channel"
                                      else "the reference's: equilibrium domain edges, on-node bounce-back cylinder"),
                       "cell_updates_per_step": upd, "reference": "Cd of FP64 storage after the run"},
            "dtype": "f32", "by_precision": out}
    print(json.dumps(line), flush=True)
    return 0


def run_warmstart(args):
    """The learned warm start (config 5): surrogate trained on --cases solver
    snapshots of the batched workload's distribution (after --snap-per-d x D
    coarse steps from rest), evaluated on --eval held-out cases.  Each
    held-out case runs --eval-per-d x D coarse steps twice as batches: plain
    FP32 from rest (cold) and, from the surrogate, FP16-shifted (warm;
    --warm-precision f32 isolates the surrogate from the storage precision).  Cd is
    sampled every 50 steps; its running mean (500 steps for steady cases,
    Re < 47; 150 D steps, at least one shedding period, otherwise) must
    settle within 0.5 % of the cold run's final running mean.  A warm start
    whose final running mean differs from the cold one by more than 0.5 %, or
    (shedding cases) whose Strouhal number over the second half of the run
    differs from the cold one's by more than 1 %, is rejected and its case
    counted at the cold start's time (fallback)."""
    import numpy as np
    import torch
    import mblbm
    from mblbm import surrogate as sg

    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    x, t, m, ids = sg.generate(range(args.cases), args.snap_per_d, "f32")
    t_data = time.perf_counter() - t0
    X, T, M = (torch.from_numpy(a).cuda() for a in (x, t, m))
    net = mblbm.UNet(sg.H, sg.W, max_batch=16, seed=1)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    hist = sg.train(net, X, T, M, epochs=args.epochs, batch=16, lr=1e-3)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t1
    n_steps_train = args.epochs * (len(ids) // 16)
    gflop_step = 16 * 3 * unet_gflop(sg.H, sg.W)
    eval_ids = list(range(100000, 100000 + args.eval))
    chunk = 50
    cold, tc = sg.drag_series(eval_ids, args.eval_per_d, "f32", chunk)
    t2 = time.perf_counter()
    warm, tw = sg.drag_series(eval_ids, args.eval_per_d, args.warm_precision, chunk, net=net, kick=args.kick)
    t_warm_total = time.perf_counter() - t2
    res = []
    for i in eval_ids:
        sc, prm, key, lc = cold[i]
        sw, lw = warm[i][0], warm[i][3]
        win = 10 if prm["Re"] < sg.RE_SHEDDING else max(10, int(np.ceil(150 * prm["D"] / chunk)))
        kern = np.ones(win) / win
        rc, rw = np.convolve(sc, kern, "valid"), np.convolve(sw, kern, "valid")
        ref = rc[-1]
        nc, nw = mblbm.settle_step(rc, ref), mblbm.settle_step(rw, ref)
        ok = abs(rw[-1] / ref - 1.0) <= 0.005
        # shedding cases: the Strouhal number of the second half of the run
        # (lift sampled every `chunk` steps) must also agree within 1 %
        st_c = st_w = None
        if prm["Re"] >= sg.RE_SHEDDING:
            half = len(lc) // 2
            st_c = mblbm.strouhal(lc, prm["D"], 0.04 * chunk, skip=half)
            st_w = mblbm.strouhal(lw, prm["D"], 0.04 * chunk, skip=half)
            if st_c is not None and (st_w is None or abs(st_w / st_c - 1.0) > 0.01):
                ok = False
        steps_c, steps_w = (nc + win) * chunk, (nw + win) * chunk
        res.append({"case": i, "Re": round(prm["Re"], 1), "D": round(prm["D"], 1), "cd": round(float(ref), 4),
                    "st_cold": None if st_c is None else round(st_c, 4),
                    "st_warm": None if st_w is None else round(st_w, 4),
                    "cold_steps": steps_c, "warm_steps": steps_w, "accepted": bool(ok),
                    "ms_cold": steps_c * tc[key], "ms_warm": steps_w * tw[key] if ok else steps_c * tc[key]})
    acc = [r for r in res if r["accepted"]]
    ratio = sum(r["ms_warm"] for r in res) / sum(r["ms_cold"] for r in res)
    steady = [r for r in res if r["Re"] < sg.RE_SHEDDING]
    shedding = [r for r in res if r["Re"] >= sg.RE_SHEDDING]
    line = {"metric": "time to Cd within 0.5% (warm start vs plain FP32 cold start)", "unit": "ratio",
            "higher_is_better": False, "value": round(ratio, 4), "n_gpus": 1, "data": "synthetic",
            "dtype": f"bf16 surrogate, {args.warm_precision} warm / f32 cold solver",
            "config": {"workload": "held-out cases of the batched distribution (mblbm.batch_case ids 100000+)",
                       "train_cases": len(ids), "snap_steps_per_D": args.snap_per_d, "epochs": args.epochs,
                       "eval_cases": len(res), "eval_steps_per_D": args.eval_per_d, "cd_sample_every": chunk,
                       "kick": args.kick},
            "accepted": len(acc),
            "steady_cases": len(steady),
            "steady_ratio": round(sum(r["ms_warm"] for r in steady) / max(1e-9, sum(r["ms_cold"] for r in steady)), 4),
            "shedding_ratio": round(sum(r["ms_warm"] for r in shedding) / max(1e-9, sum(r["ms_cold"] for r in shedding)), 4),
            "median_cold_steps": float(np.median([r["cold_steps"] for r in res])),
            "median_warm_steps_accepted": float(np.median([r["warm_steps"] for r in acc])) if acc else None,
            "loss_first_last": [round(hist[0], 5), round(hist[-1], 5)], "train_s": round(t_train, 1),
            "data_s": round(t_data, 1), "warm_eval_host_s": round(t_warm_total, 1),
            "train_tflops": round(n_steps_train * gflop_step / t_train / 1e3, 1),
            "cases": res}
    print(json.dumps(line), flush=True)
    net.close()
    return 0


def run_forces(args):
    """Config 2's flow outputs: the 3-level cylinder at Re=100 run for --steps
    coarse steps from rest with Cd and Cl recorded every step (mb_step_diag);
    mean Cd, rms Cl and the Strouhal number over the second half of the run."""
    import numpy as np
    import torch
    import mblbm

    torch.cuda.set_device(0)
    geo = mblbm.config2_geometry()
    if args.spinup > 0:
        return run_forces_developed(args, geo)
    sim = mblbm.MultiBlockLBM(geo, args.precision)
    sim.init()
    cd, cl = [], []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    chunk = 5000
    for q in range(0, args.steps, chunk):
        a, b, _ = sim.evolution_diag(min(chunk, args.steps - q))
        cd.append(a)
        cl.append(b)
    e1.record()
    torch.cuda.synchronize()
    cd, cl = np.concatenate(cd), np.concatenate(cl)
    half = len(cd) // 2
    c = geo.config
    D, U0 = 2.0 * c.R, c.U0[0]
    st = mblbm.strouhal(cl, D, U0, skip=half)
    line = {"metric": "mean Cd, rms Cl, Strouhal number", "unit": "dimensionless", "n_gpus": 1, "steps": args.steps,
            "data": "synthetic", "dtype": args.precision,
            "config": {"workload": WORKLOAD, "statistics_over": f"coarse steps {half}..{len(cd) - 1}"},
            "mean_cd": round(float(cd[half:].mean()), 5), "rms_cl": round(float(np.sqrt(np.mean(cl[half:] ** 2))), 5),
            "strouhal": None if st is None else round(float(st), 5),
            "cd_last": round(float(cd[-1]), 5), "cl_last": round(float(cl[-1]), 5),
            "max_abs_cl": round(float(np.abs(cl[half:]).max()), 5), "device_s": round(e0.elapsed_time(e1) / 1e3, 2)}
    print(json.dumps(line), flush=True)
    if args.save:
        np.save(os.path.join(args.save, f"forces_{args.precision}.npy"), np.stack([cd, cl]))
    sim.close()
    return 0


def run_forces_developed(args, geo):
    """The storage precisions on developed shedding: FP64 storage runs
    --spinup coarse steps from rest (past the onset of shedding, which the
    symmetric start delays by tens of thousands of steps), then its fields
    (rho, u, F of every block) seed one context per precision, whose ring
    slots and u_prev are rebuilt from them (mb_sync_history); each runs
    --steps more coarse steps with Cd and Cl every step.  Mean Cd, rms Cl and
    St over those steps, and their relative differences to FP64's."""
    import numpy as np
    import mblbm

    base = mblbm.MultiBlockLBM(geo, "f64")
    base.init()
    for q in range(0, args.spinup, 5000):
        base.evolution_diag(min(5000, args.spinup - q))
    state = [base.fields(a) for a in range(geo.layout.number_area)]
    base.close()
    c = geo.config
    D, U0 = 2.0 * c.R, c.U0[0]
    out = {}
    runs = [("f64", None, None), ("f32", None, None), ("f32", "w", None), ("f16s", None, None),
            ("f16s", "feq0", None), ("f16s", None, "nearest"), ("f16c", None, None), ("f16c", "w", None),
            ("f16c", None, "nearest")]
    for prec, shift, rounding in runs:
        name = prec + ("" if shift is None else f"_{shift}") + {None: "", "nearest": "_rn", "stochastic": "_sr"}[rounding]
        sim = mblbm.MultiBlockLBM(geo, prec, shift=shift, rounding=rounding)
        sim.init()
        for a, f in enumerate(state):
            sim.set_fields(a, f["rho"], f["ux"], f["uy"], f["F"])
        sim.sync_history()
        cd, cl = [], []
        for q in range(0, args.steps, 5000):
            x, y, _ = sim.evolution_diag(min(5000, args.steps - q))
            cd.append(x)
            cl.append(y)
        sim.close()
        cd, cl = np.concatenate(cd), np.concatenate(cl)
        st = mblbm.strouhal(cl, D, U0)
        out[name] = {"mean_cd": float(cd.mean()), "rms_cl": float(np.sqrt(np.mean(cl ** 2))),
                     "strouhal": None if st is None else float(st)}
        if args.save:
            np.save(os.path.join(args.save, f"forces_dev_{name}.npy"), np.stack([cd, cl]))
    for name in out:
        if name == "f64":
            continue
        for k in ("mean_cd", "rms_cl", "strouhal"):
            a, b = out[name][k], out["f64"][k]
            out[name][k + "_rel_f64"] = None if a is None or b is None else a / b - 1.0
    line = {"metric": "mean Cd, rms Cl, Strouhal number on developed shedding, by storage precision",
            "unit": "dimensionless", "n_gpus": 1, "steps": args.steps, "spinup_f64": args.spinup,
            "data": "synthetic", "config": {"workload": WORKLOAD}, "by_precision": out}
    print(json.dumps(line), flush=True)
    return 0


def run_tgv(args):
    """The 2-level periodic Taylor-Green vortex: 1024^2 coarse cells with a
    centred 256^2-cell refined patch (512^2 fine cells), u0 = 0.01, tau = 0.6
    on level 0, --steps coarse steps (5000) in FP64, FP32 and FP16-shifted
    storage: device time, MLUPS, and the vortex amplitude against the exact
    decay u0 exp(-2 nu k^2 t) and against the FP64 run."""
    import numpy as np
    import torch
    import mblbm

    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    geo = mblbm.tgv_geometry(n=1024, patch=256, u0=0.01, tau=0.6, levels=2)
    upd = mblbm.updates_per_coarse_step(geo)
    nu = (geo.Areas[0].tau - 0.5) / 3.0
    k = 2.0 * np.pi / (geo.config.LX - 2)
    out = {}
    for prec in ("f64", "f32", "f16s", "f16c"):
        sim = mblbm.MultiBlockLBM(geo, prec)
        sim.init(stream)
        sim.evolution(args.warmup, stream)  # plans and graphs built before the timed run
        sim.init(stream)
        mblbm.tgv_init(sim, geo)
        a0 = mblbm.tgv_amplitude(sim, geo)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sim.evolution(args.steps, stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        amp = mblbm.tgv_amplitude(sim, geo)
        exact = a0 * np.exp(-2.0 * nu * k * k * args.steps)
        out[prec] = {"amplitude": amp, "rel_to_exact": amp / exact - 1.0, "ms": round(ms, 2),
                     "mlups": round(upd * args.steps / ms / 1e3, 1)}
        sim.close()
    for prec in ("f32", "f16s", "f16c"):
        out[prec]["rel_to_f64"] = out[prec]["amplitude"] / out["f64"]["amplitude"] - 1.0
    line = {"metric": "periodic Taylor-Green vortex: MLUPS and amplitude error after the run", "unit": "MLUPS",
            "value": out["f16s"]["mlups"], "higher_is_better": True, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "data": "synthetic", "dtype": "f16s",
            "config": {"workload": "2-level periodic Taylor-Green vortex, 1024x1024 coarse, 256x256-cell refined "
                                   "patch (512x512 fine cells), u0=0.01, tau=0.6",
                       "cell_updates_per_step": upd, "exact": "u0 exp(-2 nu k^2 t), nu = (tau - 1/2)/3"},
            "by_precision": out}
    print(json.dumps(line), flush=True)
    return 0


def unet_gflop(H, W):
    """Forward GFLOP of the surrogate for one sample (3x3 convolutions)."""
    layers = [(16, 32, 0), (32, 32, 0), (32, 64, 1), (64, 64, 1), (64, 128, 2), (128, 128, 2), (128, 256, 3),
              (256, 256, 3), (384, 128, 2), (128, 128, 2), (192, 64, 1), (64, 64, 1), (96, 32, 0), (32, 32, 0)]
    return sum(2 * 9 * ci * co * (H >> lv) * (W >> lv) for ci, co, lv in layers) / 1e9


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--warmup", type=int, default=12)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="f32", choices=["f32", "f32u", "f16s", "f16c", "f64"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--roofline-only", type=int, default=0, metavar="N",
                    help="init, then N launches of one level's block step alone, replayed twice as one CUDA "
                         "graph (untimed, then timed; an ncu capture of that kernel takes -k regex:k_block_step "
                         "-s 3 with N >= 2); prints its roofline")
    ap.add_argument("--level", type=int, default=0, help="level of --roofline-only")
    ap.add_argument("--timeline", action="store_true",
                    help="print the CUPTI kernel records of two coarse steps (step_timeline) and exit")
    ap.add_argument("--no-in-step", action="store_true",
                    help="leave out the CUPTI record of the level-0 interior inside the step (after the timed "
                         "region; for runs under ncu, which holds CUPTI itself)")
    ap.add_argument("--variant", type=int, default=None, help="block-step variant of every level (mb_set_stb_variant)")
    ap.add_argument("--workload", default="cylinder3",
                    choices=["cylinder3", "batch256", "timetocd", "warmstart", "forces", "tgv"],
                    help="cylinder3: the single 3-level case (default); batch256: the batched form; "
                         "timetocd: Cd convergence of the 2-level case by precision; tgv: the 2-level periodic "
                         "Taylor-Green vortex by precision")
    ap.add_argument("--cases", type=int, default=256, help="cases of --workload batch256 / training cases of warmstart")
    ap.add_argument("--cd-check", type=int, default=3,
                    help="--workload batch256: cases per batch re-run alone to compare Cd with the batch")
    ap.add_argument("--eval", type=int, default=64, help="held-out cases of --workload warmstart")
    ap.add_argument("--snap-per-d", type=float, default=300.0, help="coarse steps per unit D before a training snapshot")
    ap.add_argument("--eval-per-d", type=float, default=900.0, help="coarse steps per unit D of a warm-start evaluation run")
    ap.add_argument("--warm-precision", default="f16s", choices=["f16s", "f16c", "f32"], help="solver storage of warm starts")
    ap.add_argument("--epochs", type=int, default=40, help="training epochs of --workload warmstart")
    ap.add_argument("--kick", type=float, default=0.0,
                    help="--workload warmstart: transverse velocity kick (x U0) behind the obstacle in the warm "
                         "starts of shedding cases (surrogate.warm_start)")
    ap.add_argument("--save", default=None, metavar="DIR", help="--workload forces: write Cd and Cl per step to DIR")
    ap.add_argument("--spinup", type=int, default=0,
                    help="--workload forces: FP64 coarse steps from rest before every precision continues from "
                         "that state for --steps steps")
    ap.add_argument("--bc", default="reference", choices=["reference", "channel"],
                    help="boundaries of --workload timetocd: the reference's, or free-slip top and bottom with a "
                         "half-way bounce-back cylinder")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return 0
    if args.workload == "batch256":
        return run_batch(args)
    if args.workload == "timetocd":
        return run_timetocd(args)
    if args.workload == "warmstart":
        return run_warmstart(args)
    if args.workload == "forces":
        return run_forces(args)
    if args.workload == "tgv":
        return run_tgv(args)

    import torch

    torch.cuda.set_device(local)
    import mblbm
    from mblbm import ranks

    dist = ranks.init("nccl") if world > 1 else None

    geo = mblbm.config2_geometry()
    upd = mblbm.updates_per_coarse_step(geo)
    assert upd == UPDATES_PER_STEP, upd
    stream = torch.cuda.Stream()
    sim = mblbm.MultiBlockLBM(geo, args.precision)
    if args.variant is not None:
        for lvl in range(geo.layout.LEVEL):
            sim.set_stb_variant(lvl, args.variant)
    sim.init(stream)
    if args.timeline:
        print(json.dumps({"precision": args.precision, "timeline": step_timeline(sim, stream)}))
        return 0
    if args.roofline_only:
        kms, kbytes, kcells = sim.time_block_step(args.level, args.roofline_only, stream)
        peak, src = peaks()
        print(json.dumps({"kernel": f"k_block_step level {args.level}", "precision": args.precision,
                          "ms_per_launch": kms, "alg_bytes_per_launch": kbytes, "cells": kcells,
                          "achieved_gbs": kbytes / kms / 1e6, "frac": kbytes / kms / 1e6 / peak,
                          "peak_source": src}))
        return 0
    sim.evolution(args.warmup, stream)
    torch.cuda.synchronize()
    sim.prepare(args.steps)  # plans and graphs of the timed call, compiled outside the timed region

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- timed region: K coarse steps, inputs resident in HBM ---------------
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        barrier()
        e0.record(stream)
        sim.evolution(args.steps, stream)
        e1.record(stream)
        barrier()
    ms = e0.elapsed_time(e1)
    kernels = sim.stats()["kernels_last_call"]

    # ---- dominant kernel alone: level-0 block step, CUDA events on its stream
    kms, kbytes, kcells = sim.time_block_step(0, 50, stream)
    # ---- the same kernel inside the step: CUPTI kernel records of one plan
    in_step = None if args.no_in_step else level0_in_step(sim, stream)
    # ---- end to end through the C ABI with host buffers ----------------------
    import numpy as np

    A = [geo.Areas[a] for a in range(geo.layout.number_area)]
    host = []
    for a in A:
        n = a.nx * a.ny
        host.append({k: torch.empty(n * (9 if k == "F" else 1), dtype=torch.float64).pin_memory().numpy()
                     for k in ("rho", "ux", "uy", "F")})
    ref = mblbm.MultiBlockLBM(geo, args.precision)
    ref.init(stream)
    for i, h in enumerate(host):
        f = ref.fields(i, stream)
        for k in h:
            h[k][:] = f[k].ravel()
    ref.close()
    # the result fields (rho, ux, uy and the cell types: what the reference's
    # output() writes) come back into pinned host buffers
    host_out = []
    for a in A:
        pin = lambda shp, dt: torch.empty(shp, dtype=dt).pin_memory().numpy()
        host_out.append({"rho": pin((a.ny, a.nx), torch.float64), "ux": pin((a.ny, a.nx), torch.float64),
                         "uy": pin((a.ny, a.nx), torch.float64), "solid": pin((a.ny, a.nx), torch.int32)})
    sim2 = mblbm.MultiBlockLBM(geo, args.precision)
    sim2.init(stream)
    for i, h in enumerate(host):  # sizes the library's staging buffer outside the timed region
        sim2.set_fields(i, h["rho"], h["ux"], h["uy"], h["F"], stream)
    sim2.init(stream)
    sim2.prepare_diag(args.steps)  # plans, graphs and result buffers of the timed call
    torch.cuda.synchronize()
    h2d = sum(h[k].nbytes for h in host for k in h)
    d2h = 0
    barrier()
    t0 = time.perf_counter()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for i, h in enumerate(host):
        sim2.set_fields(i, h["rho"], h["ux"], h["uy"], h["F"], stream)
    # the reference's loop: a step, getDrag_block and error_L2 every step, each
    # step's Cd, Cl and L2 change copied to the host (mb_step_diag)
    cd_series, cl_series, l2_series = sim2.evolution_diag(args.steps, stream)
    d2h += 32 * args.steps
    out = [sim2.fields(i, stream, out=host_out[i]) for i in range(len(A))]
    d2h += sum(v.nbytes for f in out for k, v in f.items() if k != "solid")
    f1.record(stream)
    barrier()
    ms_e2e = f0.elapsed_time(f1)
    wall_e2e = time.perf_counter() - t0
    sim2.close()

    ms, ms_e2e = ranks.reduce([ms, ms_e2e], "max", dist, device="cuda")  # the slowest rank's device time

    if rank == 0:
        peak, src = peaks()
        achieved = kbytes / (kms * 1e-3) / 1e9
        traffic = dram_traffic_per_launch(args.precision)
        line = {
            "metric": METRIC,
            "value": round(world * upd * args.steps / (ms * 1e-3) / 1e6, 1),
            "unit": "MLUPS",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(ms / args.steps, 5),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": args.precision,
            "data": "synthetic",
            "config": bench_config(world),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic, "peak_source": src,
                         "kernel": "k_block_step level 0", "alg_bytes_per_launch": kbytes, "cells_per_launch": kcells,
                         "ms_per_launch": round(kms, 5), "bytes_per_update": BYTES_PER_UPDATE[args.precision],
                         "in_step": None if in_step is None else {
                             "kernel": in_step[0], "ms_per_launch": round(in_step[1], 5),
                             "achieved": round(in_step[2] / (in_step[1] * 1e-3) / 1e9, 1),
                             "frac": round(in_step[2] / (in_step[1] * 1e-3) / 1e9 / peak, 4),
                             "what": "mean duration of the level-0 interior launch inside the CUDA graph of "
                                     "6 coarse steps (CUPTI kernel records via torch.profiler), beside the "
                                     "fine levels' chain; bytes per update x its cells"}},
            "e2e": {"value": round(world * upd * args.steps / (ms_e2e * 1e-3) / 1e6, 1), "unit": "MLUPS",
                    "h2d_bytes_per_step": round(h2d / args.steps), "d2h_bytes_per_step": round(d2h / args.steps),
                    "wall_s": round(wall_e2e, 3),
                    "what": "C ABI with host buffers: upload of the FP64 D2Q9 state (rho, ux, uy, F) from pinned "
                            "memory, mb_step_diag (per step: coarse step, drag and L2 change as the reference loop, "
                            "32 B of results copied to the host), download of the final rho, ux, uy (FP64)"},
            "gpu_launches": kernels,
            "clocks": clk.summary(),
        }
        if not args.no_cpu_baseline and world == 1:
            line["cpu_baseline"] = cpu_baseline()
        print(json.dumps(line), flush=True)
    sim.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
