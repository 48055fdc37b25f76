#!/usr/bin/env python3
"""bench.py -- converged ATLAS12 models per hour on B200.

Workload (the opacity-sampling configuration): ATLAS12 models with 30,000
log-spaced frequencies over 9 nm - 160 um, 72 depths and 500,000 synthetic
lines (lambda log-uniform, log gf ~ N(-2, 1.5), E_low ~ U(0, 8) eV,
log gamma_rad/Stark/vdW ~ N(8, .3)/N(-5.5, .5)/N(-7.5, .3)), each iterated
until max |FLXERR| <= 0.1 % (Delta F/F <= 1e-3) within 30 iterations (the
reference's default NUMITS); a model still above it then counts as not
converged.  A step is one set of 32
models whose stellar parameters are drawn (seeded) from the warm-start box:
Teff 3500-8000 K, log g 1-5, [M/H] -2..+0.5, vturb 0.5-3 km/s.  Populations
and continuum come from the documented synthetic surrogate.

value: converged models per hour (whole job) of this library's path --
batched models (one captured graph per iteration for all slots),
mixed-precision LINOP1, and the learned warm start (the grey start where the
network gives no valid structure) -- with inputs resident in HBM, L2 flushed (256 MB write) between
steps, CUDA events on the library's stream.  plain_fp64: the same 32 models
one at a time, all-FP64, grey start, one launch at a time (the plain FP64 GPU
path the patterns are measured against).  e2e: the same step through the
public API from host buffers (batch creation with the line list upload,
warm-start prediction, iteration, read-back of every structure).

--impl reference times the CPU restatement of the same path (oracle/, the
reference's own Fortran cannot be built in this image) on all host threads,
on the same configuration: the step's 32 models from the same starting
structures (the network's predictions evaluated on the host in FP64, grey
where they are not usable), each iterated by the oracle until it converges
or reaches 30 iterations.  A reference step is a bounded sample of that
work -- 12 oracle iterations of the model queue, carried over from step to
step -- and converged models/hr is measured on the models the timed steps
complete: converged count x 3600 / the seconds spent on them.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CFG = dict(workload="atlas12-opacity-sampling model set", numnu=30000, wl_lo=9.0, wl_hi=160000.0, nrhox=72,
           nlines=500000, line_seed=2, models_per_step=32, param_seed=13,
           params="Teff U(3500,8000) K, log g U(1,5), [M/H] U(-2,0.5), vturb U(0.5,3) km/s", tol_percent=0.1,
           max_iter=30, slots=32, vturb_solar=1.5,
           # the surrogate's line populations are 0.01 of full strength (a
           # purely radiative model with 500,000 full-strength lines has no
           # reachable radiative-equilibrium solution from the grey start)
           atlas_line_pop=0.01, populations="synthetic surrogate EOS and continuum",
           start="learned warm start (trained network), grey where its structure is not usable")
# oracle iterations per reference step (a bounded sample of the model queue)
REF_ITERS_PER_STEP = 12
WARMSTART = os.path.join(ROOT, "atlas12_b200", "data", "warmstart_c2.npz")
# FP64 flops counted per frequency in the RT kernel: LU 2/3 51^3, triangular
# solves 2*51^2, system build 2*51^2, J/H/K operators 4*51^2 + 2*51,
# INTEG/MAP1/DERIV and the mode-2 sums ~ 110 per depth (72 depths)
FLOPS_PER_NU = int(2 / 3 * 51 ** 3 + 8 * 51 ** 2 + 2 * 51 + 110 * 72)
# the part of FLOPS_PER_NU that is the scattering solve (LU, triangular
# solves, system build) and the FP64 operations of one Neumann-series step
# (a 51x51 matrix-vector product and the update)
FLOPS_PER_SOLVE = int(2 / 3 * 51 ** 3 + 4 * 51 ** 2)
FLOPS_PER_SERIES_STEP = 2 * 51 ** 2 + 3 * 51
# DRAM bytes per model of the three batched RT launches that do not depend on
# the launch shape (ncu, 4-slot capture of this workload: 337 MB per model
# less the 138 MB of partial-sum rows it wrote, one per frequency at 4 slots):
# ACONT, SIGMAC and XLINES read by the prepare and finish stages, the
# per-frequency records written and read back.  The finish stage's
# partial-sum rows (one 577-double row per finish warp) are added for the
# tuned shape (rt_partial_rows).
RT_TRAFFIC_FIXED_PER_MODEL = 199e6


def rt_partial_rows(numnu, nsm, slots, waves, warps_per_block=4):
    """Partial-sum rows per model of the split RT pass's finish stage at a
    launch shape (rt_split_shape in csrc/atlas.cuh: 16 warps per SM per wave
    over the batch, each a contiguous run of one slot's frequencies)."""
    units = max(1, nsm * 16 * waves // max(slots, 1))
    per = max(1, -(-numnu // units))
    n = -(-numnu // per)
    return -(-n // warps_per_block) * warps_per_block
# DRAM bytes per model of one batched LINOP1 launch (ncu, 4-slot capture of
# this workload: 959 MB): the prepared line records and the fixed-point XLINES
# words, whose write-backs dominate once several models' words exceed L2
LINOP_TRAFFIC_PER_MODEL = 240e6
# bytes of one prepared LINOP1 line record on the device (AtlasLine)
LINE_RECORD_BYTES = 56
# FP64 operations of one SYNTHE Weideman Voigt evaluation (31 complex Horner
# steps of 8, plus the setup and the closing terms)
WEIDEMAN_FLOP = 278


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP64 GPU comparison")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-synthe-c3", action="store_true", help="skip the 20M-line full-optical SYNTHE case")
    ap.add_argument("--slots", type=int, default=None, help="batch slots (default: one per model of a step)")
    ap.add_argument("--no-select", action="store_true", help="skip the SELECTLINES line-database rates")
    ap.add_argument("--synthe-grid", type=int, default=0,
                    help="also time N atmospheres of the batched-grid SYNTHE workload, concurrent vs one at a time")
    return ap.parse_args()


def workload():
    from atlas12_b200 import surrogate, synthetic, warmstart
    ws, rc = synthetic.geometric_waveset(CFG["wl_lo"], CFG["wl_hi"], CFG["numnu"])
    lines = synthetic.atlas_lines(CFG["nlines"], ws[2], ws[-3], seed=CFG["line_seed"])
    rank = int(os.environ.get("RANK", "0"))
    params = warmstart.sample_params(CFG["models_per_step"], CFG["param_seed"] + rank)
    grey = [warmstart.grey_start(teff, logg, mh, CFG["nrhox"]) for teff, logg, mh, _ in params]
    solar = surrogate.grey_model(5777.0, 4.44, nrhox=CFG["nrhox"], ross=surrogate.RossTable())
    return dict(ws=ws, rc=rc, lines=lines, params=params, grey=grey, solar=solar)


def operators():
    """The operator data a caller passes (package data, from the reference's files)."""
    from atlas12_b200 import operators as op
    return op.load()


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                      stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            out, _ = self.p.communicate(timeout=5)
        except Exception:
            self.p.kill()
            out = ""
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def host_starts(params, grey):
    """The GPU arm's starting structures computed on the host: the trained
    network evaluated in FP64 by the numpy restatement of the network
    (oracle/mlp_ref.py), grey where its structure is not finite and positive."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import mlp_ref
    from atlas12_b200 import warmstart
    if not os.path.exists(WARMSTART):
        return list(grey)
    d = np.load(WARMSTART)
    shape = tuple(int(x) for x in d["shape"])
    ws = warmstart.WarmStart(None, d["ymean"], d["ystd"], bool(d["residual"]) if "residual" in d.files else False)
    yn = mlp_ref.forward(d["params"].astype(np.float64), warmstart.encode_inputs(params), shape)[2]
    out = []
    for s_, g in zip(warmstart.structures(params, *ws.destandardise(yn, params, grey)), grey):
        good = all(np.all(np.isfinite(s_[k])) and np.all(s_[k] > 0) for k in ("t", "p", "rhox"))
        out.append(s_ if good else g)
    return out


class OracleQueue:
    """The step's models on the CPU oracle, one after another: each from its
    start until max |FLXERR| <= tol or max_iter iterations (the reference's
    grid scripts run one model per process in the same way).  run(k) runs k
    more oracle iterations of the queue and times each; a model's time is
    the sum of its iterations'."""

    def __init__(self, W, tables, starts):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle as po
        from atlas12_b200 import atlas
        self.po, self.atlas, self.W, self.tables, self.starts = po, atlas, W, tables, starts
        self.next_model = 0
        self.cur = None
        self.done = []  # (model, converged, iterations, seconds)

    def _open(self):
        from iteration import OracleIteration
        i = self.next_model % len(self.W["params"])
        self.next_model += 1
        teff, logg, mh, vt = self.W["params"][i]
        it = OracleIteration(self.po, self.atlas, self.tables, self.W["ws"], self.W["rc"], self.W["lines"],
                             self.starts[i], teff, vt, mh=mh, grav=10.0 ** logg)
        self.cur = dict(model=i, it=it, n=0, sec=0.0)

    def run(self, k):
        for _ in range(k):
            if self.cur is None:
                self._open()
            c = self.cur
            t0 = time.perf_counter()
            err = c["it"].step()
            c["sec"] += time.perf_counter() - t0
            c["n"] += 1
            conv = bool(err <= CFG["tol_percent"])
            if conv or not np.isfinite(err) or c["n"] >= CFG["max_iter"]:
                self.done.append((c["model"], conv, c["n"], c["sec"]))
                self.cur = None

    def rate(self):
        """(converged models/hr over the completed models, completed, converged, seconds, iterations)."""
        sec = sum(d[3] for d in self.done)
        conv = sum(d[1] for d in self.done)
        its = sum(d[2] for d in self.done)
        return (conv * 3600.0 / sec if sec > 0 else 0.0), len(self.done), conv, sec, its


def run_reference(args):
    """The CPU restatement of the same path on all host threads, on the
    same models and starting structures as the GPU arm (rank 0 only)."""
    rank, world, local = dist_setup(args)
    if rank != 0:
        return 0
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    W = workload()
    starts = host_starts(W["params"], W["grey"])
    q = OracleQueue(W, operators(), starts)
    q.run(max(args.warmup, 1))  # warm-up: the first iterations (threads, caches); the queue restarts after
    q = OracleQueue(W, operators(), starts)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        q.run(REF_ITERS_PER_STEP)
        times.append(time.perf_counter() - t0)
    v, ncomp, nconv, sec, its = q.rate()
    sample = (f"{args.steps} steps of {REF_ITERS_PER_STEP} oracle iterations over the step's model queue (same 32 "
              f"models and starting structures as the GPU arm, each to max|FLXERR| <= 0.1 % or 30 iterations): "
              f"{ncomp} models completed, {nconv} converged, {its} iterations in {sec:.1f} s on "
              f"{os.environ['OMP_NUM_THREADS']} threads")
    line = {"impl": "reference", "metric": "converged models/hr (dF/F<=1e-3)", "value": v, "unit": "models/hr",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": float(np.mean(times)) * 1e3 if times else None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(CFG, parallelism=f"replicas x{args.gpus}"),
            "execution": "CPU oracle (C restatement of the reference's iteration), OpenMP over the host threads",
            "cpu_baseline": {"value": v, "unit": "models/hr", "cores": int(os.environ["OMP_NUM_THREADS"]),
                             "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "models/hr", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def atlas_mixed_error(ctx, batch, params, starts):
    """One step of the same models from the same starts in all-FP64 and in
    mixed precision: how many converge each way, and for the models that
    converge both ways the largest relative T and P difference and the
    largest FLXERR difference (percent points) of the converged structures."""
    from atlas12_b200 import _lib
    out = {}
    res = {}
    for name, prec in (("fp64", _lib.PREC_FP64), ("mixed", _lib.PREC_MIXED)):
        ctx.set_precision(prec)
        res[name] = batch.run_queue(params, starts, max_iter=CFG["max_iter"], tol_percent=CFG["tol_percent"],
                                    keep=True)
    ctx.set_precision(_lib.PREC_MIXED)
    conv = {k: [r["status"] == _lib.SLOT_CONVERGED for r in v] for k, v in res.items()}
    both = [i for i in range(len(params)) if conv["fp64"][i] and conv["mixed"][i]]
    out["converged_fp64"] = int(sum(conv["fp64"]))
    out["converged_mixed"] = int(sum(conv["mixed"]))
    out["compared"] = len(both)
    if both:
        a, b = res["mixed"], res["fp64"]
        out["max_rel_T"] = float(max(np.max(np.abs(a[i]["t"] / b[i]["t"] - 1)) for i in both))
        out["max_rel_P"] = float(max(np.max(np.abs(a[i]["p"] / b[i]["p"] - 1)) for i in both))
        out["max_abs_flxerr_percent"] = float(max(np.max(np.abs(a[i]["flxerr"] - b[i]["flxerr"])) for i in both))
        out["iterations_fp64"] = int(sum(b[i]["iters"] for i in both))
        out["iterations_mixed"] = int(sum(a[i]["iters"] for i in both))
    return out


def warm_starts(ctx, params, grey):
    """Starting structures from the trained network; the grey start where the
    network is absent or its structure is not finite and positive."""
    from atlas12_b200 import warmstart
    if not os.path.exists(WARMSTART):
        return list(grey), False
    ws = warmstart.WarmStart.load(WARMSTART, ctx)
    starts = []
    for s, g in zip(ws.starts(params, grey), grey):
        good = all(np.all(np.isfinite(s[k])) and np.all(s[k] > 0) for k in ("t", "p", "rhox"))
        starts.append(s if good else g)
    ws.mlp.close()
    return starts, True


def run_ours(args):
    import torch
    from atlas12_b200 import _lib, atlas

    rank, world, local = dist_setup(args)
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    stream = torch.cuda.current_stream()
    W = workload()
    ops = operators()
    params, grey = W["params"], W["grey"]
    ctx = _lib.Context(local, _lib.PREC_MIXED, stream=stream.cuda_stream)
    starts, learned = warm_starts(ctx, params, grey)
    if args.slots:
        CFG["slots"] = args.slots
    batch = atlas.AtlasBatch(ctx, ops, nslots=CFG["slots"], linedata=W["lines"], waveset=W["ws"], rcoset=W["rc"])
    # launch shape chosen by the autotuner on these models (outside the timed region)
    from atlas12_b200 import autotune
    lc, rw, tuned = autotune.tune_batch(batch, params, grey)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def one_step(b=batch, st=starts, keep=False):
        return b.run_queue(params, st, max_iter=CFG["max_iter"], tol_percent=CFG["tol_percent"], keep=keep)

    for _ in range(max(args.warmup, 1)):
        one_step()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    total_ms, converged, iters, attempts = 0.0, 0, [], []
    clocks = Clocks(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    l0 = ctx.launches()
    for _ in range(args.steps):
        flush.zero_()  # L2 flush between steps (256 MB > 126 MB L2)
        ev0.record(stream)
        res = one_step()
        ev1.record(stream)
        torch.cuda.synchronize()
        total_ms += ev0.elapsed_time(ev1)
        converged += sum(r["status"] == _lib.SLOT_CONVERGED for r in res)
        iters += [r["iters"] for r in res]
        attempts += [r["attempts"] for r in res]
    gpu_launches = ctx.launches() - l0
    clk = clocks.stop()
    torch.cuda.synchronize()
    t_max = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
    conv_all = torch.tensor([converged], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
        dist.all_reduce(conv_all, op=dist.ReduceOp.SUM)
    t_max = float(t_max.item())
    value = float(conv_all.item()) * 3600.0 / (t_max / 1e3)

    # per-kernel times of one batched iteration with every slot running (CUDA events, no graph)
    for s_ in range(CFG["slots"]):
        teff, logg, mh, vt = params[s_ % len(params)]
        batch.load(s_, teff, logg, vt, mh, grey[s_ % len(params)], max_iter=3, tol_percent=0.0)
    batch.step(1)
    ctx.enable_timing(True)
    batch.step(1)
    names = ("eos", "kapcont", "kapp", "linop", "rt", "rt_pre", "rt_solve", "rt_post", "reduce", "finish")
    kms = {k: ctx.kernel_ms("batch_" + k) for k in names}
    linop_points = ctx.kernel_work("batch_linop_points")
    linop_atomics = ctx.kernel_work("batch_linop_atomics")
    rt_solves = {k: ctx.kernel_work("batch_rt_" + k) for k in ("eliminated", "series", "series_steps")}
    ctx.enable_timing(False)
    batch.run()
    per_model = {k: v / CFG["slots"] for k, v in kms.items()}
    fp64_peak = float(_lib.lib().atlasgpu_fp64_peak_tflops(ctx.handle))
    ach = CFG["slots"] * CFG["numnu"] * FLOPS_PER_NU / (kms["rt"] * 1e-3) / 1e12
    # FP64 operations the pass executed: the per-frequency work outside the
    # solve, each eliminated system's LU, each series step's matrix-vector product
    nfreq = CFG["slots"] * CFG["numnu"]
    executed = (nfreq * (FLOPS_PER_NU - FLOPS_PER_SOLVE) + rt_solves["eliminated"] * FLOPS_PER_SOLVE
                + rt_solves["series_steps"] * FLOPS_PER_SERIES_STEP)
    import torch
    rows = rt_partial_rows(CFG["numnu"], torch.cuda.get_device_properties(0).multi_processor_count, CFG["slots"],
                           batch.shape()[1])
    rt_traffic = RT_TRAFFIC_FIXED_PER_MODEL + rows * (8 * CFG["nrhox"] + 1) * 8
    roof = {"kernel": "RT pass (k_batch_rt_pre + k_batch_rt_series + k_batch_rt_solve + k_batch_rt_post, JOSH per "
                      "frequency, FP64)",
            "bound": "fp64", "achieved": ach, "peak": fp64_peak,
            "unit": "TFLOP/s", "frac": ach / fp64_peak if fp64_peak > 0 else None,
            "executed_tflops": executed / (kms["rt"] * 1e-3) / 1e12,
            "traffic": rt_traffic * CFG["slots"],
            "traffic_scaling": f"ncu capture of the three launches of a 4-slot batch (337 MB per model, 138 MB of "
                               f"them partial-sum rows); the rows rescaled to this shape's {rows} per model "
                               f"({rows * (8 * CFG['nrhox'] + 1) * 8 / 1e6:.0f} MB), times slots",
            "peak_source": "measured DFMA loop on this GPU (atlasgpu_fp64_peak_tflops); MEASURED_PEAKS.json has no FP64 figure",
            "work": f"{FLOPS_PER_NU} FP64 flop per frequency (the reference's elimination counted for every "
                    f"system) x {CFG['numnu']} frequencies x {CFG['slots']} models per pass; executed_tflops counts "
                    "the series steps and eliminations actually run",
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the RT launches (profiles/)"}
    # LINOP1 over the batch: its bound is the L2 atomics of the exact XLINES
    # sums (each wing point adds 1-3 64-bit words, the access pattern of the
    # measured atomic peak); the algorithmic bytes (prepared line records read
    # once per slot, XLINES read and written once) against HBM beside it
    hbm, hbm_src = hbm_peak()
    atom_peak = float(_lib.lib().atlasgpu_u64_atomic_peak(ctx.handle))  # 1e9 atomics/s
    linop_s = kms["linop"] * 1e-3
    linop_bytes = CFG["slots"] * (CFG["nlines"] * LINE_RECORD_BYTES + 2 * 8 * CFG["numnu"] * CFG["nrhox"])
    linop_roof = {"kernel": "k_batch_linop (LINOP1 wing walks, exact fixed-point XLINES sums)", "bound": "l2_atomics",
                  "unit": "G atomics/s", "achieved": linop_atomics / linop_s / 1e9 if linop_atomics > 0 else None,
                  "peak": atom_peak, "peak_source": "measured 64-bit atomic-add loop on this GPU "
                                                    "(atlasgpu_u64_atomic_peak; warps on 32 consecutive words)",
                  "frac": (linop_atomics / linop_s / 1e9 / atom_peak) if linop_atomics > 0 and atom_peak > 0 else None,
                  "atomics": linop_atomics, "points": linop_points,
                  "points_per_s": linop_points / linop_s if linop_points > 0 else None,
                  "hbm": {"achieved": linop_bytes / linop_s / 1e9, "peak": hbm, "peak_source": hbm_src,
                          "frac": linop_bytes / linop_s / 1e9 / hbm, "unit": "GB/s",
                          "work": f"{LINE_RECORD_BYTES} B per prepared line x {CFG['nlines']} lines + XLINES "
                                  f"({CFG['numnu']} x {CFG['nrhox']} FP64) read and written, per slot"},
                  "traffic": LINOP_TRAFFIC_PER_MODEL * CFG["slots"],
                  "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of a 4-slot k_batch_linop "
                                    "launch (profiles/), per model, times slots",
                  "work": "counted 64-bit atomic adds of one batched launch (32 slots)"}
    # the dominant kernel of the step carries the line's roofline key
    if kms["linop"] > kms["rt"]:
        roof, rooflines = linop_roof, [roof]
    else:
        rooflines = [linop_roof]

    # ATLAS mixed precision against the plain all-FP64 arithmetic on the same
    # models from the same starts (north star (1)): converged structures
    mx_err = atlas_mixed_error(ctx, batch, params, starts)

    # plain FP64 GPU path: the same models one at a time, FP64, grey start, per-launch host loop
    plain = None
    if not args.no_plain and rank == 0:
        ctx.set_precision(_lib.PREC_FP64)
        model = atlas.AtlasModel(ctx, ops, teff=5777.0, logg=4.44, vturb=1.5, linedata=W["lines"], waveset=W["ws"],
                                 rcoset=W["rc"], start=W["solar"])
        pm, pconv, pit = 0.0, 0, []
        flush.zero_()
        for (teff, logg, mh, vt), g in zip(params, grey):
            model.set_params(teff, logg, vt, mh)
            model.set_structure(g["t"], g["p"], g["rhox"])
            ev0.record(stream)
            try:
                n, hist = model.iterate(max_iter=CFG["max_iter"], tol_percent=CFG["tol_percent"], graph=False)
                ok = n > 0 and hist[-1] <= CFG["tol_percent"]
            except _lib.AtlasGPUError:
                n, ok = CFG["max_iter"], False
            ev1.record(stream)
            torch.cuda.synchronize()
            pm += ev0.elapsed_time(ev1)
            pconv += int(ok)
            pit.append(n)
        model.close()
        ctx.set_precision(_lib.PREC_MIXED)
        plain = {"value": pconv * 3600.0 / (pm / 1e3), "unit": "models/hr", "converged": pconv,
                 "models": len(params), "ms_per_model": pm / len(params), "mean_iterations": float(np.mean(pit)),
                 "path": "FP64 everywhere, one model at a time, per-launch host loop, grey start"}

    # e2e through the public API from host buffers (batch creation uploads the line list and grid)
    e2e_s = 0.0
    ne2e = max(1, min(args.steps, 2))
    h2d = d2h = 0
    for _ in range(ne2e):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        # the launch shape the autotuner chose above (also what the batch reads from its cache)
        b2 = atlas.AtlasBatch(ctx, ops, nslots=CFG["slots"], linedata=W["lines"], waveset=W["ws"], rcoset=W["rc"],
                              shape=(lc, rw))
        st2, _ = warm_starts(ctx, params, grey)
        res = one_step(b2, st2, keep=True)
        torch.cuda.synchronize()
        e2e_s += time.perf_counter() - t0
        b2.close()
        n_loads = sum(r["attempts"] for r in res)
        h2d = (W["lines"].nbytes + W["ws"].nbytes + W["rc"].nbytes + 361 * 8 + 3 * 2001 * 8 +
               n_loads * 3 * CFG["nrhox"] * 8)
        d2h = len(res) * (5 * CFG["nrhox"] * 8 + CFG["numnu"] * 8)
    e2e_all = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(e2e_all, op=dist.ReduceOp.MAX)
    e2e_value = world * ne2e * converged / max(args.steps, 1) * 3600.0 / float(e2e_all.item())

    # the single grey-start solar model (30,000 frequencies, 500,000 lines) on the batch path
    b1 = atlas.AtlasBatch(ctx, ops, nslots=1, linedata=W["lines"], waveset=W["ws"], rcoset=W["rc"])
    b1.load(0, 5777.0, 4.44, 1.5, 0.0, W["solar"], max_iter=CFG["max_iter"], tol_percent=CFG["tol_percent"])
    b1.run()
    b1.load(0, 5777.0, 4.44, 1.5, 0.0, W["solar"], max_iter=CFG["max_iter"], tol_percent=CFG["tol_percent"])
    torch.cuda.synchronize()
    ev0.record(stream)
    st1, it1, er1 = b1.run()
    ev1.record(stream)
    torch.cuda.synchronize()
    single = {"ms": ev0.elapsed_time(ev1), "iterations": int(it1[0]), "max_flxerr_percent": float(er1[0]),
              "start": "Eddington grey, Teff 5777 K, log g 4.44"}
    b1.close()

    syn = None
    if rank == 0 and world == 1:
        # C1: 20,000 atomic lines, 400-410 nm at R = 500,000, 72 depths
        syn = {"c1": synthe_rates(ctx, ops, 20000, 400.0, 410.0, 0.0, fp64_peak=fp64_peak)}
        if not args.no_synthe_c3:
            # C3: 20M lines (30 % molecular), 300-1000 nm at R = 500,000
            syn["c3"] = synthe_rates(ctx, ops, 20000000, 300.0, 1000.0, 0.3, fp64_peak=fp64_peak)
            rooflines += syn["c3"]["rooflines"]
        if args.synthe_grid:
            syn["grid"] = synthe_grid_rate(local, ops, args.synthe_grid)

    kp = None
    if rank == 0 and world == 1:
        kp = kapp_rate(ctx, ops, W)

    sel = None
    if rank == 0 and world == 1 and not args.no_select:
        sel = selectlines_rates(ctx, ops, cpu=not args.no_cpu)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(W, ops, starts, sum(iters) / args.steps, converged / args.steps)
    if rank == 0:
        line = {"metric": "converged models/hr (dF/F<=1e-3)", "value": value, "unit": "models/hr",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded lines and stellar parameters, surrogate populations/continuum)",
                "launch_shape": {"linop_ctas_per_sm": lc, "rt_waves": rw, "autotune": tuned},
                "config": dict(CFG, parallelism=f"replicas x{world}"),
                "execution": "batched models (one captured graph per iteration), mixed-precision LINOP1, FP64 "
                             "transfer" + ("" if learned else "; no trained network found: grey starts"),
                "l2": "flushed between steps (256 MB write)",
                "converged_per_step": float(conv_all.item()) / args.steps / world,
                "mean_iterations_per_model": float(np.mean(iters)),
                "kernel_ms_per_model_iteration": per_model, "rt_solves_per_iteration": rt_solves,
                "roofline": roof, "rooflines": rooflines,
                "atlas": {"mixed_error_vs_fp64": mx_err}, "cpu_baseline": cpu,
                "plain_fp64": plain, "vs_plain_fp64": (value / plain["value"]) if plain and plain["value"] else None,
                "single_model": single, "synthe": syn, "selectlines": sel, "kapp_hydrogen": kp,
                "e2e": {"value": e2e_value, "unit": "models/hr", "h2d_bytes_per_step": int(h2d),
                        "d2h_bytes_per_step": int(d2h)},
                "gpu_launches": int(gpu_launches), "clocks": clk}
        print(json.dumps(line), flush=True)
    batch.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# SELECTLINES workloads: one database loop per record format, each input
# 320 MB (larger than L2), records in file (wavelength) order
SELECT_CASES = [("gfpred LINEREC (16 B)", 1, 20_000_000), ("TiO MOL2 (32 B)", 5, 10_000_000),
                ("H2O (8 B)", 6, 40_000_000)]
# DRAM bytes of one 12M-record LINEREC call, all its kernels (ncu): 437 MB,
# 36.4 B per record (the tile-maximum pass reads the records a second time)
SELECT_TRAFFIC_PER_LINEREC = 36.4


def kapp_rate(ctx, ops, W):
    """KAPP's hydrogen continuum sources (atlasgpu_atlas_kapp_hydrogen), and with
    the helium ones (atlasgpu_atlas_kapp), over the workload's 30,000
    frequencies and 72 depths of the grey solar model:
    kernel time (CUDA events, after a warm-up call) and (frequency, depth)
    evaluations per second; the call's host copies are outside the kernel time."""
    from atlas12_b200 import atlas, surrogate
    A = atlas.Atlas(ctx, ops)
    A.set_kapp_tables(ops)
    m = W["solar"]
    e = surrogate.eos(m["t"], m["p"])
    args = (W["ws"], m["t"], e["xne"], e["rho"], e["nh"] * (1 - e["xh"]) / 2, e["nh"] * e["xh"])
    A.kapp_hydrogen(*args)
    ctx.enable_timing(True)
    A.kapp_hydrogen(*args)
    ms = ctx.kernel_ms("kapp_hydrogen")
    ctx.enable_timing(False)
    n = W["ws"].size * m["t"].size
    # the same with the helium sources (atlasgpu_atlas_kapp): helium at 0.0851
    # of hydrogen by number, its ionisation split by smooth functions of T
    t = m["t"]
    nhe = 0.0851 * e["nh"]
    f1 = 1.0 / (1.0 + np.exp(-(t - 12000.0) / 1500.0))
    f2 = 1.0 / (1.0 + np.exp(-(t - 22000.0) / 2500.0))
    xnf4 = nhe * f1 * (1.0 - f2)
    hargs = args + (nhe * (1.0 - f1), xnf4 / 2.0, nhe * f1 * f2, xnf4)
    A.kapp(*hargs)
    ctx.enable_timing(True)
    A.kapp(*hargs)
    ms_he = ctx.kernel_ms("kapp")
    ctx.enable_timing(False)
    # and with the H2 sources (H2MINOP, H2COLLOP, H2RAOP)
    A.set_kapp_h2_tables(ops)
    A.kapp(*hargs, xnf3=hargs[6])
    ctx.enable_timing(True)
    A.kapp(*hargs, xnf3=hargs[6])
    ms_h2 = ctx.kernel_ms("kapp")
    ctx.enable_timing(False)
    # HLINOP with STARK_MMM on seeded Stehle-format tables of the published shapes
    from atlas12_b200 import synthetic
    A.set_stehle_tables(synthetic.stehle_tables())
    hl_args = (W["ws"], m["t"], e["xne"], e["rho"], args[4])
    A.hlinop(*hl_args)
    ctx.enable_timing(True)
    A.hlinop(*hl_args)
    ms_hl = ctx.kernel_ms("hlinop")
    ctx.enable_timing(False)
    return {"frequencies": int(W["ws"].size), "depths": int(m["t"].size), "kernel_ms": ms,
            "evals_per_s": n / (ms * 1e-3) if ms > 0 else None,
            "sources": "HOP (n = 1..80), H2PLOP, HMINOP, HRAYOP, ELECOP and KAPP's totals",
            "with_helium": {"kernel_ms": ms_he, "evals_per_s": n / (ms_he * 1e-3) if ms_he > 0 else None,
                            "sources": "the above and HE1OP, HE2OP, HEMIOP, HERAOP"},
            "with_helium_h2": {"kernel_ms": ms_h2, "evals_per_s": n / (ms_h2 * 1e-3) if ms_h2 > 0 else None,
                               "sources": "the above and H2MINOP, H2COLLOP, H2RAOP"},
            "hlinop": {"kernel_ms": ms_hl, "evals_per_s": n / (ms_hl * 1e-3) if ms_hl > 0 else None,
                       "sources": "HLINOP, STARK_MMM on seeded Stehle-format tables"}}


def hbm_peak():
    """Measured copy bandwidth of this pool's B200s, else the stated fallback (GB/s)."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs"
    except (OSError, KeyError, ValueError, TypeError):
        return 6650.0, "fallback 6.65 TB/s (no MEASURED_PEAKS.json)"


def selectlines_rates(ctx, ops, cpu=True, reps=3):
    """SELECTLINES (one database loop) per record format: the device passes'
    time (CUDA events in the library around all of them, best of reps after
    a warm-up, inputs resident in HBM), their HBM roofline (records read +
    LINEDATA written), the host entry point end to end (records from host
    memory, LINEDATA back; best of two calls), and the oracle on a 2M-record
    sample (one core)."""
    import torch
    from atlas12_b200 import atlas, linelists, synthetic
    wt = ops["wavetab"]
    xn, hckt, tc = synthetic.selectlines_tables(wt)
    S = linelists.SelectLines(ctx, 72, xn, hckt, tc, atlas.iwavetab(wt), wt)
    peak, src = hbm_peak()
    out = {"tables": "synthetic XNFDOP/TABCONT over the reference's WAVETAB (361 bins), 1006 species, 72 depths",
           "peak_gbs": peak, "peak_source": src, "cases": []}
    ctx.enable_timing(True)
    for name, kind, n in SELECT_CASES:
        recs = synthetic.selectlines_records(kind, n, wt, seed=1)
        raw = np.ascontiguousarray(recs).view(np.uint8)
        d_in = torch.from_numpy(raw).cuda()
        d_out = torch.empty((n, 4), dtype=torch.int32, device="cuda")
        ms = []
        for _ in range(reps + 1):
            st = linelists.initial_state(wt)
            m = S.select_dev(kind, d_in, n, st, d_out, n)
            ms.append(ctx.kernel_ms("k_selectlines"))
        k_ms = min(ms[1:])
        algo = raw.nbytes + 16 * m
        e2e = float("inf")
        for _ in range(2):  # the first call also grows the context's buffers
            t0 = time.perf_counter()
            st = linelists.initial_state(wt)
            host_out = S.select(kind, recs, st)
            e2e = min(e2e, time.perf_counter() - t0)
        case = {"database": name, "records": n, "selected": m, "kernel_ms": k_ms,
                "records_per_s": n / (k_ms * 1e-3), "algorithmic_bytes": int(algo),
                "roofline": {"bound": "hbm", "achieved": algo / (k_ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                             "frac": algo / (k_ms * 1e-3) / 1e9 / peak,
                             "traffic": SELECT_TRAFFIC_PER_LINEREC * n if kind == 1 else None},
                "e2e": {"records_per_s": n / e2e, "h2d_bytes": int(raw.nbytes),
                        "d2h_bytes": int(host_out.nbytes)}}
        if cpu:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import pyoracle as po
            sub = recs[:2_000_000]
            tb = {k: ops[k] for k in ("molcodes", "isox", "tio_isocorr", "h2o_isocorr")}
            xmax = po.xnfdopmax(72, xn, tc)
            t0 = time.perf_counter()
            po.selectlines(tb, kind, sub, linelists.initial_state(wt), xmax, hckt[-1], atlas.iwavetab(wt), wt)
            dt = time.perf_counter() - t0
            case["cpu_baseline"] = {"records_per_s": len(sub) / dt, "cores": 1, "kind": "port",
                                    "sample": f"first {len(sub)} records of the same database"}
        out["cases"].append(case)
        del d_in, d_out
    ctx.enable_timing(False)
    return out


def synthe_rates(ctx, ops, nlines, wlbeg, wlend, mol_frac, seed=1, fp64_peak=None):
    """SYNTHE line opacity and spectrum on a synthetic case (CUDA events in the
    library, second run of each precision): line-depth evaluations per second
    of the line-opacity kernels (binning and continuum excluded) in mixed
    precision and all-FP64, and the spectrum's two JOSH solves per lambda.
    Rooflines (mixed precision): the core pass against the FP64 pipe (counted
    Weideman evaluations x 278 flop), and the far-wing gather's bin updates
    per second."""
    from atlas12_b200 import _lib, synthe, synthetic
    case = synthetic.synthe_case(nlines=nlines, wlbeg=wlbeg, wlend=wlend, seed=seed, mol_frac=mol_frac)
    S = synthe.Synthe(ctx, ops)
    out = {"lines": nlines, "depths": 72, "window_nm": [wlbeg, wlend], "resolu": case["resolu"]}
    res = {}
    for name, prec in (("mixed", _lib.PREC_MIXED), ("fp64", _lib.PREC_FP64)):
        ctx.set_precision(prec)
        S.run(case)
        ctx.enable_timing(True)
        _, flux, _, op = S.run(case)
        res[name] = (flux, op)
        ms = {k: ctx.kernel_ms(k) for k in ("synthe_core", "synthe_farfill", "synthe_farwing", "josh_spectrum")}
        work = {k: ctx.kernel_work(k) for k in ("synthe_voigt_evals", "synthe_farwing_updates",
                                                "synthe_farwing_expansions", "synthe_farwing_direct_pairs")}
        ctx.enable_timing(False)
        line_ms = ms["synthe_core"] + ms["synthe_farfill"] + ms["synthe_farwing"]
        out[name] = {"line_depth_evals_per_s": nlines * 72 / (line_ms * 1e-3), "line_opacity_ms": line_ms,
                     "spectrum_ms": ms["josh_spectrum"], "kernel_ms": ms, "work": work}
        out["points"] = int(flux.size)
    ctx.set_precision(_lib.PREC_MIXED)
    out["mixed_vs_fp64_line_opacity"] = out["fp64"]["line_opacity_ms"] / out["mixed"]["line_opacity_ms"]
    # mixed precision against the all-FP64 GPU path (which matches the FP64 oracle to ~1e-12)
    (fm, om), (f64, o64) = res["mixed"], res["fp64"]
    cont = S.continuum(case["wledge"], case["continall"], synthe.synthe_grid(wlbeg, wlend, case["resolu"]))
    out["mixed_error_vs_fp64"] = {
        "kappa_line_max_rel_to_kappa_plus_cont": float(np.max(np.abs(om.astype(np.float64) - o64) /
                                                              (o64.astype(np.float64) + cont))),
        "flux_max_rel": float(np.max(np.abs(fm - f64) / np.abs(f64)))}
    m = out["mixed"]
    tag = f"{nlines // 1000000}M lines" if nlines >= 1000000 else f"{nlines // 1000}k lines"
    rl = []
    if m["work"]["synthe_voigt_evals"] > 0 and m["kernel_ms"]["synthe_core"] > 0:
        ach = m["work"]["synthe_voigt_evals"] * WEIDEMAN_FLOP / (m["kernel_ms"]["synthe_core"] * 1e-3) / 1e12
        rl.append({"kernel": f"k_core (SYNTHE Weideman core, {tag})", "bound": "fp64", "unit": "TFLOP/s",
                   "achieved": ach, "peak": fp64_peak, "frac": ach / fp64_peak if fp64_peak else None,
                   "peak_source": "measured DFMA loop on this GPU (atlasgpu_fp64_peak_tflops)",
                   "work": f"{int(m['work']['synthe_voigt_evals'])} Voigt evaluations x {WEIDEMAN_FLOP} flop"})
    if m["work"]["synthe_farwing_updates"] > 0 and m["kernel_ms"]["synthe_farwing"] > 0:
        rl.append({"kernel": f"k_farwing (SYNTHE far-wing gather, {tag})", "bound": "issue",
                   "unit": "bin updates/s",
                   "achieved": m["work"]["synthe_farwing_updates"] / (m["kernel_ms"]["synthe_farwing"] * 1e-3),
                   "work": f"{int(m['work']['synthe_farwing_updates'])} far-wing bin updates (x/n^2 terms): "
                           f"{int(m['work']['synthe_farwing_expansions'])} (line, 128-bin sub-tile) pairs summed "
                           f"as Taylor expansions, {int(m['work']['synthe_farwing_direct_pairs'])} bin by bin"})
    out["rooflines"] = rl
    return out


def synthe_grid_rate(device, ops, n, lanes=8):
    """Spectra of n atmospheres of the batched-grid workload (own windows of
    5-100 nm at R = 500,000, 0.2-5M lines each): wall time through the public
    API one after another on one context, and on `lanes` contexts (streams)
    at once; spectra per hour both ways, and the largest difference between
    the two runs' fluxes (same arithmetic: 0 up to atomics order)."""
    from atlas12_b200 import synthe, synthe_batch, synthetic
    cases = synthetic.grid_cases(n)
    one = synthe_batch.SyntheBatch(device, ops, lanes=1)
    many = synthe_batch.SyntheBatch(device, ops, lanes=lanes)
    tiny = [synthetic.synthe_case(nlines=2000, wlbeg=500.0, wlend=500.5, seed=3)] * lanes
    one.run(tiny[:1])
    many.run(tiny)
    t0 = time.perf_counter()
    r1 = one.run(cases)
    t1 = time.perf_counter()
    r8 = many.run(cases)
    t2 = time.perf_counter()
    one.close()
    many.close()
    dflux = max(float(np.max(np.abs(a[1] - b[1]) / np.abs(b[1]))) for a, b in zip(r8, r1))
    pts = int(sum(r[1].size for r in r1))
    lines = int(sum(c["lines"]["wlvac"].size for c in cases))
    return {"atmospheres": n, "points": pts, "lines": lines, "lanes": lanes,
            "sequential_s": t1 - t0, "concurrent_s": t2 - t1,
            "spectra_per_hr_sequential": n * 3600.0 / (t1 - t0), "spectra_per_hr_concurrent": n * 3600.0 / (t2 - t1),
            "speedup": (t1 - t0) / (t2 - t1), "max_rel_flux_difference": dflux,
            "timing": "host wall clock around the public API calls (host inputs, host outputs)"}


def cpu_baseline(W, ops_t, starts, step_iters, step_converged, steps=2):
    """The oracle on the host cores on a bounded sample of the same work:
    `steps` reference steps (12 oracle iterations each) of the step's model
    queue from the GPU arm's starting structures, all host threads.  The
    sample gives the oracle's seconds per model iteration; the step's own
    work (the iterations and converged models the GPU arm's step ran, the
    same iteration within the parity tolerances) at that rate gives
    converged models/hr."""
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    q = OracleQueue(W, ops_t, starts)
    q.run(1)  # warm-up
    q = OracleQueue(W, ops_t, starts)
    t0 = time.perf_counter()
    q.run(steps * REF_ITERS_PER_STEP)
    dt = time.perf_counter() - t0
    t_it = dt / (steps * REF_ITERS_PER_STEP)
    v = step_converged * 3600.0 / (t_it * step_iters) if step_iters else 0.0
    _, ncomp, nconv, _, _ = q.rate()
    return {"value": v, "unit": "models/hr", "cores": int(os.environ["OMP_NUM_THREADS"]), "kind": "port",
            "seconds_per_iteration": t_it,
            "sample": f"{steps * REF_ITERS_PER_STEP} oracle iterations of the step's model queue from the same "
                      f"starts ({dt:.1f} s, {t_it:.3f} s per iteration; {ncomp} models completed, {nconv} "
                      f"converged); converged models/hr = the step's {step_converged:g} converged models x 3600 / "
                      f"(its {step_iters:g} model iterations x the oracle's seconds per iteration)"}


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
