#!/usr/bin/env python3
"""bench.py -- converged ATLAS12 models per hour on B200.

Workload (the opacity-sampling configuration the metric is quoted on): one
ATLAS12 model with 30,000 log-spaced frequencies over 9 nm - 160 um, 72
depths, 500,000 synthetic lines (lambda log-uniform, log gf ~ N(-2, 1.5),
E_low ~ U(0, 8) eV, log gamma_rad/Stark/vdW ~ N(8, .3)/N(-5.5, .5)/N(-7.5, .3)),
Teff 5777 K, log g 4.44, vturb 1.5 km/s, iterated from the Eddington grey
start until max |FLXERR| <= 0.1 % (Delta F/F <= 1e-3; cap 60 iterations).
Populations and continuum come from the documented synthetic surrogate.

A step is one model run to convergence; value = converged models/hr (whole
job).  Inputs stay resident in HBM during the timed region; L2 is flushed
between steps.  e2e repeats the measurement through the public API
(atlas12_b200.atlas.AtlasModel) with host buffers: model creation (upload of
the line list, grids and tables), the iterations, and the read-back of the
converged structure are all inside the wall-clock timed region.

--impl reference times the CPU restatement of the same path (oracle/, the
reference's own Fortran cannot be built in this image) on all host threads:
each step is one full iteration; models/hr uses the iteration count the
method needs to converge on this workload.
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

CFG = dict(workload="atlas12-opacity-sampling", numnu=30000, wl_lo=9.0, wl_hi=160000.0, nrhox=72,
           nlines=500000, teff=5777.0, logg=4.44, vturb_kms=1.5, tol_percent=0.1, max_iter=60, seed=2,
           start="eddington-grey")
# iterations the method needs from the grey start on this workload (oracle run, same
# method); used only to turn the reference arm's per-iteration time into models/hr
REF_ITERS_TO_CONVERGE = 40
# FP64 flops counted per frequency in the RT kernel: LU 2/3 51^3, triangular
# solves 2*51^2, system build 2*51^2, J/H/K operators 4*51^2 + 2*51,
# INTEG/MAP1/DERIV and the mode-2 sums ~ 110 per depth (72 depths)
FLOPS_PER_NU = int(2 / 3 * 51 ** 3 + 8 * 51 ** 2 + 2 * 51 + 110 * 72)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP64 GPU comparison")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    return ap.parse_args()


def workload():
    from atlas12_b200 import surrogate, synthetic
    ws, rc = synthetic.geometric_waveset(CFG["wl_lo"], CFG["wl_hi"], CFG["numnu"])
    lines = synthetic.atlas_lines(CFG["nlines"], ws[2], ws[-3], seed=CFG["seed"])
    ross = surrogate.RossTable()
    grey = surrogate.grey_model(CFG["teff"], CFG["logg"], nrhox=CFG["nrhox"], ross=ross)
    return dict(ws=ws, rc=rc, lines=lines, grey=grey, ross=ross)


def operators():
    t = np.load(os.path.join(ROOT, "tests", "golden", "reference_tables.npz"))
    return {k: t[k] for k in t.files}


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


def run_reference(args):
    """CPU restatement of the same path on all host threads."""
    rank, world, local = dist_setup(args)
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    from atlas12_b200 import atlas
    W = workload()
    t = operators()
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    step = oracle_iteration_factory(po, atlas, t, W)
    for _ in range(args.warmup):
        step()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        step()
        times.append(time.perf_counter() - t0)
    t_it = float(np.mean(times))
    v = 3600.0 / (t_it * REF_ITERS_TO_CONVERGE)
    line = {"impl": "reference", "metric": "converged models/hr (dF/F<=1e-3)", "value": v, "unit": "models/hr",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_it * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(CFG, parallelism="host threads", flush="host"),
            "cpu_baseline": {"value": v, "unit": "models/hr", "cores": int(os.environ["OMP_NUM_THREADS"]),
                             "kind": "port",
                             "sample": f"one full ATLAS12 iteration per step (LINOP1 + 30,000-frequency RT pass + "
                                       f"TCORR(3)) on the host; models/hr = 3600 / (t_iteration x "
                                       f"{REF_ITERS_TO_CONVERGE} iterations to convergence)"},
            "e2e": {"value": v, "unit": "models/hr", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def oracle_iteration_factory(po, atlas, tables, W):
    """One ATLAS12 iteration of the oracle on the grey start (state carried)."""
    from atlas12_b200 import surrogate as sg
    ops = po.Ops.from_tables(tables)
    h0, h1, h2 = po.tabvoigt(tables["tabvi"], tables["tabh1"])
    tl = po.build_tablog()
    cut = atlas.cutoff_grid()
    iw = atlas.iwavetab(cut)
    g = W["grey"]
    nr = g["t"].size
    st = dict(t=g["t"].copy(), rhox=g["rhox"].copy(), p=g["p"].copy(), xne=np.zeros(nr), abross=np.zeros(nr),
              prad=np.zeros(nr), vturb=np.full(nr, CFG["vturb_kms"] * 1e5), pturb=np.zeros(nr),
              tauros=g["tauros"].copy(), accrad=np.zeros(nr), raden=np.zeros(nr), oldt1=np.zeros(nr),
              teff=CFG["teff"], grav=g["grav"])
    store = po.RossStore()
    state = {"it": 0, "tabcont": None}

    def step():
        state["it"] += 1
        it = state["it"]
        if it > 1:
            p = st["grav"] * st["rhox"] - st["prad"]
            st["p"] = np.where(p <= 0, np.maximum(st["grav"] * st["rhox"] * 1e-4, 1e-10), p)
        pop = sg.populations(st["t"], st["p"], CFG["vturb_kms"], sg.ATLAS_LINE_POP)
        t = st["t"]
        xd = np.zeros((270, nr))
        dp = np.ones((270, nr))
        xx = np.where(pop["dopple"] > 0, pop["xnfp"] / np.maximum(pop["dopple"], 1e-300) / pop["rho"][:, None], 0.0)
        xd[:] = xx[:, :270].T
        dp[:] = np.where(pop["dopple"][:, :270].T > 0, pop["dopple"][:, :270].T, 1.0)
        hkt = sg.HPLANCK / (sg.KBOL * t)
        hckt = hkt * sg.CLIGHT
        txnxn = (pop["nh"] * (1 - pop["xh"]) + 0.42 * 0.085 * pop["nh"]) * (t / 1e4) ** 0.3
        st["xne"] = pop["xne"]
        if state["tabcont"] is None:
            ka, sgm = sg.continuum_opacity(cut, t, st["p"], pop)
            stc = 1 - np.exp(-(sg.CLIGHT_NMS / cut)[:, None] * hkt[None, :])
            tab = (ka + sgm) * 1e-3 / stc
            state["tabcont"] = np.vstack([tab, tab[-1:]])
        atm = dict(xnfdop=xd, dopple=dp, xne=pop["xne"], txnxn=txnxn, hckt=hckt)
        xl, _ = po.atlas_linop1(h0, h1, h2, tl, W["lines"], atm, state["tabcont"], iw, W["ws"])
        ac, sgm = sg.continuum_opacity(W["ws"], t, st["p"], pop)
        acc, _ = po.atlas_rt_pass(ops, W["ws"], W["rc"], ac, sgm, xl, st["rhox"], t, hkt, CFG["teff"])
        err, st["finish"] = po.atlas_finish(st, acc, it, store)
        return err

    step.state = st
    return step


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
    g = W["grey"]
    ctx = _lib.Context(local, _lib.PREC_MIXED, stream=stream.cuda_stream)
    model = atlas.AtlasModel(ctx, ops, teff=CFG["teff"], logg=CFG["logg"], vturb=CFG["vturb_kms"],
                             linedata=W["lines"], waveset=W["ws"], rcoset=W["rc"], start=g)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def one_model(graph=True):
        model.set_structure(g["t"], g["p"], g["rhox"])
        return model.iterate(max_iter=CFG["max_iter"], tol_percent=CFG["tol_percent"], graph=graph)

    for _ in range(max(args.warmup, 1)):
        one_model()
    iters, converged = [], 0
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    total_ms = 0.0
    clocks = Clocks(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    l0 = ctx.launches()
    for _ in range(args.steps):
        flush.zero_()  # L2 flush between models (256 MB > 126 MB L2)
        ev0.record(stream)
        n, hist = one_model()
        ev1.record(stream)
        torch.cuda.synchronize()
        total_ms += ev0.elapsed_time(ev1)
        iters.append(n)
        converged += int(n > 0 and hist[-1] <= CFG["tol_percent"])
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

    # per-kernel times of one iteration (non-graph, CUDA events in the library)
    ctx.enable_timing(True)
    model.set_structure(g["t"], g["p"], g["rhox"])
    model.iterate(max_iter=3, tol_percent=0.0, graph=False)
    kms = {k: ctx.kernel_ms(k) for k in ("model_eos", "model_kapp", "atlas_linop", "atlas_rt", "atlas_reduce",
                                        "atlas_finish")}
    ctx.enable_timing(False)
    fp64_peak = float(_lib.lib().atlasgpu_fp64_peak_tflops(ctx.handle))

    # plain FP64 GPU path: same method, FP64 everywhere, one launch at a time, grey start
    plain = None
    if not args.no_plain:
        ctx.set_precision(_lib.PREC_FP64)
        one_model(graph=False)
        pm, pi = 0.0, []
        for _ in range(min(args.steps, 3)):
            flush.zero_()
            ev0.record(stream)
            n, hist = one_model(graph=False)
            ev1.record(stream)
            torch.cuda.synchronize()
            pm += ev0.elapsed_time(ev1)
            pi.append(n)
        ctx.set_precision(_lib.PREC_MIXED)
        plain = {"value": 3600.0 * len(pi) / (pm / 1e3), "unit": "models/hr", "ms_per_model": pm / len(pi),
                 "iterations": float(np.mean(pi)), "path": "FP64, per-launch host loop, grey start"}

    # e2e through the public API, host buffers in and out
    e2e_s = 0.0
    h2d = W["lines"].nbytes + W["ws"].nbytes + W["rc"].nbytes + 361 * 8 + 3 * 2001 * 8 + 4 * CFG["nrhox"] * 8
    d2h = 5 * CFG["nrhox"] * 8 + CFG["numnu"] * 8
    ne2e = max(1, min(args.steps, 3))
    for _ in range(ne2e):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        m2 = atlas.AtlasModel(ctx, ops, teff=CFG["teff"], logg=CFG["logg"], vturb=CFG["vturb_kms"],
                              linedata=W["lines"], waveset=W["ws"], rcoset=W["rc"], start=g)
        m2.iterate(max_iter=CFG["max_iter"], tol_percent=CFG["tol_percent"], graph=True)
        m2.structure()
        torch.cuda.synchronize()
        e2e_s += time.perf_counter() - t0
        m2.close()
    e2e_all = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(e2e_all, op=dist.ReduceOp.MAX)
    e2e_value = world * ne2e * 3600.0 / float(e2e_all.item())

    # roofline of the dominant kernel
    dom = max((k for k in kms if kms[k] > 0), key=lambda k: kms[k])
    if dom == "atlas_rt":
        ach = CFG["numnu"] * FLOPS_PER_NU / (kms[dom] * 1e-3) / 1e12
        roof = {"kernel": "k_atlas_rt", "bound": "fp64", "achieved": ach, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": ach / fp64_peak if fp64_peak > 0 else None, "traffic": None,
                "peak_source": "measured DFMA loop (atlasgpu_fp64_peak_tflops)",
                "work": f"{FLOPS_PER_NU} FP64 flop per frequency x {CFG['numnu']}"}
    else:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
            os.path.join(ROOT, "MEASURED_PEAKS.json")) else {"hbm_gbs": 6650.0}
        byts = CFG["nlines"] * 16 + CFG["nrhox"] * CFG["numnu"] * 8
        ach = byts / (kms[dom] * 1e-3) / 1e9
        roof = {"kernel": dom, "bound": "hbm", "achieved": ach, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": ach / peaks["hbm_gbs"], "traffic": None,
                "work": "16 B per LINEDATA record + 8 B per XLINES element"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(W, ops, float(np.mean(iters)))
    if rank == 0:
        line = {"metric": "converged models/hr (dF/F<=1e-3)", "value": value, "unit": "models/hr",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded lines, surrogate populations/continuum)",
                "config": dict(CFG, parallelism=f"replicas x{world}", l2="flushed between steps (256 MB write)"),
                "iterations_to_converge": float(np.mean(iters)), "converged": int(conv_all.item()),
                "kernel_ms_per_iteration": kms, "roofline": roof, "cpu_baseline": cpu,
                "plain_fp64": plain, "vs_plain_fp64": (value / plain["value"]) if plain else None,
                "e2e": {"value": e2e_value, "unit": "models/hr", "h2d_bytes_per_step": int(h2d),
                        "d2h_bytes_per_step": int(d2h)},
                "gpu_launches": int(gpu_launches), "clocks": clk}
        print(json.dumps(line), flush=True)
    model.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def cpu_baseline(W, ops_t, iters_gpu):
    """The oracle on the host: two iterations of the same model, all host threads."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    from atlas12_b200 import atlas
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    step = oracle_iteration_factory(po, atlas, ops_t, W)
    step()
    t0 = time.perf_counter()
    step()
    t_it = time.perf_counter() - t0
    return {"value": 3600.0 / (t_it * iters_gpu), "unit": "models/hr", "cores": int(os.environ["OMP_NUM_THREADS"]),
            "kind": "port",
            "sample": f"one ATLAS12 iteration of this model on the host ({t_it:.2f} s), models/hr for the "
                      f"{iters_gpu:.1f} iterations the GPU run needed"}


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
