"""Benchmark: SIMPLE outer iterations/s (+ assembled elements/s) on the
128^3 skewed lid-driven cavity (2.1M hex8, interior nodes displaced by
U(-0.2h, 0.2h), Gaussian initial velocity sigma 0.1, seeded), mixed FP32/FP64
form against the plain FP64 GPU form.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one SIMPLE outer iteration (momentum assembly + solve, mass-flow
update, pressure-correction assembly + solve to rtol 1e-8, corrections,
gradients). Inputs are generated on the host, uploaded once, and the timed
region runs with every field resident in HBM (working set > L2, so no flush).
With N > 1 (torchrun) every rank runs an independent replica: the path has no
exchange step at this size ("replicas only").
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

HBM_FALLBACK = 6650.0


def max_over_ranks(value, device, world):
    """The largest of every rank's value (time-like measurements are reported
    as the slowest rank's); identity for one process."""
    if world <= 1:
        return value
    import torch

    t = torch.tensor([float(value)], device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return HBM_FALLBACK, "fallback"


class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                self.samples.append([v.strip() for v in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            try:
                sm.append(float(s[0]))
                smax = max(smax, float(s[1]))
                for n, v in zip(names, s[3:7]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def workload(n):
    from openaccel_b200 import meshgen

    m = meshgen.cavity(n, perturb=0.2, seed=12345)
    U0 = meshgen.initial_velocity(m, sigma=0.1, seed=12345)
    return m, U0


def algorithmic_bytes_momentum(nn, ne, nnz, mixed):
    """Algorithmic bytes of one momentum assembly: nodal inputs
    13 doubles (x3, U3, mu, rho, V, grad p3, div) = 104 B/node; element inputs
    32 B connectivity + 96 B mDot; outputs 3x3 blocks + rhs + DU."""
    val = 4 if mixed else 8
    return 104 * nn + 128 * ne + 9 * val * nnz + 3 * val * nn + 24 * nn


def run_ours(args, rank, world):
    import torch

    from openaccel_b200 import runtime as rt

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    m, U0 = workload(args.n)
    gm = rt.Mesh(m)

    def make(prec):
        # both forms run the same graph mode (default: each outer iteration as
        # one CUDA graph), so the ratio of the two measures precision, not
        # launch overhead
        f = rt.Flow(gm, rt.default_settings(precision=prec, pc_rtol=args.pc_rtol, mom_rtol=args.mom_rtol,
                                            mom_maxit=args.mom_maxit, use_graphs=graph_mode(args)))
        f.set_field("U", U0)
        f.initialize()
        if not args.no_autotune:
            # set-up, not timed: the flow's state is restored afterwards
            tuning[prec] = f.autotune(iters=3)
        return f

    tuning = {}

    def timed(f, steps, warmup):
        stream = torch.cuda.ExternalStream(f.stream_handle(), device=dev)
        stats = []
        for _ in range(warmup):
            stats += f.simple_iterate(1)
        f.sync()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = rt.launch_count()
        e0.record(stream)
        for _ in range(steps):
            stats += f.simple_iterate(1)
        e1.record(stream)
        e1.synchronize()
        launches = rt.launch_count() - l0
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        ms = max_over_ranks(ms, dev, world)
        return ms, stats, launches

    # mixed form: headline
    fm = make(rt.OA_PREC_MIXED)
    with ClockSampler(dev.index) as clk:
        ms_mixed, st_mixed, launches = timed(fm, args.steps, args.warmup)
    if args.only_mixed:  # profiling runs: the mixed form's timed steps only
        return {"metric": "SIMPLE outer iters/s (mixed form only)", "value": world * args.steps / (ms_mixed * 1e-3),
                "unit": "outer_iters/s", "steps": args.steps, "ms_per_step": ms_mixed / args.steps,
                "gpu_launches": launches, "pc_iters_last": st_mixed[-1]["pc_iters"]}
    # FP64 form: same workload, same steps
    f64 = make(rt.OA_PREC_FP64)
    ms_64, st_64, _ = timed(f64, args.steps, args.warmup)

    # kernel timing for the roofline and elements/s (CUDA events on the flow stream)
    t_mom = fm.time_kernel("momentum", reps=5)
    t_pc = fm.time_kernel("pcorr", reps=5)
    t_mom64 = f64.time_kernel("momentum", reps=5)
    t_pc64 = f64.time_kernel("pcorr", reps=5)

    # e2e: public API with pinned host buffers, copies inside the timed region
    fe = make(rt.OA_PREC_MIXED)
    Uh = torch.empty(3 * m.nn, dtype=torch.float64, pin_memory=True)
    ph = torch.empty(m.nn, dtype=torch.float64, pin_memory=True)
    Uh.copy_(torch.from_numpy(U0.ravel()))
    ph.zero_()
    import ctypes as C

    L = rt.lib()
    dp = C.POINTER(C.c_double)

    def e2e_step():
        rt._check(L.oa_flow_set_field(fe.h, b"U", C.cast(Uh.data_ptr(), dp), Uh.numel()))
        rt._check(L.oa_flow_set_field(fe.h, b"p", C.cast(ph.data_ptr(), dp), ph.numel()))
        fe.simple_iterate(1)
        rt._check(L.oa_flow_get_field(fe.h, b"U", C.cast(Uh.data_ptr(), dp), Uh.numel()))
        rt._check(L.oa_flow_get_field(fe.h, b"p", C.cast(ph.data_ptr(), dp), ph.numel()))

    for _ in range(args.warmup):
        e2e_step()
    stream_e = torch.cuda.ExternalStream(fe.stream_handle(), device=dev)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream_e)
    for _ in range(args.steps):
        e2e_step()
    e1.record(stream_e)
    e1.synchronize()
    ms_e2e = e0.elapsed_time(e1)
    ms_e2e = max_over_ranks(ms_e2e, dev, world)

    conv = converge(args, gm, U0, dev, world, tuning) if args.converge_iters > 0 else None

    peak, peak_kind = measured_peaks()
    alg = algorithmic_bytes_momentum(m.nn, m.ne, gm.nnz, True)
    achieved = alg / (t_mom * 1e-3) / 1e9
    value = world * args.steps / (ms_mixed * 1e-3)
    value64 = world * args.steps / (ms_64 * 1e-3)
    res = {
        "metric": "SIMPLE outer iters/s (mixed FP32/FP64 form; FP64 form and assembled elems/s beside it)",
        "value": value,
        "unit": "outer_iters/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_mixed / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32+f64",
        "data": "synthetic",
        "config": cavity_config(args, args.n, m.ne, m.nn, gm.nnz, world),
        "fp64_outer_iters_per_s": value64,
        "graphs": GRAPH_MODES[graph_mode(args)],
        "autotune": {("mixed" if k == rt.OA_PREC_MIXED else "fp64"): v for k, v in tuning.items()} or "off",
        "mixed_over_fp64": value / value64,
        "assembled_elems_per_s": {"mixed": 2 * m.ne / ((t_mom + t_pc) * 1e-3),
                                  "fp64": 2 * m.ne / ((t_mom64 + t_pc64) * 1e-3)},
        "kernel_ms": {"momentum_mixed": t_mom, "pcorr_mixed": t_pc, "momentum_fp64": t_mom64,
                      "pcorr_fp64": t_pc64},
        "continuity_rms_last": {"mixed": st_mixed[-1]["continuity_rms"], "fp64": st_64[-1]["continuity_rms"]},
        "phase_ms_per_step": {form: {k[3:]: float(np.mean([x[k] for x in st[-args.steps:]])) for k in rt.PHASES}
                              for form, st in (("mixed", st_mixed), ("fp64", st_64))},
        "pc_iters_last": {"mixed": st_mixed[-1]["pc_iters"], "fp64": st_64[-1]["pc_iters"]},
        "pc_krylov": "GCR(2) with the AMG V-cycle (one V-cycle per iteration)",
        "roofline": {"bound": "hbm", "kernel": "k_momentum (mixed)", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                     "algorithmic_bytes": alg, "traffic": None,
                     "traffic_ncu": "not measured in this run; per-launch DRAM bytes of an ncu capture of the same "
                                    "kernel are in profiles/"},
        "converge": conv,
        "e2e": {"value": world * args.steps / (ms_e2e * 1e-3), "unit": "outer_iters/s",
                "h2d_bytes_per_step": 32 * m.nn, "d2h_bytes_per_step": 32 * m.nn},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    return res


def converge(args, gm, U0, dev, world, tuning=None):
    """Both forms from the same initial state for up to --converge-iters SIMPLE
    outer iterations (or until the continuity residual, RMS of the nodal mass
    imbalance / (rho U_lid h^2), falls to --converge-target). Device time of
    every iteration on the flow's stream (CUDA events); the first iteration,
    which also builds the AMG hierarchy on the host, is run untimed. Reports
    the time each form needs to reach the smallest residual both reach (the
    target when both get there), their ratio, and the mixed form's field error
    against the FP64 form after the same number of iterations."""
    import torch

    from openaccel_b200 import runtime as rt

    out = {}
    fields = {}
    for name, prec in (("mixed", rt.OA_PREC_MIXED), ("fp64", rt.OA_PREC_FP64)):
        f = rt.Flow(gm, rt.default_settings(precision=prec, pc_rtol=args.pc_rtol, mom_rtol=args.mom_rtol,
                                            mom_maxit=args.mom_maxit, use_graphs=graph_mode(args)))
        f.set_field("U", U0)
        f.initialize()
        if tuning and prec in tuning:  # the timed legs' tuning
            f.set_tuning(**tuning[prec])
        stream = torch.cuda.ExternalStream(f.stream_handle(), device=dev)
        # iteration 1 builds the pressure solve's AMG hierarchy on the host
        # (about 1.8 s at 128^3, the same in both forms): run it untimed
        st = f.simple_iterate(1)[0]
        res, t = [st["continuity_rms"]], [0.0]
        for _ in range(args.converge_iters - 1):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st = f.simple_iterate(1)[0]
            e1.record(stream)
            e1.synchronize()
            t.append(e0.elapsed_time(e1))
            res.append(st["continuity_rms"])
            if st["continuity_rms"] <= args.converge_target:
                break
        fields[name] = (f.get_field("U"), f.get_field("p"), len(res))
        out[name] = {"iters": len(res), "residual_first": res[0], "residual_last": res[-1], "residual_min": min(res),
                     "ms_total": float(np.sum(t)), "cum_ms": np.cumsum(t), "res": np.array(res)}
        f.close()
    target = max(args.converge_target, out["mixed"]["residual_min"], out["fp64"]["residual_min"])
    summary = {"target": args.converge_target, "max_iters": args.converge_iters,
               "residual_definition": "RMS over nodes of the pressure-correction rhs before the solve / (rho U_lid h^2), "
                                      "h = mean element edge length",
               "common_residual": target, "timed_from_iteration": 2}
    t_to = {}
    for name, o in out.items():
        k = int(np.argmax(o["res"] <= target))
        t_to[name] = float(o["cum_ms"][k])
        summary[name] = {"iters_run": o["iters"], "residual_first": o["residual_first"],
                         "residual_last": o["residual_last"], "iters_to_common": k + 1, "ms_to_common": t_to[name],
                         "ms_per_iter": o["ms_total"] / max(o["iters"] - 1, 1)}
    summary["time_to_residual_ratio_fp64_over_mixed"] = t_to["fp64"] / t_to["mixed"]
    (Um, pm, nm), (Ud, pd, nd) = fields["mixed"], fields["fp64"]
    if nm == nd:
        summary["field_err_mixed_vs_fp64"] = {
            "iters": nm, "U": float(np.abs(Um - Ud).max() / np.abs(Ud).max()),
            "p": float(np.abs(pm - pd).max() / max(np.abs(pd).max(), 1e-300))}
    return summary


def algorithmic_bytes_diffusion(nn, ne, nnz, mixed):
    """Algorithmic bytes of one tet4 diffusion assembly: nodal inputs x3, phi,
    Gamma, source, dual volume (56 B/node), 16 B connectivity per element,
    outputs the CSR values and the FP64 rhs."""
    val = 4 if mixed else 8
    return 56 * nn + 16 * ne + val * nnz + 8 * nn


def run_conduction(args, rank, world):
    """tet4 conduction (96^3 x 6 Kuhn tets, lognormal Gamma sigma 1, U[0,1]
    source, T = 0 / 1 on x = 0 / 1): a step is one thermal-equation step
    (assembly, BiCGStab-AMG to 1e-10, clipped correction) from T = 0."""
    import torch

    from openaccel_b200 import meshgen
    from openaccel_b200 import runtime as rt

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    m, gam, src, _ = meshgen.conduction(args.n, sigma=1.0, seed=4242)
    gm = rt.Mesh(m)

    def make(prec):
        d = rt.Diffusion(gm, rt.default_diffusion_settings(precision=prec, rtol=args.diff_rtol,
                                                           use_graphs=graph_mode(args)))
        d.set_field("gamma", gam)
        d.set_field("src", src)
        return d

    zero = np.zeros(m.nn)

    def timed(d, steps, warmup):
        stream = torch.cuda.ExternalStream(d.stream_handle(), device=dev)
        for _ in range(warmup):
            d.set_field("phi", zero)
            d.step()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        total, stats, launches = 0.0, [], 0
        for _ in range(steps):
            d.set_field("phi", zero)  # every step solves the same first step
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            l0 = rt.launch_count()
            e0.record(stream)
            stats.append(d.step())
            e1.record(stream)
            e1.synchronize()
            launches += rt.launch_count() - l0
            total += e0.elapsed_time(e1)
        total = max_over_ranks(total, dev, world)
        return total, stats, launches

    dm = make(rt.OA_PREC_MIXED)
    with ClockSampler(dev.index) as clk:
        ms_mixed, st_mixed, launches = timed(dm, args.steps, args.warmup)
    d64 = make(rt.OA_PREC_FP64)
    ms_64, st_64, _ = timed(d64, args.steps, args.warmup)
    phi_m, phi_64 = dm.get_field("phi"), d64.get_field("phi")
    t_asm = dm.time_assembly(reps=10)
    t_asm64 = d64.time_assembly(reps=10)
    peak, peak_kind = measured_peaks()
    alg = algorithmic_bytes_diffusion(m.nn, m.ne, gm.nnz, True)
    achieved = alg / (t_asm * 1e-3) / 1e9
    value = world * args.steps / (ms_mixed * 1e-3)
    value64 = world * args.steps / (ms_64 * 1e-3)
    return {
        "metric": "tet4 conduction steps/s (assembly + Krylov to 1e-10, mixed FP32/FP64 form)",
        "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_mixed / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": f"conduction {args.n}^3 hex -> 6 tet4 (Kuhn), lognormal Gamma sigma 1, U[0,1] source",
                   "elements": m.ne, "nodes": m.nn, "nnz": gm.nnz, "rtol": args.diff_rtol,
                   "l2": "inputs larger than L2 (no flush)", "parallelism": f"replicas x{world}"},
        "fp64_steps_per_s": value64, "mixed_over_fp64": value / value64,
        "mixed_vs_fp64_field_maxrel": float(np.abs(phi_m - phi_64).max() / np.abs(phi_64).max()),
        "assembled_elems_per_s": {"mixed": m.ne / (t_asm * 1e-3), "fp64": m.ne / (t_asm64 * 1e-3)},
        "kernel_ms": {"assembly_mixed": t_asm, "assembly_fp64": t_asm64},
        "krylov_iters": {"mixed": st_mixed[-1]["iters"], "fp64": st_64[-1]["iters"],
                         "refinements_mixed": st_mixed[-1]["refinements"]},
        "roofline": {"bound": "hbm",
                     "kernel": "tet4 diffusion assembly, all passes (k_tet_elem, k_tet_face, k_tet_gather, k_tet_rhs; "
                               "mixed)",
                     "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind, "algorithmic_bytes": alg,
                     "traffic": None},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }


def run_batch(args, rank, world):
    """64 independent unit-cube cavities (edge counts U{16..64}, viscosities
    log-uniform 1e-3..1e-1, seeded): one outer iteration of all of them per
    step. The batched form assembles and solves the whole batch as one
    disjoint-union system (one launch per kernel, mixed precision, Krylov
    chunks replayed as CUDA graphs); the baseline loops over the cavities with
    the plain FP64 form, one flow per cavity."""
    import torch

    from openaccel_b200 import meshgen
    from openaccel_b200 import runtime as rt

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    bt = meshgen.batch_cavities(count=args.batch_count, seed=2024)
    kw = dict(pc_rtol=args.pc_rtol, mom_rtol=args.mom_rtol, mom_maxit=args.mom_maxit)
    gm = rt.Mesh(bt.mesh)
    fb = rt.Flow(gm, rt.default_settings(precision=rt.OA_PREC_MIXED, ref_node=-1,
                                         use_graphs=graph_mode(args), **kw))
    fb.set_field("mu", bt.mu)
    fb.set_reference_nodes(bt.ref_nodes)
    fb.initialize()
    singles = []
    for m, n in enumerate(bt.sizes):
        c = meshgen.cavity(int(n))
        g1 = rt.Mesh(c)
        f1 = rt.Flow(g1, rt.default_settings(mu=float(bt.viscosities[m]), precision=rt.OA_PREC_FP64, **kw))
        f1.initialize()
        singles.append((g1, f1))

    def timed(step, streams, steps, warmup):
        for _ in range(warmup):
            step()
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = rt.launch_count()
        e0.record(streams[0])
        for _ in range(steps):
            step()
        # the last work of a step may sit on any flow's stream: join them all
        for st in streams[1:]:
            ev = torch.cuda.Event()
            ev.record(st)
            streams[0].wait_event(ev)
        e1.record(streams[0])
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        ms = max_over_ranks(ms, dev, world)
        return ms, rt.launch_count() - l0

    sb = [torch.cuda.ExternalStream(fb.stream_handle(), device=dev)]
    with ClockSampler(dev.index) as clk:
        stats = []
        ms_b, launches = timed(lambda: stats.extend(fb.simple_iterate(1)), sb, args.steps, args.warmup)
    ss = [torch.cuda.ExternalStream(f.stream_handle(), device=dev) for _, f in singles]
    ms_l, launches_l = timed(lambda: [f.simple_iterate(1) for _, f in singles], ss, args.steps, args.warmup)
    value = world * args.steps / (ms_b * 1e-3)
    value_l = world * args.steps / (ms_l * 1e-3)
    return {
        "metric": "batched SIMPLE outer iters/s (all cavities of the batch per iteration, mixed form, one launch "
                  "per kernel) against a loop over the plain FP64 form",
        "value": value, "unit": "batch_outer_iters/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_b / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": f"{args.batch_count} unit-cube cavities, edges U{{16..64}}, mu logU[1e-3,1e-1], seed 2024",
                   "nodes": bt.mesh.nn, "elements": bt.mesh.ne, "pc_rtol": args.pc_rtol, "mom_rtol": args.mom_rtol,
                   "l2": "inputs larger than L2 (no flush)", "parallelism": f"replicas x{world}"},
        "loop_fp64_batch_iters_per_s": value_l, "batched_over_loop": value / value_l,
        "gpu_launches": launches, "gpu_launches_loop": launches_l,
        "pc_iters_last": stats[-1]["pc_iters"], "continuity_rms_last": stats[-1]["continuity_rms"],
        "clocks": clk.summary(),
    }


def run_sst(args, rank, world):
    """Fused k-omega SST node kernel (turbulent viscosity, F1, production, k and
    omega node terms) on the 256 x 96 x 96 channel's node count (2,418,113
    nodes) with seeded fields in the ranges of that case; a step is one launch."""
    import torch

    from openaccel_b200 import runtime as rt

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    nn = 257 * 97 * 97
    rng = np.random.default_rng(3)
    host = dict(k=1e-3 * np.exp(0.2 * rng.standard_normal(nn)), omega=1e2 * np.exp(0.2 * rng.standard_normal(nn)),
                rho=np.ones(nn), mu=np.full(nn, 1e-5), ymin=rng.uniform(1e-5, 0.5, nn),
                gradU=rng.normal(0, 10, 9 * nn), gradK=rng.normal(0, 1e-3, 3 * nn), gradW=rng.normal(0, 10, 3 * nn),
                div=rng.normal(0, 1e-6, nn), vol=np.full(nn, 1.0 / nn), mut_old=np.zeros(nn))
    host["k_prev"] = host["k"].copy()
    d = {n: torch.from_numpy(v).to(dev) for n, v in host.items()}
    d["wall_node"] = torch.from_numpy((rng.uniform(size=nn) < 0.02).astype(np.int32)).to(dev)
    for n in rt.SST_OUTPUTS:
        d[n] = torch.empty(nn, dtype=torch.float64, device=dev)
    ptrs = {n: t.data_ptr() for n, t in d.items()}
    stream = torch.cuda.current_stream(dev)
    for _ in range(args.warmup):
        rt.sst_node_update(nn, ptrs, stream=stream.cuda_stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = rt.launch_count()
    with ClockSampler(dev.index) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            rt.sst_node_update(nn, ptrs, stream=stream.cuda_stream)
        e1.record(stream)
        e1.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), dev, world)
    # algorithmic bytes: 9 scalars + grad U (9) + grad k (3) + grad omega (3)
    # doubles and a wall flag in, 7 doubles out (no wall production supplied)
    alg = nn * (8 * (9 + 9 + 3 + 3) + 4 + 8 * 7)
    t = ms * 1e-3 / args.steps
    peak, peak_kind = measured_peaks()
    return {
        "metric": "SST node updates per second (fused mu_t, F1, P_k, k/omega node terms)", "value": world / t,
        "unit": "launches/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "SST node kernel, 257 x 97 x 97 nodes (256 x 96 x 96 channel)", "nodes": nn,
                   "l2": "inputs larger than L2 (no flush)"},
        "roofline": {"bound": "hbm", "kernel": "k_sst_nodes", "achieved": alg / t / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": alg / t / 1e9 / peak, "peak_kind": peak_kind, "algorithmic_bytes": alg,
                     "traffic": None},
        "gpu_launches": rt.launch_count() - l0, "clocks": clk.summary(),
    }


def run_channel(args, rank, world):
    """Fused u/v/w/k/omega assembly on the 256 x 96 x 96 channel mesh (y
    stretched 1.05 from both walls, no-slip y walls, symmetry planes at the
    spanwise z faces; the inlet and outlet planes are no-slip walls standing in
    for the channel's inlet/outlet conditions), mu = 1e-5, k0 = 1e-3 LN(0.2), omega0 = 1e2
    LN(0.2) seeded, diffusivities mu + sigma mu_t with mu_t = rho k / omega and
    the SST inner-layer sigmas. A step is one assembly launch of all five
    equations; the momentum-only launch is timed beside it, and whole outer
    iterations with the SST equations (oa_flow_sst_iterate) are reported."""
    import torch

    from openaccel_b200 import meshgen
    from openaccel_b200 import runtime as rt

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    m = meshgen.channel(256, 96, 96, ratio=1.05)
    rng = np.random.default_rng(7)
    k = 1e-3 * np.exp(0.2 * rng.standard_normal(m.nn))
    w = 1e2 * np.exp(0.2 * rng.standard_normal(m.nn))
    mu, mut = 1e-5, k / w
    U0 = meshgen.initial_velocity(m, sigma=0.1, seed=7)
    gm = rt.Mesh(m)
    out = {}
    for prec, name in ((rt.OA_PREC_MIXED, "mixed"), (rt.OA_PREC_FP64, "fp64")):
        f = rt.Flow(gm, rt.default_settings(precision=prec, pc_rtol=args.pc_rtol, mom_rtol=args.mom_rtol,
                                            mom_maxit=args.mom_maxit))
        f.set_boundary_types([rt.OA_BTYPE_WALL, rt.OA_BTYPE_WALL, rt.OA_BTYPE_SYMMETRY])
        f.set_field("U", U0)
        f.set_field("mu", np.full(m.nn, mu))
        f.initialize()
        f.simple_iterate(1)  # a mass-flow field of the flow
        t_plain = f.time_kernel("momentum", reps=args.steps)
        f.enable_turbulence(0.8, 0.8)
        for n, v in (("k", k), ("omega", w), ("gammaK", mu + 0.85 * mut), ("gammaOmega", mu + 0.5 * mut)):
            f.set_field(n, v)
        l0 = rt.launch_count()
        with ClockSampler(dev.index) as clk:
            t_fused = f.time_kernel("momentum", reps=args.steps)
        out[name] = {"ms_fused": t_fused, "ms_momentum_only": t_plain, "launches": rt.launch_count() - l0,
                     "clocks": clk.summary()}
        # whole outer iterations with the SST equations (oa_flow_sst_iterate:
        # flow iteration with the fused launch, k/omega solves, gradients,
        # node update, diffusivities), CUDA events on the flow's stream
        y = m.coords[:, 1]
        sst_in = {"ymin": torch.from_numpy(np.minimum(y, 1.0 - y) + 1e-4).to(dev),
                  "wall": torch.from_numpy((np.isclose(y, 0.0) | np.isclose(y, 1.0)).astype(np.int32)).to(dev),
                  "mu": torch.full((m.nn,), mu, dtype=torch.float64, device=dev)}
        sst_args = (sst_in["ymin"].data_ptr(), sst_in["wall"].data_ptr(), sst_in["mu"].data_ptr())
        try:
            f.sst_iterate(1, *sst_args, mut_urf=0.7, rtol=1e-6)
            stream = torch.cuda.ExternalStream(f.stream_handle(), device=dev)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            n_sst = 3
            e0.record(stream)
            sst_stats = f.sst_iterate(n_sst, *sst_args, mut_urf=0.7, rtol=1e-6)
            e1.record(stream)
            e1.synchronize()
            out[name]["sst_outer_iteration_ms"] = e0.elapsed_time(e1) / n_sst
            out[name]["sst_pc_iters"] = [st["pc_iters"] for st in sst_stats]
            # the flow's phases inside it (event nodes); the rest is the k / omega
            # solves and corrections, their gradients, the node update and the
            # diffusivities
            phases = {k[3:]: sum(st[k] for st in sst_stats) / n_sst for k in rt.PHASES}
            out[name]["sst_phase_ms"] = dict(phases, turbulence=out[name]["sst_outer_iteration_ms"] - sum(phases.values()))
        except rt.OpenAccelError as exc:
            out[name]["sst_outer_iteration_error"] = str(exc)
        f.close()
    ms = max_over_ranks(out["mixed"]["ms_fused"], dev, world)
    ne, nn, nnz = m.ne, m.nn, gm.nnz
    # algorithmic bytes of the fused launch (mixed): the momentum assembly's, plus
    # k, omega, two diffusivities and four node sources in (64 B/node) and two
    # FP32 scalar systems out
    alg = algorithmic_bytes_momentum(nn, ne, nnz, True) + 64 * nn + 2 * (4 * nnz + 4 * nn)
    peak, peak_kind = measured_peaks()
    return {
        "metric": "assembled elems/s, u/v/w/k/omega in one fused launch (element-equations per second)",
        "value": world * 5 * ne / (ms * 1e-3), "unit": "elem_eq/s", "n_gpus": world, "steps": args.steps,
        "warmup": 1, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": "channel 256x96x96 hex8, wall-normal stretching 1.05, mu 1e-5, k/omega lognormal",
                   "elements": ne, "nodes": nn, "nnz": nnz, "l2": "inputs larger than L2 (no flush)",
                   "boundaries": "no-slip y walls, symmetry z planes, x planes no-slip (inlet/outlet not modelled)",
                   "pc_rtol": args.pc_rtol, "mom_rtol": args.mom_rtol, "mom_maxit": args.mom_maxit},
        "fused": out,
        "fused_over_momentum_only": {p: out[p]["ms_fused"] / out[p]["ms_momentum_only"] for p in out},
        "roofline": {"bound": "hbm", "kernel": "k_momentum (fused u/v/w/k/omega, mixed)", "achieved": alg / ms / 1e6,
                     "peak": peak, "unit": "GB/s", "frac": alg / ms / 1e6 / peak, "peak_kind": peak_kind,
                     "algorithmic_bytes": alg, "traffic": None},
        "gpu_launches": out["mixed"]["launches"], "clocks": out["mixed"]["clocks"],
    }


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cavity_config(args, n, ne, nn, nnz, world):
    """The config dict of the cavity workload (both arms print the same one)."""
    return {"workload": f"lid-driven cavity {n}^3 hex8 skewed +-20%, Re=100, U0~N(0,0.1)",
            "elements": ne, "nodes": nn, "nnz": nnz, "pc_rtol": args.pc_rtol, "mom_rtol": args.mom_rtol,
            "mom_maxit": args.mom_maxit, "l2": "inputs larger than L2 (no flush)",
            "parallelism": f"replicas x{world}"}


def cpu_sample(args, threads, warmup, steps, budget_s):
    """The oracle (CPU FP64 restatement of the same assembly and SIMPLE
    sequence) on the same workload, with the linear solvers of the reference's
    cavity example in a form that converges here: Krylov preconditioned by
    block-Jacobi ILU(0), one block of contiguous rows per thread as PETSc
    bjacobi / Ifpack2 give one block per MPI rank (examples/cavity/input.i:61-77
    names GMRES; restarted GMRES(50) with the same ILU(0) needed about 20,000
    iterations per pressure solve at 64^3, BiCGStab about 200, so BiCGStab is
    used for both systems). `warmup` untimed outer iterations, then up to
    `steps` timed ones (at least 2, fewer if they would exceed budget_s);
    then one momentum and one pressure-correction assembly timed with all
    threads and with one thread (assembled elements/s)."""
    from oracle import pyoracle as po

    po.set_threads(threads)
    m, U0 = workload(args.cpu_n)
    c = po.FlowCase(m, po.default_settings(pc_rtol=args.pc_rtol, mom_rtol=args.mom_rtol, pc_maxit=20000,
                                           mom_maxit=args.mom_maxit), U0=U0)
    c.set_solver("ilu-bicgstab")
    c.initialize()
    t_w = []
    for _ in range(warmup):
        t0 = time.perf_counter()
        c.simple_iteration()
        t_w.append(time.perf_counter() - t0)
    k = steps
    if t_w:
        k = max(2, min(steps, int(budget_s / max(t_w))))
    t_s, st = [], None
    for _ in range(k):
        t0 = time.perf_counter()
        st = c.simple_iteration()
        t_s.append(time.perf_counter() - t0)
    asm = {}
    for nt in (threads, 1):
        po.set_threads(nt)
        t0 = time.perf_counter()
        c.assemble_momentum()
        t1 = time.perf_counter()
        c.assemble_pcorr()
        t2 = time.perf_counter()
        asm[nt] = (t1 - t0, t2 - t1)
    po.set_threads(threads)
    total = float(np.sum(t_s))
    return {
        "value": k / total, "unit": "outer_iters/s", "cores": threads, "kind": "port", "cpu": cpu_model(),
        "steps": k, "warmup": warmup, "ms_per_step": 1e3 * total / k,
        "sample": f"{k} SIMPLE outer iterations of the {args.cpu_n}^3 workload after {warmup} untimed, FP64 oracle "
                  f"restatement, {threads} host threads; solvers: BiCGStab with block-Jacobi ILU(0) (one block per "
                  "thread) for the momentum and pressure-correction systems",
        "pc_iters_last": st["pc_iters"] if st else None,
        "assembled_elems_per_s": {
            "all_threads": 2 * m.ne / sum(asm[threads]), "one_thread": 2 * m.ne / sum(asm[1]),
            "ms": {"momentum_all_threads": 1e3 * asm[threads][0], "pcorr_all_threads": 1e3 * asm[threads][1],
                   "momentum_one_thread": 1e3 * asm[1][0], "pcorr_one_thread": 1e3 * asm[1][1]}},
        "nnz": c.nnz, "elements": m.ne, "nodes": m.nn,
    }


GRAPH_MODES = {0: "off", 1: "Krylov chunks replayed as CUDA graphs in both forms",
               2: "each outer iteration after the first replayed as one CUDA graph (solver loops as device-side "
                  "conditional nodes) in both forms"}


def graph_mode(args):
    if args.graphs is not None:
        return args.graphs
    return 0 if args.no_graphs else 2


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--cpu-n", type=int, default=128)
    ap.add_argument("--pc-rtol", type=float, default=1e-8)
    # momentum solver settings of the reference's cavity example
    # (examples/cavity/input.i: linear_solver_settings default, rtol 1e-1, 20 iterations)
    ap.add_argument("--mom-rtol", type=float, default=1e-1)
    ap.add_argument("--mom-maxit", type=int, default=20)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-graphs", action="store_true")
    ap.add_argument("--graphs", type=int, default=None, choices=[0, 1, 2],
                    help="0 none, 1 Krylov chunks as CUDA graphs, 2 each outer iteration as one CUDA graph")
    ap.add_argument("--no-autotune", action="store_true", help="skip the launch-shape / solve-schedule autotuning")
    ap.add_argument("--only-mixed", action="store_true", help="time the mixed form only (profiling)")
    ap.add_argument("--workload", default="cavity", choices=["cavity", "conduction", "batch", "sst", "channel"],
                    help="cavity: the headline SIMPLE workload; conduction: the tet4 diffusion case (--n 96); "
                         "batch: 64 independent cavities, batched mixed form against a loop over the FP64 form")
    ap.add_argument("--batch-count", type=int, default=64)
    ap.add_argument("--converge-iters", type=int, default=200,
                    help="outer iterations of the time-to-residual comparison (0: skip it)")
    ap.add_argument("--converge-target", type=float, default=1e-8)
    ap.add_argument("--cpu-budget", type=float, default=120.0,
                    help="seconds of timed CPU outer iterations at most (the CPU baseline's steps are cut to fit)")
    ap.add_argument("--diff-rtol", type=float, default=1e-10)
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    threads = os.cpu_count() or 1

    if args.impl == "reference":
        if rank != 0:
            return
        cb = cpu_sample(args, threads, warmup=min(args.warmup, 1), steps=args.steps, budget_s=args.cpu_budget)
        v = cb["value"]
        print(json.dumps({
            "impl": "reference",
            "metric": "SIMPLE outer iters/s (mixed FP32/FP64 form; FP64 form and assembled elems/s beside it)",
            "value": v, "unit": "outer_iters/s", "higher_is_better": True, "n_gpus": world,
            "steps": cb["steps"], "warmup": cb["warmup"], "steps_requested": args.steps,
            "ms_per_step": cb["ms_per_step"], "dtype": "f64", "data": "synthetic", "scaling": "weak",
            "config": cavity_config(args, args.cpu_n, cb["elements"], cb["nodes"], cb["nnz"], world),
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "outer_iters/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }))
        return

    if world > 1:
        import torch

        torch.distributed.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    if args.workload in ("batch", "sst", "channel"):
        res = {"batch": run_batch, "sst": run_sst, "channel": run_channel}[args.workload](args, rank, world)
        if rank == 0:
            print(json.dumps(res))
        if world > 1:
            import torch

            torch.distributed.destroy_process_group()
        return
    if args.workload == "conduction":
        res = run_conduction(args, rank, world)
        if rank == 0 and not args.no_cpu:
            from oracle import pyoracle as po
            from openaccel_b200 import meshgen

            po.set_threads(threads)
            mc, gam, src, _ = meshgen.conduction(args.n, sigma=1.0, seed=4242)
            c = po.DiffCase(mc, gam, src, po.default_diff_settings(rtol=args.diff_rtol, maxit=20000))
            t0 = time.perf_counter()
            c.step()
            dt = time.perf_counter() - t0
            res["cpu_baseline"] = {"value": 1.0 / dt, "unit": "steps/s", "cores": threads, "kind": "port",
                                   "cpu": cpu_model(),
                                   "sample": f"1 step of the {args.n}^3 x 6 conduction case, FP64 oracle "
                                             "(Jacobi-BiCGStab), all host threads"}
        if rank == 0:
            print(json.dumps(res))
        if world > 1:
            import torch

            torch.distributed.destroy_process_group()
        return
    res = run_ours(args, rank, world)
    if rank == 0 and not args.no_cpu and not args.only_mixed:
        res["cpu_baseline"] = cpu_sample(args, threads, warmup=1, steps=2, budget_s=args.cpu_budget)
    if rank == 0:
        print(json.dumps(res))
    if world > 1:
        import torch

        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
