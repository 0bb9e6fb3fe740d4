#!/usr/bin/env python
"""Benchmark of the T-mixer step on B200 (one JSON line on stdout).

Workload (N=1): the single-mixer configuration of the benchmark set, a T-mixer
of width W=32 (inlet 256x32x32, mixing 64x128x32: 524,288 fluid nodes), flow
tau 0.6 (see WORKLOAD), species tau 0.6, k = 1e-3, inlet profile maximum 0.05,
outlet and initial density 1, by default in the plain FP64 form (bit-exact with
the reference); --form fp32 / fp16 selects a reduced-precision form, and the
line always carries all three forms' throughput under "forms".
A "step" is one full lattice-Boltzmann time step of the mixer (flow + 3
species, all nodes); MLUPS counts node updates of all four fields.

  value      MLUPS over all GPUs: N x nodes x K / (max over ranks of the device
             time of K steps), CUDA events on the solver's stream, inputs
             resident in HBM (the 319 MB population set exceeds the 126 MB L2,
             so no flush is needed between steps).
  e2e        the whole configured solve (create, init with the host inlet
             profile, 20,000 steps with the outlet mixing index read back every
             100 steps, all fields copied to host) through the public API.
  roofline   the bulk (interior) kernel: algorithmic bytes per node update
             (76 populations read and written: 1216 B FP64, 608 B FP32; the
             FP16 form 304 B + 64 B of moments) over its average launch time,
             against the measured HBM copy bandwidth.
  cpu_baseline  the reference's own OpenMP build (oracle/_ref) on this host's
             cores, on a bounded number of steps of the same workload.

Multi-GPU (torchrun): every rank solves its own mixer (replicas, no data-path
collective); the job's value is the sum.  ``--impl reference`` times the
reference's CPU build instead (rank 0 only).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MLUPS & %HBM roofline, served FP16-storage vs plain FP64; p50/p99 solve latency"
UNIT = "MLUPS"
# The single-mixer configuration (W=32, u_max 0.05, tau_c 0.6, k 1e-3, rho 1,
# 20000 steps) with the flow relaxation time of the reference case, 0.6: at
# the configuration's 0.56 the reference's own boundary closures diverge (the
# reference-exact oracle and the FP64 GPU form both turn non-finite after about
# 1000 steps, even at u_max 0.02), and a step costs the same at either value.
WORKLOAD = dict(W=32, u_max=0.05, tau_f=0.6, tau_c=0.6, k=1e-3, rho=1.0, steps=20000)
CONFIG_TAU_F = 0.56
BYTES_PER_LUP_FP64 = 4 * 19 * 8 * 2
# algorithmic bytes per lattice update of each form: populations read + written
# (76 values), plus for the FP16 form the writer's FP32 moments (2 x float4)
# written once and read once
FORM_BYTES = {"fp64": 1216, "fp32": 608, "fp16": 304 + 64}
# interior kernel shape of the single-mixer FP16 form: 32 x 4 tiles swept
# through 8 planes (65 us per W=32 step against 69 us for the flat kernel)
FP16_SHAPE = (2, 8)  # (TMX_SHAPE_SWEEP4, planes per tile)
FALLBACK_HBM_GBS = 6650.0


def measured_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return dict(hbm_gbs=float(d["hbm_gbs"]), source="measured")
    return dict(hbm_gbs=FALLBACK_HBM_GBS, source="fallback")


def workload_spec(form: str = "fp64"):
    import tmixer_b200 as T

    w = WORKLOAD
    return T.w_layout(w["W"], w["u_max"], w["tau_f"], w["tau_c"], w["k"], w["rho"], steps=w["steps"],
                      precision=T.PRECISIONS[form])


def workload_params() -> dict:
    """The workload's case constants without the CUDA library."""
    w = WORKLOAD
    return w_layout_params(w["W"], w["u_max"], w["tau_f"], w["tau_c"], w["k"], w["rho"])


def case_nodes(p: dict) -> int:
    return p["inx"] * p["iny"] * p["nz"] + p["mnx"] * p["mny"] * p["nz"]


def interior_nodes(s) -> int:
    """Interior (non-boundary) nodes of a case: the inlet box's inner nodes
    plus its row y = 1 over the opening (mnx - 2 columns), and the mixing
    box's inner columns over rows 2..mny (row mny joins the inlet box)."""
    inlet = (s.nz - 2) * ((s.inx - 2) * (s.iny - 2) + (s.mnx - 2))
    mixing = (s.mnx - 2) * (s.mny - 1) * (s.nz - 2)
    return inlet + mixing


def w_layout_umean(W: int, u_max: float) -> float:
    """The reference's Umean for a W-layout mixer whose duct profile peaks at
    u_max, computed without the CUDA library (the reference arm must not load
    it): the duct series of GenerateInletVelocity (Tmixer.cpp:1426-1539) for
    iny = nz = W in its own loop order, scaled to mean 1, shifted as the
    reference shifts it, and Umean = u_max / its maximum.  The terms with an
    even m or n are exact zeros ((1 - cos(m*pi)) rounds to 0), so the sums
    skip them without changing a bit; each (j, k) sum runs as a numpy vector
    operation whose elements round exactly as the scalar loop does.  libm's
    sin/cos (the ``math`` module) supply the same values as the host code's."""
    import math

    import numpy as np

    iny = nz = int(W)
    pi = 3.14159265358979323846
    d = (nz - 1.0) / 2.0
    w = (iny - 1.0) / 2.0
    AR = 1.0 * w / d
    den_m, den_n, AR2 = 2.0 * AR * d, 2.0 * d, AR * AR
    odd = range(1, 101, 2)
    one_m_cos = {m: 1.0 - math.cos(m * pi) for m in odd}
    sj = {m: np.array([math.sin(((m * pi) / den_m) * j) for j in range(iny)]) for m in odd}
    sk = {n: np.array([math.sin(((n * pi) / den_n) * k) for k in range(nz)]) for n in odd}
    nsum = np.zeros((iny, nz))
    for n in odd:
        msum = np.zeros((iny, nz))
        for m in odd:
            N = ((one_m_cos[m] * one_m_cos[n]) * sj[m])[:, None] * sk[n][None, :]
            D = float(m * n * ((m * m) + (AR2 * n * n)))
            msum = msum + N / D
        nsum = nsum + msum
    # the average in the host's order: rows j, then columns k, one at a time
    s = 0.0
    for v in nsum.ravel():
        s += float(v)
    average = s / (iny * nz)
    U1 = np.zeros((iny + 3, nz + 3))
    U1[1:iny + 1, 1:nz + 1] = nsum * (1.0 / average)
    U1[1:iny + 1, 0:nz] = U1[1:iny + 1, 1:nz + 1].copy()
    U1[1:iny + 1, 1] = 0.0
    return u_max / float(U1.max())


def w_layout_params(W: int, u_max: float, tau_f: float, tau_c: float, k: float, rho: float) -> dict:
    """The reference's case constants (oracle/build_ref.py's parameter names)
    of a W-layout mixer: inlet 8W x W x W, mixing 2W x 4W x W, species A at
    inlet 1 and B at inlet 2 with c = 1, rho0 = rho_out = rho, profile maximum
    u_max.  The same case as the library's tmx_case_wlayout, without loading
    the library."""
    return dict(inx=8 * W, iny=W, nz=W, mnx=2 * W, mny=4 * W, tau=float(tau_f), tau_c=float(tau_c),
                umean=w_layout_umean(W, u_max), rateconst=float(k), rho0=float(rho), rho_out=float(rho),
                ca_in1=1.0, ca_in2=0.0, cb_in1=0.0, cb_in2=1.0, cp_in1=0.0, cp_in2=0.0)


def workload_ref_params(spec) -> dict:
    return dict(inx=spec.inx, iny=spec.iny, nz=spec.nz, mnx=spec.mnx, mny=spec.mny, tau=spec.tau,
                tau_c=spec.tau_a, umean=spec.umean, rateconst=spec.rateconst, rho0=spec.rho0,
                rho_out=spec.rho_out, ca_in1=spec.c_in[0][0], ca_in2=spec.c_in[0][1], cb_in1=spec.c_in[1][0],
                cb_in2=spec.c_in[1][1], cp_in1=spec.c_in[2][0], cp_in2=spec.c_in[2][1])


def config_dict(p: dict, n_gpus: int) -> dict:
    """The workload as both arms report it (identical dicts: the form of the
    arithmetic is the line's "form" key, not part of the workload)."""
    return {"workload": "single T-mixer W=%d (inlet %dx%dx%d + mixing %dx%dx%d, %d fluid nodes)"
                        % (WORKLOAD["W"], p["inx"], p["iny"], p["nz"], p["mnx"], p["mny"], p["nz"], case_nodes(p)),
            "fluid_nodes": case_nodes(p), "bbox_nodes": p["inx"] * (p["iny"] + p["mny"]) * p["nz"],
            "tau_f": p["tau"], "tau_f_note": "configuration says %.2f; the reference's closures diverge there"
                                             % CONFIG_TAU_F,
            "tau_c": p["tau_c"], "k": p["rateconst"], "u_max": WORKLOAD["u_max"], "rho": p["rho0"],
            "solve_steps": WORKLOAD["steps"], "parallelism": "replicas x%d" % n_gpus,
            "l2": "state (2 x 319 MB FP64) larger than L2, no flush"}


# ---------------------------------------------------------------------------
# distributed plumbing (one process per GPU; replicas)
# ---------------------------------------------------------------------------
class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = False

    def init(self, backend: str) -> None:
        if self.world > 1:
            import datetime

            import torch.distributed as dist

            dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
            self.pg = True

    def barrier(self) -> None:
        if self.pg:
            import torch.distributed as dist

            dist.barrier()

    def max(self, x: float, device=None) -> float:
        if not self.pg:
            return x
        import torch
        import torch.distributed as dist

        t = torch.tensor([x], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def close(self) -> None:
        if self.pg:
            import torch.distributed as dist

            dist.destroy_process_group()
            self.pg = False


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self) -> None:
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.QUERY,
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict | None:
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as fh:
            for line in fh:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx.append(float(parts[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# the reference's CPU build (oracle/_ref), used as cpu_baseline and as the
# reference arm.  The oracle package is test infrastructure; only this
# baseline leg runs it.
# ---------------------------------------------------------------------------
# Timed steps of the reference's CPU build, the same count in the cpu_baseline
# leg and in the reference arm: its cost per step grows over the first
# hundreds of steps (the species fronts spread), so both time steps 2..257 of
# the solve, after one warm-up step.
REF_SAMPLE_STEPS = 256


def reference_cpu_run(params: dict, budget_s: float, steps: int = REF_SAMPLE_STEPS) -> dict:
    """Time ``steps`` steps (after one warm-up step) of the reference's own
    OpenMP build for the case ``params`` on all of this host's cores; fewer if
    a probe says they would take more than ``budget_s`` seconds."""
    from oracle import build_ref, oracle as O

    binary = build_ref.binary_path("bench_w%d" % WORKLOAD["W"], params)
    cores = os.cpu_count() or 1
    if not os.path.exists(binary):
        if os.path.exists(build_ref.REF_SRC):
            binary = build_ref.build("bench_w%d" % WORKLOAD["W"], params)
        else:
            return {"error": "reference binary for this workload not built"}
    # probe: 1 warm-up + 2 timed steps to size the sample
    _, _, t2 = O.run_ref(binary, 3, threads=cores, warmup=1)
    per = max(t2 / 2.0, 1e-4)
    n = int(max(3, min(steps, budget_s / per)))
    # the host's cores are shared with other work, so one sample can take
    # twice as long as the next: time it twice (when the budget allows) and
    # keep the faster
    runs = []
    for _ in range(2 if 2 * n * per <= budget_s else 1):
        _, _, secs = O.run_ref(binary, n + 1, threads=cores, warmup=1)
        runs.append(secs)
    secs = min(runs)
    value = case_nodes(params) * n / secs / 1e6
    return {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": "%d timed steps (steps 2..%d of the solve, after 1 warm-up step) of the same W=%d mixer, "
                      "reference OpenMP build (g++ -O2 -fopenmp), OMP_NUM_THREADS=%d; the faster of %d runs: "
                      "%s s" % (n, n + 1, WORKLOAD["W"], cores, len(runs), " / ".join("%.2f" % r for r in runs)),
            "seconds": secs, "steps": n}


def profile_traffic(form: str = "fp64") -> dict | None:
    """DRAM bytes per launch of the bulk kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "k_bulk_%s_w32.json" % form)
    if not os.path.exists(p):
        return None
    with open(p) as fh:
        return json.load(fh)


# ---------------------------------------------------------------------------
def pattern_ceiling(precision: int, nodes: int, achieved: float, device: int) -> dict | None:
    """The ceiling of the interior kernel's own access pattern
    (tmx_pattern_ceiling: the same bytes per lattice update in the same
    layout, no arithmetic) over the nodes of one launch, and the kernel's
    achieved bandwidth as a fraction of it; None where it cannot run."""
    import tmixer_b200 as T

    try:
        pc = T.pattern_ceiling(precision, max(int(nodes), 3 * 32768), reps=10, device=device)
    except T.TmxError:
        return None
    return {"gbs": pc["gbs"], "frac": achieved / pc["gbs"], "blocks_per_sm": pc["blocks_per_sm"],
            "nodes": pc["nodes"],
            "what": "the interior kernel's loads and stores (19 direction planes read at the upstream nodes and "
                    "written at the node, FP16 also the moment record) with no arithmetic: what DRAM gives "
                    "this 38-stream pattern, beside the plain copy's peak"}


def run_ours(args, dist: Dist) -> dict | None:
    import torch

    import tmixer_b200 as T

    torch.cuda.set_device(dist.local_rank)
    dist.init("nccl")
    dev = torch.device("cuda", dist.local_rank)
    spec = workload_spec(args.form)
    nodes = spec.nodes()
    peaks = measured_peaks()

    def measure(form: str, steps: int, warmup: int, clocks=None):
        """K steps of one form (events on the solver's stream, max over
        ranks), then per-launch kernel times for the roofline.  The FP16 form
        runs its interior as 32 x 4 tiles of 8 planes (FP16_SHAPE), whose
        kernel also updates the z wall faces."""
        sp = workload_spec(form)
        s = T.Solver(sp, device=dist.local_rank)
        if form == "fp16":
            s.set_shape(*FP16_SHAPE)
        s.init()
        s.step(warmup)
        s.sync()
        counts = s.counts()
        torch.cuda.synchronize()
        dist.barrier()
        if clocks:
            clocks.start()
        ms = s.time_steps(steps)
        torch.cuda.synchronize()
        dist.barrier()
        clk = clocks.stop() if clocks else None
        ms_max = dist.max(ms, dev)
        kr = min(steps, 400)
        tb, tbd, _ = s.step_timed(kr)
        s.close()
        bulk_ms, bnd_ms = tb / kr, tbd / kr
        bpl = FORM_BYTES[form]
        # nodes the interior kernel updates: the interior ones, and with the
        # sweep shape the z wall faces (one per interior column at each end)
        bulk_nodes = counts["interior"] + (2 * counts["interior"] // (sp.nz - 2) if form == "fp16" else 0)
        bulk_bytes = bulk_nodes * bpl
        achieved = bulk_bytes / (bulk_ms * 1e-3) / 1e9
        return dict(counts=counts, ms_max=ms_max, clk=clk, bulk_ms=bulk_ms, bnd_ms=bnd_ms, bulk_bytes=bulk_bytes,
                    bulk_nodes=bulk_nodes,
                    achieved=achieved, mlups=dist.world * nodes * steps / (ms_max * 1e-3) / 1e6,
                    step_gbs=nodes * bpl / (ms_max / steps * 1e-3) / 1e9)

    # --- value: K steps of the main form -----------------------------------
    main = measure(args.form, args.steps, args.warmup, ClockSampler(dist.local_rank))
    counts, ms_max, clk, value = main["counts"], main["ms_max"], main["clk"], main["mlups"]
    prof = profile_traffic(args.form)
    traffic = prof.get("dram_bytes_per_launch") if prof and prof.get("nodes") == nodes else None
    roofline = {"bound": "hbm", "achieved": main["achieved"], "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": main["achieved"] / peaks["hbm_gbs"], "traffic": traffic,
                "kernel": ("k_sweep4_f16 (interior nodes and z wall faces, %d per launch)" % main["bulk_nodes"]
                           if args.form == "fp16" else
                           "k_bulk_%s (interior nodes, %d per launch)" % (args.form, counts["interior"])),
                "peak_source": peaks["source"],
                "algorithmic_bytes_per_lup": FORM_BYTES[args.form],
                "algorithmic_bytes_per_launch": main["bulk_bytes"],
                "boundary_kernels_ms": main["bnd_ms"], "bulk_kernel_ms": main["bulk_ms"],
                "step_effective_gbs": main["step_gbs"]}
    roofline["pattern_ceiling"] = pattern_ceiling(T.PRECISIONS[args.form], main["bulk_nodes"], main["achieved"],
                                                  dist.local_rank)
    # --- the other forms, for comparison (same workload) --------------------
    forms = {}
    if not args.no_forms:
        for form in ("fp64", "fp32", "fp16"):
            m = main if form == args.form else measure(form, min(args.steps, 1000), args.warmup)
            forms[form] = {"mlups": m["mlups"], "ms_per_step": m["ms_max"] / (args.steps if form == args.form
                                                                               else min(args.steps, 1000)),
                           "bulk_gbs": m["achieved"], "bulk_frac": m["achieved"] / peaks["hbm_gbs"],
                           "bytes_per_lup": FORM_BYTES[form],
                           "interior_kernel": "sweep4:%d" % FP16_SHAPE[1] if form == "fp16" else "flat"}
            pc = pattern_ceiling(T.PRECISIONS[form], m["bulk_nodes"], m["achieved"], dist.local_rank)
            forms[form]["bulk_pattern_frac"] = pc["frac"] if pc else None

    # --- e2e: the configured solve through the public API ---------------
    e2e_steps = args.e2e_steps
    dist.barrier()
    t0 = time.perf_counter()
    s2 = T.Solver(spec, device=dist.local_rank)
    if args.form == "fp16":
        s2.set_shape(*FP16_SHAPE)
    s2.init()
    done = 0
    im_reads = 0
    while done < e2e_steps:
        c = min(100, e2e_steps - done)
        s2.step(c)
        done += c
        s2.mixing()  # outlet mixing index read back (D2H) every 100 steps
        im_reads += 1
    outs = [s2.field(b, f) for b in (0, 1) for f in T.FIELDS]
    s2.close()
    t1 = time.perf_counter()
    e2e_s = dist.max(t1 - t0, dev)
    h2d = 2 * (spec.iny + 3) * (spec.nz + 3) * 8 + counts["boundary"] * 5
    d2h = sum(o.nbytes for o in outs) + im_reads * (spec.mny + spec.iny) * 9 * 8
    e2e = {"value": dist.world * nodes * e2e_steps / e2e_s / 1e6, "unit": UNIT,
           "h2d_bytes_per_step": h2d / e2e_steps, "d2h_bytes_per_step": d2h / e2e_steps,
           "steps": e2e_steps, "seconds": e2e_s,
           "what": "create + init + %d steps + mixing index every 100 steps + all fields to host" % e2e_steps}

    # the reference's own case (401x51x51 + 101x750x51, 4.9M nodes), plain FP64
    refcase = None
    if not args.no_forms:
        rs = T.Solver(T.reference_case(), device=dist.local_rank).init()
        rs.step(args.warmup)
        rs.sync()
        n_ref = min(args.steps, 300)
        ms_ref = dist.max(rs.time_steps(n_ref), dev)
        nodes_ref = rs.spec.nodes()
        rs.close()
        refcase = {"workload": "the reference's own case (inlet 401x51x51 + mixing 101x750x51), plain FP64",
                   "fluid_nodes": nodes_ref, "steps": n_ref, "ms_per_step": ms_ref / n_ref,
                   "mlups": dist.world * nodes_ref * n_ref / (ms_ref * 1e-3) / 1e6,
                   "hbm_frac_step": nodes_ref * FORM_BYTES["fp64"] / (ms_ref / n_ref * 1e-3) / 1e9 / peaks["hbm_gbs"]}

    batched = served = None
    # the batched and served forms are one-GPU configurations (minutes of
    # work): measured at N=1 only, so that a scaling run holds its GPUs for
    # the replicas' timed steps and not for N copies of the served loop
    if not args.no_batched and dist.world == 1:
        fp64 = forms.get("fp64", {}).get("mlups") or (value if args.form == "fp64" else None)
        batched = run_batched(args, dist, fp64, peaks)
        if not args.no_served:
            served = run_served(args, dist, batched["mlups"], batched["launch_shape"])
            served["vs_plain_fp64"] = served["mlups"] / fp64 if fp64 else None

    cpu = None
    if dist.world == 1 and dist.rank == 0 and not args.no_cpu_baseline:
        cpu = reference_cpu_run(workload_params(), budget_s=args.cpu_budget)
    dist.close()
    if dist.rank != 0:
        return None
    form_text = {"fp64": "plain FP64 (bit-exact with the reference)", "fp32": "FP32 storage and arithmetic",
                 "fp16": "FP32 arithmetic, FP16 storage of the non-equilibrium populations + FP32 moments"}
    return {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": {"fp64": "f64", "fp32": "f32", "fp16": "f32/f16"}[args.form],
            "data": "synthetic",
            "form": form_text[args.form], "config": config_dict(workload_params(), dist.world),
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk,
            "gpu_launches": 3 * args.steps, "forms": forms, "reference_case": refcase, "batched": batched,
            "served": served}


# ---------------------------------------------------------------------------
# batched and served forms (FP16 storage, FP32 arithmetic)
# ---------------------------------------------------------------------------
# Mixer parameter distributions of the batched and served configurations,
# drawn from numpy's PCG64 seeded with BATCH_SEED.  The flow relaxation time is
# drawn from [0.6, 0.8] instead of the configurations' [0.52, 0.8]: below 0.6
# the reference's boundary closures diverge (see WORKLOAD).
BATCH_SEED = 20261203
BATCH_W = (16, 24, 32, 48)
SERVED_W = (16, 24, 32, 48, 64)
TAU_F_RANGE = (0.6, 0.8)
CONFIG_TAU_F_RANGE = (0.52, 0.8)
SERVED_BUDGET = 150 * 10**9


def draw_mixers(n: int, widths, seed: int, precision):
    import numpy as np

    import tmixer_b200 as T

    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        W = int(rng.choice(widths))
        u_max = float(rng.uniform(0.02, 0.08))
        tau_f = float(rng.uniform(*TAU_F_RANGE))
        tau_c = float(rng.uniform(0.52, 0.7))
        k = float(10 ** rng.uniform(-4, -2))
        out.append(T.w_layout(W, u_max, tau_f, tau_c, k, 1.0, precision=precision))
    return out


def run_batched(args, dist: Dist, fp64_mlups: float, peaks: dict) -> dict:
    """64 mixers of uneven size and parameters in one batch, autotuned launch
    shape, K steps each, timed on the device."""
    import tmixer_b200 as T

    specs = draw_mixers(args.batched_mixers, BATCH_W, BATCH_SEED, T.TMX_FP16)
    nodes = sum(s.nodes() for s in specs)
    budget = sum(T.Batch.footprint(s) for s in specs) + (64 << 20)
    with T.Batch(T.TMX_FP16, budget=budget, device=dist.local_rank) as B:
        for s in specs:
            B.add(s)
        if args.batched_shape:
            # a fixed interior kernel instead of the autotuner (profiling)
            kind, z = args.batched_shape.split(":")
            if kind == "flat":
                B.set_shape(256, int(z))
            else:
                B.set_sweep(T.SHAPE_KINDS[kind], int(z))
            tuned = dict(B.shape(), ms_per_step=None, steps_per_trial=0, fixed=args.batched_shape)
        else:
            tuned = B.tune(steps_per_trial=20)
        B.step(args.warmup, write_macro=False)
        B.sync()
        ms = B.time_steps(args.batched_steps)
        # each kernel alone (the interior kernel after the boundary kernels)
        kt = min(args.batched_steps, 50)
        t_int, t_bnd, _ = B.step_timed(kt)
        B.step(1, write_macro=True)
        im = B.outlet_im()
        B_shape = B.shape()
    # nodes the interior kernel updates: the interior ones, and with a sweep
    # shape the z wall faces (one at each end of every interior column)
    swept = B_shape["kernel"] != "flat"
    upd = sum(interior_nodes(s) * (s.nz / (s.nz - 2) if swept else 1) for s in specs)
    int_gbs = upd * FORM_BYTES["fp16"] / (t_int / kt * 1e-3) / 1e9
    int_pc = pattern_ceiling(T.TMX_FP16, upd, int_gbs, dist.local_rank)
    mlups = nodes * args.batched_steps / (ms * 1e-3) / 1e6
    bpl = FORM_BYTES["fp16"]
    gbs = mlups * 1e6 * bpl / 1e9
    return {"mixers": len(specs), "fluid_nodes": nodes, "steps": args.batched_steps, "ms": ms, "mlups": mlups,
            "vs_plain_fp64": mlups / fp64_mlups if fp64_mlups else None,
            "roofline": {"bound": "hbm", "achieved": gbs, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": gbs / peaks["hbm_gbs"], "algorithmic_bytes_per_lup": bpl,
                         "frac_populations_only": mlups * 1e6 * 304 / 1e9 / peaks["hbm_gbs"],
                         "interior_kernel": {
                             "what": "the interior kernel alone (%d timed steps, boundary kernels before it), "
                                     "%d nodes per launch x %d B" % (kt, int(upd), bpl),
                             "ms": t_int / kt, "achieved": upd * bpl / (t_int / kt * 1e-3) / 1e9,
                             "frac": upd * bpl / (t_int / kt * 1e-3) / 1e9 / peaks["hbm_gbs"],
                             "pattern_ceiling": int_pc},
                         "boundary_kernels_ms": t_bnd / kt},
            "tuned": tuned, "launch_shape": B_shape,
            "nonfinite_outlet_im": int(sum(1 for r in im for v in r if v != v)),
            "config": "%d mixers, W from %s, u_max U[0.02,0.08], tau_f U%s (configuration U%s), tau_c U[0.52,0.7], "
                      "k log-U[1e-4,1e-2], seed %d, FP16 storage / FP32 arithmetic, one launch per kernel "
                      "kind per step, CUDA-graph step" % (len(specs), list(BATCH_W), list(TAU_F_RANGE),
                                                           list(CONFIG_TAU_F_RANGE), BATCH_SEED)}


def run_served(args, dist: Dist, batched_mlups: float, shape: dict) -> dict:
    """Poisson arrivals of mixers from the served distribution, continuous
    batching until each converges (outlet index within 1e-6 over 500 steps)
    or reaches max_steps; p50/p99 time to solution and aggregate MLUPS."""
    import numpy as np
    import torch

    import tmixer_b200 as T

    specs = draw_mixers(args.served_requests, SERVED_W, BATCH_SEED + 1, T.TMX_FP16)
    mean_lups = float(np.mean([s.nodes() for s in specs])) * args.served_max_steps * 0.5
    mu = batched_mlups * 1e6 / mean_lups  # completions per second at full occupancy
    lam = 2.0 * mu  # arrivals outpace completions: the queue stays occupied
    rng = np.random.default_rng(BATCH_SEED + 2)
    arrivals = np.cumsum(rng.exponential(1.0 / lam, size=len(specs)))
    arrivals -= arrivals[0]
    reqs = [T.Request(s, float(a), max_steps=args.served_max_steps, window=500, tol=1e-6)
            for s, a in zip(specs, arrivals)]
    free = torch.cuda.mem_get_info(dist.local_rank)[0]
    budget = int(min(SERVED_BUDGET, free - (8 << 30)))
    with T.Batch(T.TMX_FP16, budget=budget, device=dist.local_rank) as B:
        B.set_from(shape)  # the batched form's tuned shape
        res, summ = T.serve(B, reqs, check_every=100)
    steps = [r["steps"] for r in res]
    bpl = FORM_BYTES["fp16"]
    gbs = summ["mlups"] * 1e6 * bpl / 1e9
    hbm = measured_peaks()["hbm_gbs"]
    return {"requests": len(reqs), "budget_bytes": budget, "arrival_rate_per_s": lam,
            "roofline": {"bound": "hbm", "achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm,
                         "algorithmic_bytes_per_lup": bpl,
                         "what": "aggregate served MLUPS x algorithmic bytes per lattice update over the makespan"},
            "p50_time_to_solution_s": summ["p50_s"], "p99_time_to_solution_s": summ["p99_s"],
            "mlups": summ["mlups"], "makespan_s": summ["makespan_s"], "max_active": summ["max_active"],
            "mean_active": summ["mean_active"], "converged": sum(r["status"] == "converged" for r in res),
            "steps_min_median_max": [min(steps), int(np.median(steps)), max(steps)],
            "config": "%d requests, W from %s, parameters as the batched form (seed %d), Poisson arrivals at twice "
                      "the full-occupancy completion rate, retire when the outlet index moves < 1e-6 over 500 steps "
                      "or at %d steps, FP16 storage, budget %.0f GB"
                      % (len(reqs), list(SERVED_W), BATCH_SEED + 1, args.served_max_steps, budget / 1e9)}


def reference_cpu_samples(params: dict, samples: int, warm: int, budget_s: float) -> dict:
    """The reference arm's timing: ``warm`` untimed and then ``samples``
    timed samples of the reference's own OpenMP build on all of this host's
    cores, one sample being m consecutive steps of the solve, m sized so that
    the whole run fits ``budget_s`` (one process: steps 1 .. warm*m untimed,
    the next samples*m timed)."""
    from oracle import build_ref, oracle as O

    binary = build_ref.binary_path("bench_w%d" % WORKLOAD["W"], params)
    cores = os.cpu_count() or 1
    if not os.path.exists(binary):
        if os.path.exists(build_ref.REF_SRC):
            binary = build_ref.build("bench_w%d" % WORKLOAD["W"], params)
        else:
            return {"error": "reference binary for this workload not built"}
    _, _, t2 = O.run_ref(binary, 3, threads=cores, warmup=1)  # probe: 2 timed steps
    per = max(t2 / 2.0, 1e-4)
    m = int(max(1, min(REF_SAMPLE_STEPS, budget_s / ((samples + warm) * per))))
    _, _, secs = O.run_ref(binary, (warm + samples) * m, threads=cores, warmup=warm * m)
    value = case_nodes(params) * samples * m / secs / 1e6
    return {"value": value, "unit": UNIT, "cores": cores, "kind": "reference", "seconds": secs,
            "steps_per_sample": m,
            "sample": "%d timed samples of %d steps each (steps %d..%d of the solve, after %d untimed samples) of "
                      "the same W=%d mixer, reference OpenMP build (g++ -O2 -fopenmp), OMP_NUM_THREADS=%d: %.2f s"
                      % (samples, m, warm * m + 1, (warm + samples) * m, warm, WORKLOAD["W"], cores, secs)}


def run_reference(args, dist: Dist) -> dict | None:
    """The reference arm: the reference's own OpenMP build (oracle/_ref,
    compiled from its source) on this host's cores, for the same case and
    config as our arm; each of its --warmup and --steps steps is a sample of
    m reference steps.  Nothing here loads the CUDA library: the case
    constants come from w_layout_params."""
    if dist.rank != 0:
        return None
    params = workload_params()
    r = reference_cpu_samples(params, args.steps, args.warmup, budget_s=args.ref_budget)
    if "error" in r:
        return {"impl": "reference", "unavailable": r["error"]}
    return {"impl": "reference", "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": dist.world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["seconds"] / args.steps * 1e3,
            "steps_per_sample": r["steps_per_sample"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "form": "the reference's OpenMP CPU build (FP64)", "config": config_dict(params, dist.world),
            "cpu_baseline": {"value": r["value"], "unit": UNIT, "cores": r["cores"], "kind": "reference",
                             "sample": r["sample"]},
            "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--e2e-steps", type=int, default=WORKLOAD["steps"])
    ap.add_argument("--cpu-budget", type=float, default=60.0,
                    help="at most this many seconds of reference CPU steps in the cpu_baseline leg")
    ap.add_argument("--ref-budget", type=float, default=90.0,
                    help="at most this many seconds of reference CPU steps in the reference arm")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--form", choices=["fp64", "fp32", "fp16"], default="fp64",
                    help="form of the main line (fp64: the plain form, bit-exact with the reference)")
    ap.add_argument("--no-forms", action="store_true", help="skip the comparison of the three forms")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched and served forms")
    ap.add_argument("--no-served", action="store_true", help="skip the served form")
    ap.add_argument("--batched-mixers", type=int, default=64)
    ap.add_argument("--batched-steps", type=int, default=5000)
    ap.add_argument("--served-requests", type=int, default=64)
    ap.add_argument("--batched-shape", default=None,
                    help="fix the batched interior kernel instead of autotuning: flat:CELLS or sweep4:PLANES / "
                         "sweep8:PLANES")
    ap.add_argument("--served-max-steps", type=int, default=50000)

    args = ap.parse_args(argv)
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    dist = Dist()
    if dist.world != args.gpus and "WORLD_SIZE" in os.environ:
        print("warning: --gpus %d but WORLD_SIZE %d" % (args.gpus, dist.world), file=sys.stderr)
    out = run_reference(args, dist) if args.impl == "reference" else run_ours(args, dist)
    if out is not None:
        print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
