#!/usr/bin/env python
"""Headline benchmark: FP64 VL2 + PLM + HLLD + CT on the uneven 2D blast batch.

Workload (the uneven parameter sweep the headline metric is quoted on): 64
independent 2D MHD blast-wave runs, side lengths drawn from the seed in
{64, 96, 128, 192, 256, 384, 512}, outflow boundaries, per-instance CFL dt,
gamma = 5/3, VL2 + PLM (van Leer limiter, the reference default) + HLLD + CT.
Synthetic seeded initial conditions (no dataset exists).  One "step" advances
every instance by one VL2 step; a zone-update is one active cell advanced one
step.  The batch state (~0.5 GB) is larger than L2, so no flush is needed.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  Under torchrun each rank runs its own batch
(weak scaling: the instances are independent, there is no data-path
collective); the timed region is bracketed by barriers and the max over ranks
is reported.
"""
import argparse
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mzone-updates/s, 1 B200: batched FP64 VL2+HLLD+CT vs plain; adjoint/fwd ratio"
UNIT = "Mzone-updates/s"
BYTES_PER_ZONE = 192  # 9 conserved + 3 face-B doubles read once and written once
# Corrector launch (the dominant kernel): reads w^n (9 doubles, u^n is rebuilt
# from it), b^n (3), w^(n+1/2) (9) and b^(n+1/2) (3); writes w^(n+1) (9) and
# b^(n+1) (3): 36 doubles per active zone.  The predictor reads 12 and writes
# 12 per zone it covers (active zones plus two ghost rings).
CORR_BYTES_PER_ZONE = 288
# DRAM bytes per active zone of one corrector launch (dram__bytes_read.sum +
# dram__bytes_write.sum), from an ncu capture of the persistent corrector on
# the first 16 instances of this batch (scaled per zone).
CORR_TRAFFIC_PER_ZONE = 269.9
# FP64 flops per zone-update of the persistent kernels (2 x DFMA + DADD + DMUL
# thread instructions, those of the division and square-root sequences
# included), from the same capture: predictor 1196 + corrector 1343.
FLOPS_PER_ZONE = 2539


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--path", default="batch", choices=["batch", "plain", "fused"])
    ap.add_argument("--no-plain", action="store_true", help="skip the plain per-instance comparison")
    ap.add_argument("--instances", type=int, default=64)
    ap.add_argument("--variant", type=int, default=None, help="fixed kernel variant instead of the autotuner's choice")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint/forward measurement")
    ap.add_argument("--adjoint-only", action="store_true", help="print only the adjoint/forward measurement")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the 3D configurations (256^3 turbulence, 384^3 conduction; about a minute of set-up)")
    ap.add_argument("--configs-only", action="store_true",
                    help="print only the 3D configurations (no 2D batch, adjoint or CPU baseline)")
    ap.add_argument("--n3d", type=int, default=0,
                    help="side of the 3D configurations' grids instead of 256 / 384 (batch: half of it); small "
                         "cases for profiling")
    ap.add_argument("--config-names", default="turbulence,conduction,batch",
                    help="which 3D configurations to run (profiling one of them)")
    ap.add_argument("--config-paths", default="fused,split,plain",
                    help="which kernel paths the single-grid 3D configurations run on")
    return ap.parse_args()


def build_batch(n, seed, rank=0):
    """The rank's share of the sweep (bonzo_b200.parallel: seed + rank)."""
    from bonzo_b200 import problems as P
    from bonzo_b200.parallel import sweep_shard
    out = []
    for q in sweep_shard(n, seed, rank):
        gc = P.make_grid(q["N"], q["N"], 1, dims=2, bc=1)
        prim, bfld = P.blast(gc, b_mag=q["b_mag"], b_angle=q["b_angle"], center=q["center"],
                             p_ratio=q["p_ratio"])
        out.append((q, gc, prim, bfld))
    return out


METHOD = dict(dims=2, bc=((1, 1), (1, 1), (1, 1)), gam=5. / 3, cour=0.4, rsolver="hlld",
              reconstr="linear", limiter="vl")


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    """Samples SM clock and clock-event reasons every 50 ms (NVML)."""

    REASONS = {
        "hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
        "sw_power_cap": 0x4, "hw_power_brake_slowdown": 0x80,
    }

    def __init__(self, device_index):
        self.samples = []
        self.reasons = set()
        self.max_mhz = None
        self._stop = threading.Event()
        self._t = None
        try:
            import pynvml
            pynvml.nvmlInit()
            import torch
            uuid = str(torch.cuda.get_device_properties(device_index).uuid)
            try:
                self.h = pynvml.nvmlDeviceGetHandleByUUID("GPU-" + uuid)
            except Exception:
                self.h = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.nv = pynvml
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nv = None

    def _run(self):
        nv = self.nv
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for name, bit in self.REASONS.items():
                    if r & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            self._stop.wait(0.05)

    def __enter__(self):
        if self.nv is not None:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join()

    def record(self):
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None,
                "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                "samples": len(self.samples)}


# ---------------------------------------------------------------------------
# CPU reference (the reference's compiled kernels through the oracle driver)
# ---------------------------------------------------------------------------

def cpu_sample(batch, min_zones=1_200_000):
    """Instances (in seeded order) until the sample holds >= min_zones cells."""
    sample, z = [], 0
    for item in batch:
        sample.append(item)
        z += item[0]["N"] ** 2
        if z >= min_zones:
            break
    return sample, z


def run_cpu_reference(batch, steps, warmup, rows_parallel=1):
    """One VL2 step of a bounded sample of the batch on the host cores.
    rows_parallel=1: OpenMP over the rows of every sweep (the stronger, labelled
    variant); rows_parallel=0: the reference's own structure, prange over k for
    the x / y sweeps (godunov.pyx:20-209), one active thread in 2D."""
    from oracle import oracle as O
    use_ref = O.ref_lib() is not None
    sample, zones = cpu_sample(batch)
    sims = []
    for q, gc, prim, bfld in sample:
        s = O.OracleSim(Nx=q["N"], Ny=q["N"], Nz=1, use_ref_kernels=use_ref, nthreads=0,
                        rows_parallel=rows_parallel, **METHOD)
        s.set_state(prim, bfld)
        s.init()
        sims.append(s)
    times = []
    for it in range(warmup + steps):
        t0 = time.perf_counter()
        for s in sims:
            s.advance(1e30, max_steps=1)
        dt = time.perf_counter() - t0
        if it >= warmup:
            times.append(dt)
    per_step = statistics.median(times)
    value = zones / per_step / 1e6
    desc = ("one VL2 step on the first %d instances of the batch (%d zones, N=%s); %s; %s" %
            (len(sample), zones, ",".join(str(x[0]["N"]) for x in sample),
             "reference C kernels (src/mhd/fluxes_c.c, src/coordinates/reconstr_c.c, "
             "src/mhd/eos_c.c) driven by the oracle's C restatement of the Cython sweeps"
             if use_ref else "oracle C restatement",
             "OpenMP rows-parallel over all host threads" if rows_parallel else
             "the reference's OpenMP structure (prange over k: one active thread in 2D)"))
    return dict(value=round(value, 3), unit=UNIT, cores=os.cpu_count() if rows_parallel else 1,
                kind="reference" if use_ref else "port", sample=desc,
                per_step_s=round(per_step, 4))


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def _timed(stream, step_fn, steps, dist, multi=None):
    """ms of `steps` steps (max over ranks), CUDA events on the launching
    stream.  multi(k), when given, runs k steps in one call (a batch replays
    its captured two-step CUDA graph)."""
    import torch
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev0.record(stream)
    if multi is not None:
        multi(steps)
    else:
        for _ in range(steps):
            step_fn()
    ev1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = ev0.elapsed_time(ev1)
    from bonzo_b200.parallel import max_over_ranks
    return max_over_ranks(ms, dist, device="cuda")


def make_engine(kind, batch, stream):
    """kind 'batch': one bnz_batch for all instances (one launch per stage);
    'plain' / 'fused': one context per instance, one graph launch per instance."""
    from bonzo_b200._lib import Batch, Context
    if kind == "batch":
        grids = [dict(Nx=q["N"], Ny=q["N"], Nz=1, dims=2, bc=METHOD["bc"]) for q, _, _, _ in batch]
        meth = {k: v for k, v in METHOD.items() if k not in ("dims", "bc")}
        eng = Batch(grids, **meth)
        eng.set_stream(stream.cuda_stream)
        ctxs = eng.instances
        step = lambda: eng.advance(1e30, 1)
        multi = lambda k: eng.advance(1e30, k)
        count = eng.launch_count
    else:
        ctxs = []
        for q, gc, prim, bfld in batch:
            c = Context(Nx=q["N"], Ny=q["N"], Nz=1, path=kind, **METHOD)
            c.set_stream(stream.cuda_stream)
            ctxs.append(c)
        eng = ctxs

        def step():
            for c in ctxs:
                c.advance_graph(1e30, 1)

        multi = None
        count = lambda: sum(c.launch_count() for c in ctxs)
    for c, (q, gc, prim, bfld) in zip(ctxs, batch):
        c.set_state(prim, bfld)
        c.init()
    return eng, ctxs, step, multi, count


def run_ours(args, rank, world, dist):
    import torch
    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    batch = build_batch(args.instances, args.seed, rank)
    zones = sum(q["N"] ** 2 for q, _, _, _ in batch)
    from bonzo_b200.parallel import sum_over_ranks
    zones_all = sum_over_ranks(zones, dist, device="cuda")  # every rank's sweep members
    stream = torch.cuda.Stream()

    # the plain one-instance-per-launch path (the comparison the headline quotes)
    plain_ms = None
    if args.path == "batch" and not args.no_plain:
        eng, ctxs, step, multi, count = make_engine("plain", batch, stream)
        for _ in range(args.warmup):
            step()
        plain_steps = max(3, args.steps // 4)
        plain_ms = _timed(stream, step, plain_steps, dist) / plain_steps
        for c in ctxs:
            c.check()
        del eng, ctxs, step, multi, count
        torch.cuda.synchronize()
        torch.cuda.empty_cache()

    eng, ctxs, step, multi, count = make_engine(args.path, batch, stream)
    tune = None
    if args.path == "batch":
        from bonzo_b200._lib import variant_label, variants
        vs = variants()
        if args.variant is not None:
            # a fixed variant (profiling runs: the autotuner's choice under a profiler is not the real one)
            eng.set_variant(args.variant)
            best, ms = args.variant, {}
        else:
            # autotuner: tile shape / staging on this workload (state restored after each trial)
            from bonzo_b200 import autotune
            best, ms = autotune.tune_batch(eng, [q["N"] for q, _, _, _ in batch], METHOD["rsolver"],
                                           METHOD["limiter"], steps=2, use_cache=False)
        tune = {"chosen": {"tile": "%dx%d" % vs[best][:2], "staged_predictor": bool(vs[best][2]),
                           "persistent": ["none", "corrector", "predictor and corrector"][vs[best][3]]},
                "ms_per_step": {variant_label(vs[v]): round(t, 4)
                                for v, t in ms.items()}}
    for _ in range(args.warmup):
        step()
    if multi is not None:
        multi(2)  # untimed: captures the two-step graph at the current state parity
    torch.cuda.synchronize()
    launches0 = count()
    with ClockSampler(dev) as clk:
        ms_max = _timed(stream, step, args.steps, dist, multi)
    launches = count() - launches0
    ms_step = ms_max / args.steps
    value = zones_all * args.steps / (ms_max * 1e-3) / 1e6

    # e2e: host state in pinned memory, copied in and out every step through the C ABI;
    # one pinned allocation holds every instance's prim then bfld, back to back
    host = []
    ncs = [int(np.prod(c.shape)) for c in ctxs]
    pool = torch.empty(12 * sum(ncs), dtype=torch.float64, pin_memory=True).numpy()
    off = 0
    for c, nc in zip(ctxs, ncs):
        P = pool[off:off + 9 * nc].reshape((9,) + c.shape)
        B = pool[off + 9 * nc:off + 12 * nc].reshape((3,) + c.shape)
        off += 12 * nc
        c.get_state_into(P, None, B)
        host.append((P, B))
    h2d = sum(P.nbytes + B.nbytes for P, B in host)
    ke = max(1, args.e2e_steps)

    if args.path == "batch":
        prims, bflds = [P for P, _ in host], [B for _, B in host]
        e2e_how = ("bnz_batch_step_host: every instance's state (one pinned host allocation, instances "
                   "back to back) copied in, one batch step, ghosts filled, copied back out; one copy each "
                   "way per group of instances through a device staging buffer, copies in, steps and "
                   "copies out of 32 groups overlapping on three streams")

        def e2e_step():
            eng.step_host(prims, bflds, 1e30, 1)
        e2e_step()  # untimed: creates the copy streams and events
    else:
        e2e_how = "bnz_set_state of every instance, one step each, bnz_get_state of every instance, pinned host buffers"

        def e2e_step():
            for c, (P, B) in zip(ctxs, host):
                c.set_state(P, B)
            step()
            for c, (P, B) in zip(ctxs, host):
                c.get_state_into(P, None, B)

    ems = _timed(stream, e2e_step, ke, dist)
    e2e = zones_all * ke / (ems * 1e-3) / 1e6
    for c in ctxs:
        c.check()

    from bonzo_b200.peaks import hbm_peak
    peak, peak_src = hbm_peak()
    # the step is FP64-issue bound: its FP64 rate against the measured FMA peak
    from bonzo_b200._lib import fp64_fma_peak
    fp64_peak = fp64_fma_peak()
    fp64_achieved = FLOPS_PER_ZONE * zones / (ms_step * 1e-3) / 1e12
    fp64 = {"achieved_tflops": round(fp64_achieved, 3), "peak_tflops": round(fp64_peak, 3),
            "frac": round(fp64_achieved / fp64_peak, 4) if fp64_peak > 0 else None,
            "flops_per_zone": FLOPS_PER_ZONE,
            "peak_source": "measured in this run (bnz_fp64_fma_peak: independent FMA chains on every SM)",
            "flops_source": "ncu FP64 instruction counts of the persistent kernels on the first 16 instances"}
    step_achieved = BYTES_PER_ZONE * zones / (ms_step * 1e-3) / 1e9
    step_roof = {"achieved": round(step_achieved, 1), "frac": round(step_achieved / peak, 4),
                 "bytes_per_zone": BYTES_PER_ZONE,
                 "what": "whole step (%s path, %d launches per step over %d instances)" %
                         (args.path, launches // max(1, args.steps), len(ctxs))}
    if args.path == "batch":
        # the dominant kernel, timed live: the same batch steps launched one by
        # one with CUDA events on the batch stream around every launch
        if dist:
            dist.barrier()
        kms = eng.advance_timed(1e30, args.steps)
        for c in ctxs:
            c.check()
        # achieved in the zone-update unit: 192 B per active zone per launch
        achieved = BYTES_PER_ZONE * zones / (kms["corrector"] * 1e-3) / 1e9
        own = CORR_BYTES_PER_ZONE * zones / (kms["corrector"] * 1e-3) / 1e9
        traffic = None if CORR_TRAFFIC_PER_ZONE is None else int(CORR_TRAFFIC_PER_ZONE * zones)
        roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                    "frac": round(achieved / peak, 4), "traffic": traffic, "peak_source": peak_src,
                    "kernel": ("k_corr2d_pq (persistent corrector, one launch covers every instance)"
                               if tune and vs[best][3] else
                               "k_corr2d (corrector, one launch covers every instance)"),
                    "bytes_per_zone": BYTES_PER_ZONE,
                    "algorithmic_bytes_per_launch": BYTES_PER_ZONE * zones,
                    "corrector_own_bytes": {"bytes_per_zone": CORR_BYTES_PER_ZONE,
                                            "achieved": round(own, 1), "frac": round(own / peak, 4),
                                            "what": "w^n, b^n, w^(n+1/2), b^(n+1/2) read, w^(n+1), "
                                                    "b^(n+1) written: the launch's own inputs and outputs"},
                    "ms_per_launch": round(kms["corrector"], 4),
                    "kernel_ms_per_launch": {k: round(v, 4) for k, v in kms.items()},
                    "step": step_roof}
    else:
        roofline = {"bound": "hbm", "achieved": step_roof["achieved"], "peak": peak, "unit": "GB/s",
                    "frac": step_roof["frac"], "traffic": None, "peak_source": peak_src,
                    "kernel": step_roof["what"], "bytes_per_zone": BYTES_PER_ZONE}
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded blast-wave initial conditions)",
        "config": {"workload": "uneven 2D MHD blast batch: %d instances, N^2 with N in "
                               "{64,96,128,192,256,384,512} (seed %d), outflow BCs, VL2+PLM(vl)+HLLD+CT, "
                               "per-instance CFL dt" % (len(ctxs), args.seed),
                   "instances": len(ctxs), "zones_per_step_per_gpu": zones, "path": args.path,
                   "l2": "inputs larger than L2 (%.0f MB of state)" % (
                       sum(12 * 8 * np.prod(c.shape) for c in ctxs) / 1e6),
                   "parallelism": "instances sharded per GPU (dp%d, no collective)" % world,
                   "autotune": tune},
        "e2e": {"value": round(e2e, 3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(h2d),
                "how": e2e_how},
        "gpu_launches": int(launches),
        "roofline": roofline,
        "fp64": fp64,
        "clocks": clk.record(),
    }
    if plain_ms is not None:
        pv = zones_all / (plain_ms * 1e-3) / 1e6
        line["plain_one_instance_per_launch"] = {"value": round(pv, 3), "unit": UNIT,
                                                 "ms_per_step": round(plain_ms, 4)}
        line["batched_vs_plain"] = round(value / pv, 3)
    return line


def run_adjoint(warmup=1, reps=5):
    """adjoint/forward cost of a differentiable rollout: 256^2 periodic vortex
    with a seeded smooth perturbation (Fourier modes |k| <= 4, amplitude 1e-2 on
    v and Az), VL2 + PLM(mc) + HLLD + CT, 100 steps of fixed dt = 1e-4, loss =
    squared misfit of the final density, checkpoint every 10 steps.  Forward =
    the autograd Function's forward (state in, 100 recorded steps, state out);
    adjoint = its backward (segment recompute + reverse steps)."""
    import torch
    from bonzo_b200 import problems as P
    from bonzo_b200._lib import Context
    from bonzo_b200.adjoint import rollout
    n, nsteps, dt, every = 256, 100, 1e-4, 10
    gc = P.make_grid(n, n, 1, dims=2, bc=0)
    prim, bfld = P.otvortex(gc, pert_amp=1e-2, seed=0)
    eng = Context(Nx=n, Ny=n, Nz=1, dims=2, bc=((0, 0), (0, 0), (0, 0)), gam=5. / 3, cour=0.4,
                  rsolver="hlld", limiter="mc", path="fused")
    eng.set_state(prim, bfld)
    eng.init()
    P0, _, B0 = eng.get_state()
    p0 = torch.from_numpy(P0).cuda()
    b0 = torch.from_numpy(B0).cuda()
    target = p0[0].clone() * 1.01
    stream = torch.cuda.current_stream()
    fwd, adj = [], []
    for it in range(warmup + reps):
        p = p0.clone().requires_grad_(True)
        b = b0.clone().requires_grad_(True)
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        torch.cuda.synchronize()
        e0.record(stream)
        xp, xb = rollout(p, b, eng, nsteps, dt, checkpoint_every=every)
        e1.record(stream)
        loss = ((xp[0] - target) ** 2).sum()
        g = torch.autograd.grad(loss, (p, b), retain_graph=False)
        e2.record(stream)
        torch.cuda.synchronize()
        if it >= warmup:
            fwd.append(e0.elapsed_time(e1))
            adj.append(e1.elapsed_time(e2))
        del g
    f, a = statistics.median(fwd), statistics.median(adj)
    return {"workload": "256^2 periodic vortex + smooth perturbation, VL2+PLM(mc)+HLLD+CT, 100 steps of "
                        "dt=1e-4, checkpoint every 10 steps, loss = density misfit",
            "fwd_ms": round(f, 3), "adj_ms": round(a, 3), "ratio": round(a / f, 3),
            "fwd_mzone_updates_per_s": round(n * n * nsteps / (f * 1e-3) / 1e6, 1),
            "how": "CUDA events on the current stream around the autograd Function's forward and around "
                   "backward (incl. the loss); median of %d after %d warm-up" % (reps, warmup)}


def _time_ctx(c, steps, graph, stream, clk=None):
    """ms per step of `steps` steps of a context (CUDA events on its stream);
    graph: replayed from the captured two-step graph, else bnz_advance (host
    loop; needed with conduction, whose stage count is chosen on the host)."""
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    nsts = 0
    e0.record(stream)
    if graph:
        c.advance_graph(1e30, steps)
    else:
        for _ in range(steps):
            c.advance(1e30, 1)
            nsts += c.last_nsts()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps, nsts / steps


def run_configs(fused_steps=6, plain_steps=2, n3d=0, names=("turbulence", "conduction", "batch"),
                paths=("fused", "split", "plain")):
    """The 3D configurations on seeded synthetic initial states, on the fused
    z-marching path, the split path (fluxes once per face, fused update) and
    the plain one-launch-per-loop path:
    256^3 decaying turbulence (rms Mach 1, beta 1, VL2+PLM(vl)+HLLD+CT, CFL 0.3)
    and 384^3 field-aligned conduction (kappa_par 0.01, RKL2 super-time-stepping
    interleaved with VL2+HLLD+CT).  Each path: two warm-up steps, then timed
    steps with CUDA events on the context's stream and the SM clock sampled.
    Throughput counts hyperbolic zone-updates; the HBM figure counts 192 B per
    zone-update plus 96 B per RKL2 zone-stage."""
    import torch
    from bonzo_b200 import problems as P
    from bonzo_b200._lib import Context
    from bonzo_b200.peaks import hbm_peak
    peak, peak_src = hbm_peak()
    out = {}
    stream = torch.cuda.Stream()
    dev = torch.cuda.current_device()
    nt, nc = (n3d, n3d) if n3d else (256, 384)
    for name, n, kw, gen, graph in (
            ("turbulence_%d^3" % nt, nt, dict(cour=0.3), lambda gc: P.turbulence3d(gc, seed=0), True),
            ("conduction_%d^3" % nc, nc, dict(cour=0.4, kappa0=0.01, thcond_type="aniso"),
             lambda gc: P.conduction3d(gc, seed=0), False)):
        if name.split("_")[0] not in names:
            continue
        gc = P.make_grid(n, n, n, dims=3, bc=0)
        prim, bfld = gen(gc)
        rec = {}
        for path, steps in (("fused", fused_steps), ("split", fused_steps), ("plain", plain_steps)):
            if path not in paths:
                continue
            c = Context(Nx=n, Ny=n, Nz=n, dims=3, bc=((0, 0), (0, 0), (0, 0)), gam=5. / 3, rsolver="hlld",
                        limiter="vl", path=path, **kw)
            c.set_stream(stream.cuda_stream)
            c.set_state(prim, bfld)
            c.init()
            _time_ctx(c, 2, graph, stream)
            with ClockSampler(dev) as clk:
                ms, nsts = _time_ctx(c, steps, graph, stream)
            c.check()
            zones = n ** 3
            byts = BYTES_PER_ZONE * zones + 96 * zones * nsts
            achieved = byts / (ms * 1e-3) / 1e9
            rec[path] = {"ms_per_step": round(ms, 3), "mzone_updates_per_s": round(zones / (ms * 1e-3) / 1e6, 1),
                         "rkl2_stages_per_step": round(nsts, 2), "steps_timed": steps,
                         "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                                      "frac": round(achieved / peak, 4), "peak_source": peak_src,
                                      "bytes": "192 B per zone-update + 96 B per RKL2 zone-stage, whole step"},
                         "clocks": clk.record()}
            c.close()
            torch.cuda.empty_cache()
        for p in ("fused", "split"):
            if p in rec and "plain" in rec:
                rec[p + "_vs_plain"] = round(rec["plain"]["ms_per_step"] / rec[p]["ms_per_step"], 3)
        rec["workload"] = ("%d^3 periodic, seeded synthetic %s, VL2+PLM(vl)+HLLD+CT%s" %
                           (n, name.split("_")[0], ", RKL2 conduction kappa_par 0.01" if kw.get("kappa0") else ""))
        out[name] = rec
        del prim, bfld
    nb = n3d // 2 if n3d else 192
    if "batch" in names:
        out["conduction_batch_4x%d^3" % nb] = run_batch3d(stream, dev, peak, peak_src, fused_steps, n=nb)
    return out


def run_batch3d(stream, dev, peak, peak_src, steps, n=192, count=4):
    """The conduction configuration's batch: 4 instances of 192^3 (seeds 0..3)
    advanced together -- one launch per hyperbolic stage for all instances, then
    each instance's RKL2 stages over its own dt -- beside the same instances as
    separate fused contexts and as separate split-path contexts stepped one
    after another; and the same batch on the split path (each instance's
    launches in turn)."""
    import torch
    from bonzo_b200 import problems as P
    from bonzo_b200._lib import Batch, Context
    ics = []
    for q in range(count):
        gc = P.make_grid(n, n, n, dims=3, bc=0)
        ics.append(P.conduction3d(gc, seed=q))
    meth = dict(gam=5. / 3, cour=0.4, rsolver="hlld", limiter="vl", kappa0=0.01, thcond_type="aniso")
    grid = dict(Nx=n, Ny=n, Nz=n, dims=3, bc=((0, 0), (0, 0), (0, 0)))
    rec = {"workload": "%d instances of %d^3 periodic field-aligned conduction (seeds 0..%d), VL2+PLM(vl)+HLLD+CT "
                       "with RKL2, per-instance CFL dt" % (count, n, count - 1)}
    zones = count * n ** 3
    for path, key in (("fused", "batch"), ("split", "split_batch")):
        b = Batch([grid] * count, path=path, **meth)
        b.set_stream(stream.cuda_stream)
        for q, (prim, bfld) in enumerate(ics):
            b[q].set_state(prim, bfld)
            b[q].init()
        b.advance(1e30, 2)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        with ClockSampler(dev) as clk:
            e0.record(stream)
            b.advance(1e30, steps)
            e1.record(stream)
            torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        nsts = sum(b[q].last_nsts() for q in range(count))
        for q in range(count):
            b[q].check()
        byts = BYTES_PER_ZONE * zones + 96 * n ** 3 * nsts
        ach = byts / (ms * 1e-3) / 1e9
        rec[key] = {"ms_per_step": round(ms, 3), "mzone_updates_per_s": round(zones / (ms * 1e-3) / 1e6, 1),
                    "rkl2_stages_per_step_all_instances": nsts, "steps_timed": steps,
                    "roofline": {"bound": "hbm", "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                                 "frac": round(ach / peak, 4), "peak_source": peak_src},
                    "clocks": clk.record()}
        b.close()
        del b
        torch.cuda.empty_cache()
    ms = rec["batch"]["ms_per_step"]
    for path, key in (("fused", "separate_contexts"), ("split", "separate_split_contexts")):
        ctxs = []
        for prim, bfld in ics:
            c = Context(path=path, **grid, **meth)
            c.set_stream(stream.cuda_stream)
            c.set_state(prim, bfld)
            c.init()
            c.advance(1e30, 2)
            ctxs.append(c)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(steps):
            for c in ctxs:
                c.advance(1e30, 1)
        e1.record(stream)
        torch.cuda.synchronize()
        ms_sep = e0.elapsed_time(e1) / steps
        rec[key] = {"ms_per_step": round(ms_sep, 3), "mzone_updates_per_s": round(zones / (ms_sep * 1e-3) / 1e6, 1)}
        for c in ctxs:
            c.check()
            c.close()
        del ctxs
        torch.cuda.empty_cache()
    rec["batch_vs_separate"] = round(rec["separate_contexts"]["ms_per_step"] / ms, 3)
    rec["split_contexts_vs_batch"] = round(ms / rec["separate_split_contexts"]["ms_per_step"], 3)
    rec["split_batch_vs_batch"] = round(ms / rec["split_batch"]["ms_per_step"], 3)
    return rec


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if args.impl == "reference":
        if rank != 0:
            return 0
        batch = build_batch(args.instances, args.seed)
        cb = run_cpu_reference(batch, args.steps, args.warmup)
        line = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": round(cb["per_step_s"] * 1e3, 3), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded blast-wave initial conditions)", "impl": "reference",
                "config": {"workload": "uneven 2D MHD blast batch (bounded CPU sample, see cpu_baseline)",
                           "instances": args.instances},
                "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
                "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        cs = run_cpu_reference(batch, steps=1, warmup=1, rows_parallel=0)
        line["cpu_baseline_reference_structure"] = {k: cs[k] for k in ("value", "unit", "cores", "kind",
                                                                          "sample")}
        print(json.dumps(line), flush=True)
        return 0
    if args.configs_only:
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        if rank == 0:
            print(json.dumps({"metric": METRIC, "configs_3d": run_configs(n3d=args.n3d, names=args.config_names.split(","),
                                                                         paths=args.config_paths.split(","))}),
                  flush=True)
        return 0
    if args.adjoint_only:
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        if rank == 0:
            print(json.dumps({"metric": METRIC, "adjoint": run_adjoint()}), flush=True)
        return 0
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    line = run_ours(args, rank, world, dist)
    if rank == 0 and not args.no_adjoint:
        line["adjoint"] = run_adjoint()
    if rank == 0 and world == 1 and not args.no_configs:
        line["configs_3d"] = run_configs(n3d=args.n3d, names=args.config_names.split(","),
                                         paths=args.config_paths.split(","))
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        batch = build_batch(args.instances, args.seed)
        cb = run_cpu_reference(batch, steps=2, warmup=1)
        line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
        cs = run_cpu_reference(batch, steps=1, warmup=1, rows_parallel=0)
        line["cpu_baseline_reference_structure"] = {k: cs[k] for k in ("value", "unit", "cores", "kind",
                                                                          "sample")}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
