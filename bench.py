#!/usr/bin/env python3
"""Benchmark: packets/s of one iteration of the transport + balance path.

A step is one iteration of the reference driver loop (main.f90:128-185) on
the Stromgren workload (stromgren64: 64^3 Cartesian grid, n_H = 100, 40 kK
point source, Q(H) = 1e49 s^-1, 1e6 Owen-scrambled Sobol packets, case B,
T_e = 1e4 K, FP64): the transport pass (launch, DDA walk, rate tallies,
energy ledger, rate normalisation) followed by the per-leaf balance and the
absorber-column refresh.  Before timing, the nebula is iterated (untimed,
as input preparation) to a converged ionisation structure so every timed
step walks the converged Stromgren sphere, as the bulk of a real run does.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

value     packets / device time of the K steps (CUDA events on the
          library's stream), L2 flushed between steps (a 256 MiB write).
e2e       the same metric through the C ABI with host buffers: each step
          uploads the leaf ionisation state from pinned host memory and
          reads back the new state and Gamma_HI, copies inside the timing.
roofline  the transport kernel: algorithmic bytes (56 B per scored
          segment: one FP64 absorber column read and three FP64 tally
          read-modify-writes) per launch / its event-timed duration.
N > 1     one process per GPU, each an independent nebula (replicas: the
          packets of one nebula are not split across GPUs), value = sum.
--impl reference
          the CPU restatement of the reference's path (the oracle port) on
          every host thread, on a bounded packet sample of the same
          workload per step.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "packets/s on 1 B200 (transport + balance iteration)"
UNIT = "packets/s"
WORKLOAD = "stromgren64"
NPHOT = 1_000_000
GRID = 64
BYTES_PER_SEGMENT = 56
# DRAM bytes per scored segment of the transport kernel, from the ncu
# capture summarised in profiles/transport_stromgren64.md (None until
# captured).
DRAM_BYTES_PER_SEGMENT = None


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.3)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out = ""
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            p = [x.strip() for x in l.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def oracle_baseline(nphot_sample, nthreads):
    """The oracle port (FP64 CPU restatement, OpenMP) on a bounded sample:
    one converged-state transport pass + balance of nphot_sample packets."""
    from mochii_b200 import configs
    from oracle import pyorc
    nl = configs.stromgren64(nphotons=nphot_sample, n=GRID)
    sim = pyorc.Sim(nl, nthreads=nthreads)
    return sim


def converged_state(neb, max_iter=60, tol=1e-3):
    it = 0
    for it in range(1, max_iter + 1):
        neb.ionizing_field_and_rates()
        dx, _ = neb.gas_equilibrium_update()
        neb.gas_opacity_fill()
        if dx < tol:
            break
    return it


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    import numpy as np
    from oracle import pyorc
    from mochii_b200 import configs
    nthreads = os.cpu_count() or 1
    sample = int(os.environ.get("MOCHII_REF_SAMPLE", "200000"))
    nl = configs.stromgren64(nphotons=sample, n=GRID)
    sim = pyorc.Sim(nl, nthreads=nthreads)
    # the same converged structure as the GPU arm: a converged x_HI taken
    # from a cheap oracle iteration at this sample size
    for _ in range(40):
        sim.transport_pass()
        dx, _ = sim.equilibrium_update()
        if dx < 2e-3:
            break
    for _ in range(args.warmup):
        sim.transport_pass()
        sim.equilibrium_update()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        sim.transport_pass()
        sim.equilibrium_update()
    dt = time.perf_counter() - t0
    value = sample * args.steps / dt
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "grid": f"{GRID}^3", "packets_per_step": sample,
                       "note": "bounded packet sample of the 1e6-packet step"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": "port",
                             "sample": f"{sample} packets per step, converged Stromgren state"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mochii_b200")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"],
                    help="transport arithmetic (the workload is defined in fp64)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    rank, world, local = dist_env()
    import numpy as np
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    from mochii_b200 import Nebula, configs, parse_namelist
    from mochii_b200.build import build
    if rank == 0 or not os.path.exists(os.path.join(ROOT, "mochii_b200", "libmochii_gpu.so")):
        build()
    if dist is not None:
        dist.barrier()

    par = parse_namelist(configs.stromgren64(nphotons=NPHOT, n=GRID, seed=12345 + rank, precision=args.precision))
    neb = Nebula(par)
    prep_iters = converged_state(neb)
    tuning = neb.autotune(1 << 18)   # launch shape for this grid / precision / device
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    for _ in range(args.warmup):
        neb.ionizing_field_and_rates()
        neb.gas_equilibrium_update()
        neb.gas_opacity_fill()

    # ---- device-timed steps ---------------------------------------------
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    pass_ms, kern_ms, bal_ms, segs = [], [], [], []
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        t_wall = time.perf_counter()
        for k in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            st = neb.ionizing_field_and_rates()
            neb.gas_equilibrium_update()
            neb.gas_opacity_fill()
            pass_ms.append(st.pass_ms)
            kern_ms.append(st.kernel_ms)
            bal_ms.append(neb.last_metrics.kernel_ms)
            segs.append(st.direct_segments)
        torch.cuda.synchronize()
        t_wall = time.perf_counter() - t_wall
    # Each API call synchronises its own stream and reports the device time
    # (CUDA events on the library's stream) of its work: the pass (tally
    # reset, transport, rate normalisation) and the balance (solve + column
    # refresh); a step is their sum.
    step_ms = [a + b for a, b in zip(pass_ms, bal_ms)]
    total_ms = sum(step_ms)
    if dist is not None:
        t = torch.tensor([total_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = NPHOT * args.steps * world / (total_ms * 1e-3)

    # ---- end-to-end through the C ABI with host buffers --------------------
    nleaf = neb.nleaf
    x_host = torch.from_numpy(neb.get("x_HI")).pin_memory()
    x_out = torch.empty(nleaf, dtype=torch.float64).pin_memory()
    g_out = torch.empty(nleaf, dtype=torch.float64).pin_memory()
    lib, ctx = neb.lib, neb.ctx
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = time.perf_counter()
    for k in range(args.steps):
        rc = lib.mochii_set_field(ctx, b"x_HI", x_host.data_ptr(), nleaf)
        rc |= lib.mochii_opacity_fill(ctx)
        neb.ionizing_field_and_rates()
        neb.gas_equilibrium_update()
        rc |= lib.mochii_get_field(ctx, b"x_HI", x_out.data_ptr(), nleaf)
        rc |= lib.mochii_get_field(ctx, b"gamma_HI", g_out.data_ptr(), nleaf)
        assert rc == 0
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - e0
    if dist is not None:
        t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = NPHOT * args.steps * world / e2e_s

    # ---- roofline of the transport kernel -------------------------------------
    peak, peak_kind = peaks()
    mean_seg = float(np.mean(segs))
    mean_ms = float(np.mean(kern_ms))
    achieved = BYTES_PER_SEGMENT * mean_seg / (mean_ms * 1e-3) / 1e9
    traffic = DRAM_BYTES_PER_SEGMENT * mean_seg if DRAM_BYTES_PER_SEGMENT else None

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import pyorc
        nthreads = os.cpu_count() or 1
        sample = int(os.environ.get("MOCHII_CPU_SAMPLE", "200000"))
        sim = pyorc.Sim(configs.stromgren64(nphotons=sample, n=GRID), nthreads=nthreads)
        sim.set("x_HI", x_host.numpy())
        t0 = time.perf_counter()
        reps = 0
        while True:
            sim.transport_pass()
            sim.equilibrium_update()
            sim.set("x_HI", x_host.numpy())
            reps += 1
            if time.perf_counter() - t0 > 10.0 or reps >= 20:
                break
        dt = time.perf_counter() - t0
        cpu = {"value": sample * reps / dt, "unit": UNIT, "cores": nthreads, "kind": "port",
               "sample": f"{reps} iterations of {sample} packets on the same converged state"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
            "data": "synthetic", "config": {"workload": WORKLOAD, "grid": f"{GRID}^3", "packets_per_step": NPHOT,
                       "precision": args.precision, "state": f"converged Stromgren sphere ({prep_iters} prep iterations)",
                       "l2": "flushed between steps (256 MiB write)",
                       "tuning": tuning,
                       "parallelism": "replicas" if world > 1 else "single"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 8 * nleaf,
                    "d2h_bytes_per_step": 16 * nleaf},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": traffic, "kernel": "k_transport",
                         "bytes_per_segment": BYTES_PER_SEGMENT, "segments_per_launch": mean_seg,
                         "kernel_ms": mean_ms},
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
            "gpu_launches": 3 * args.steps,
            "breakdown_ms": {"transport": float(np.mean(pass_ms)), "balance": float(np.mean(bal_ms))},
            "wall_s": t_wall,
        }
        print(json.dumps(line), flush=True)
    neb.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
