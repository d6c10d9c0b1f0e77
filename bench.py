#!/usr/bin/env python3
"""Benchmark: packets/s of one iteration of the transport + balance path.

A step is one iteration of the reference driver loop (main.f90:128-185):
the transport pass (Sobol launch, DDA walk, rate tallies, diffuse Milne
packets, energy ledger, rate normalisation) followed by the per-leaf balance
(thermal balance where the workload solves T_e) and the opacity refresh.

Workloads (--workload):
  hii_metals128  (default) the H+He+metals H II region with the thermal
                 balance: 128^3 grid, n_H = 100, He/H 0.1, eleven metals,
                 45 kK blackbody with Q(H) = 5e49 s^-1, case A with explicit
                 diffuse Milne packets, 1e7 stellar packets per pass, FP32
                 segments with FP64 atomic tallies (--tally compensated for
                 the (hi, lo) FP32 pairs; metal rates from
                 the energy-moment tallies).  Untimed preparation iterations
                 bring the ionized start to a developed H II region first.
  stromgren64    the pure-H Stromgren sphere: 64^3, 40 kK, Q(H) = 1e49,
                 1e6 packets, case B, T_e = 1e4 K, FP64; prepared to the
                 converged sphere.
  clumpy_dusty   the dusty clumpy nebula on an octree of about 3e6 leaves
                 (log-normal n_H, mean 30, from a seeded 256^3 random field;
                 base level 6, refined towards level 10), three point
                 sources (35/40/50 kK, Q(H) = 2e49 each), MW R_V = 3.1 grains
                 with <cos> = 0.6 and scattering, FUV band from 6 eV, T_e
                 solved (H + He), 3e7 packets per pass, FP32 segments.  The
                 leaf list is generated once into the temp directory.
  batch64        64 independent H II regions advanced together (the batch
                 API: one CUDA graph per iteration, one persistent thermal
                 launch for all): seeded cubic grids of 32^3..128^3, n_H
                 log-uniform in 10-1000, T_eff 30-50 kK, Q(H) 1e48-1e50,
                 He/H 0.1 and the eleven metals, case A, 2e6 packets per
                 instance per iteration, T_e solved, FP32 segments.  A step
                 is one iteration of all 64.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload W] [--impl reference]

value     packets transported (stellar + diffuse) / device time of the K
          steps (CUDA events on the library's stream), L2 flushed between
          steps (a 256 MiB write).
e2e       the same metric through the C ABI with host buffers: each step
          uploads the leaf state (x_HI, T_e) from pinned host memory and
          reads back x_HI, T_e and Gamma_HI, copies inside the timing.
roofline  the transport kernels: algorithmic bytes per scored segment
          B_seg = 4 F_state + 16 F_tally (state words read, 8-byte tallies
          (FP64, or a compensated FP32 pair) read and written; FP64 state
          words count 8 B) over their
          event-timed duration; the metal state words are counted per
          segment in the kernel (one per active transition).
N > 1     one process per GPU, each an independent nebula (replicas: the
          packets of one nebula are not split across GPUs), value = sum.
--impl reference
          the CPU restatement of the reference's path (the oracle port) on
          every host thread: a bounded packet sample of the same workload
          and the thermal solve on a sample of its leaves, scaled to the
          step's packet and leaf counts.
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

METRIC = "packets/s on 1 B200 (transport + balance iteration)"
UNIT = "packets/s"


# DRAM bytes (read + written) per scored segment of the transport pass (keys, sort, launch,
# coherent walk, diffuse launch and walk) from the ncu launch list summarised
# in profiles/walk_coh_hii96.md: hii_metals at 96^3 (FP32 segments, FP64
# tallies, FP32 moments), 15.33 GB over 5.554e8 segments; scaled to the
# 128^3 pass by its segment count.
DRAM_BYTES_PER_SEGMENT = {"hii_metals128": (27.6, "derived: ncu DRAM bytes of the 96^3 case's transport-pass "
                                                  "launches per scored segment, times this pass's segments")}


# FP64 work of the thermal solve per net-rate evaluation: DADD + DMUL +
# 2 DFMA thread instructions of the per-lane solve's 96^3 update (ncu,
# profiles/thermal_lane_hii96.md), 69.9e9 FLOP over 1 659 987 evaluations.
FP64_FLOP_PER_EVALUATION = 42100.0
FP64_PEAK_TFLOPS = 148 * 64 * 2 * 1.965e9 / 1e12


class Workload:
    """A benchmark configuration: its namelist and how a step is run."""

    def __init__(self, name, grid=None, packets=None):
        """grid / packets override the workload's grid side and stellar
        packets per pass (smaller cases for profiling)."""
        from mochii_b200 import configs
        self.name = name
        if name == "hii_metals128":
            self.grid, self.nphot, self.thermal, self.prep = grid or 128, packets or 10_000_000, True, 8
            self.default_precision = "fp32"
            n = self.grid
            self.make = lambda nphot, prec, seed: configs.hii_metals(nphotons=nphot, niter=20, n=n,
                                                                      precision=prec, seed=seed)
        elif name == "stromgren64":
            self.grid, self.nphot, self.thermal, self.prep = grid or 64, packets or 1_000_000, False, 60
            self.default_precision = "fp64"
            n = self.grid
            self.make = lambda nphot, prec, seed: configs.stromgren64(nphotons=nphot, n=n, precision=prec, seed=seed)
        elif name == "clumpy_dusty":
            import tempfile
            cases = os.path.join(tempfile.gettempdir(), "mochii_b200_cases")
            self.grid, self.nphot, self.thermal, self.prep = None, packets or 30_000_000, True, 3
            self.default_precision = "fp32"
            self.make = lambda nphot, prec, seed: configs.clumpy_dusty(cases, nphotons=nphot, precision=prec,
                                                                        qmc_seed=seed)
        elif name == "batch64":
            self.grid, self.nphot, self.thermal, self.prep = None, packets or 2_000_000, True, 0
            self.default_precision = "fp32"
            self.count = 64
            self.make = None   # one namelist per instance: instances()
        else:
            raise SystemExit(f"unknown workload {name}")

    def instances(self, prec, extra=""):
        """batch64: the instances' namelists (with extra keys) and their
        (n, n_H, T_eff, Q) parameters."""
        from mochii_b200 import configs
        nls, par = configs.batch_instances(count=self.count, nphotons=self.nphot, precision=prec)
        return [nl.replace("/\n", extra + "/\n") for nl in nls], par

    def balance(self, neb):
        return neb.gas_thermal_update() if self.thermal else neb.gas_equilibrium_update()

    def state(self):
        """The analytic developed state every step starts from (Cartesian
        workloads; configs.prepared_state), or None: the octree and batch
        workloads run from their configured start after preparation
        iterations."""
        from mochii_b200 import configs
        if self.name == "hii_metals128":
            return configs.prepared_state(self.grid, front=0.7, he=True)
        if self.name == "stromgren64":
            return configs.prepared_state(self.grid, front=1.0, he=False, T_in=1.0e4, T_out=1.0e4)
        return None

    def cpu_fraction(self):
        """The CPU reference times 1/f of a step: 1/f of the stellar packets
        (and so of the diffuse ones) and the balance of every f-th leaf."""
        if not self.thermal:
            return 1
        return 200 if (self.grid or 0) >= 96 else 100


def set_state(target, state):
    """Upload a state dict (x_HI, x_HeI, x_HeII, n_e, T_e) to a Nebula or an
    oracle Sim and refresh the opacities it implies."""
    for k, v in state.items():
        target.set(k, v)
    if hasattr(target, "gas_opacity_fill"):
        target.gas_opacity_fill()


def bytes_per_segment(wl, precision, tally="fp64"):
    """B_seg = 4 F_state + 16 F_tally without the per-segment metal words
    (added from the kernel's count), state words 8 B in FP64; the six metal
    moment words are FP32 (8 B each, read and written) with FP32 segments and
    FP64 tallies."""
    w = 8 if precision == "fp64" else 4
    if wl.name == "stromgren64":
        return w * 2 + 16 * 3          # n_H, x_HI; Gamma_HI, H_HI, jt_ion
    if wl.name == "clumpy_dusty":
        return w * 5 + 16 * 9          # n_H, x_HI, x_HeI, x_HeII, rhokap; 6 H/He + jt_ion + dust_abs + FUV
    if wl.name == "batch64":
        return w * 4 + 16 * 7          # n_H, x_HI, x_HeI, x_HeII; 6 H/He + jt_ion (metal words per segment)
    mom = 8 if precision == "fp32" and tally == "fp64" else 16
    return w * 4 + 16 * 7 + mom * 6   # n_H, x_HI, x_HeI, x_HeII; 6 H/He + jt_ion; 6 metal moments


def prepare(neb, wl):
    it = 0
    for it in range(1, wl.prep + 1):
        neb.ionizing_field_and_rates()
        m = wl.balance(neb)
        neb.gas_opacity_fill()
        if not wl.thermal and m[0] < 1e-3:
            break
    return it


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


def cpu_threads(wl):
    """Host threads for the CPU port: all cores, capped so the per-thread
    tally copies (the reference's per-rank tallies) use at most half the
    host memory."""
    n = os.cpu_count() or 1
    try:
        mem = os.sysconf("SC_PAGE_SIZE") * os.sysconf("SC_PHYS_PAGES")
    except (ValueError, OSError):
        mem = 64 << 30
    nleaf = wl.grid ** 3 if wl.grid else (128 ** 3 if wl.name == "batch64" else 3_100_000)
    metals = wl.name in ("hii_metals128", "batch64")
    per = nleaf * 8 * (6 + 16 + (2 * 32 if metals else 0) + (2 if wl.name == "clumpy_dusty" else 0))
    return max(1, min(n, int(0.5 * mem // max(per, 1))))


def cpu_reference(wl, nthreads, steps=1, warmup=1, state=None):
    """The reference's algorithm (the oracle port: FP64, OpenMP over packets
    and leaves, the reference's damped n_e fixed point and bisection on T_e)
    on 1/f of the workload's step, measured: a transport pass of nphot/f
    stellar packets (and the diffuse packets their luminosity implies) and
    the thermal bisection of every f-th leaf (f = wl.cpu_fraction(); the
    ionisation-only workload runs whole steps).  Every step starts from the
    workload's analytic state (or `state`), as the device steps do; warm-up
    steps first give the metal stage fractions the rates of a pass on that
    state.  Returns (packets/s, description, seconds per sample step, packets
    per sample step)."""
    from oracle import pyorc
    f = wl.cpu_fraction()
    nph = max(wl.nphot // f, 1)
    sim = pyorc.Sim(wl.make(nph, "fp64", 12345), nthreads=nthreads)
    st0 = state if state is not None else wl.state()
    idx = np.arange(0, sim.nleaf, f, dtype=np.int64)
    times, pk = [], []
    # the sample steps leave the state as they find it (the pass writes
    # tallies and rates, the sampled solve returns its leaves without writing
    # them), so the state is set once, and again after the warm-up so that the
    # metal stage fractions carry the rates of a pass on it, as on the device
    if st0 is not None:
        sim.set_state(st0)
    for k in range(warmup + steps):
        if st0 is not None and (k == warmup or (k > 0 and not wl.thermal)):   # the ionisation solve writes the state
            sim.set_state(st0)
        t0 = time.perf_counter()
        sim.transport_pass()
        if wl.thermal:
            sim.thermal_cells(idx)
        else:
            sim.equilibrium_update()
        dt = time.perf_counter() - t0
        if k >= warmup:
            times.append(dt)
            pk.append(nph + sim.diffuse_count)
    t_step = float(np.mean(times))
    value = float(np.sum(pk)) / float(np.sum(times))
    what = (f"the thermal bisection of every {f}th leaf ({idx.size} leaves)" if wl.thermal
            else "the ionisation solve of every leaf")
    desc = (f"{'1/' + str(f) + ' of ' if f > 1 else ''}a step, measured: {nph} stellar packets plus their "
            f"{int(np.mean(pk)) - nph} diffuse packets, then {what}, from the workload's analytic state; "
            f"{steps} timed step(s) after {warmup} warm-up; {nthreads} threads")
    return value, desc, t_step, float(np.mean(pk))


class InstanceWorkload:
    """One batch64 instance as a single-nebula workload (for the CPU port),
    from its configured ionized start."""

    def __init__(self, p, nphot):
        from mochii_b200 import configs
        self.name, self.grid, self.nphot, self.thermal = "batch_instance", p["n"], nphot, True
        self.make = lambda nphot_, prec, seed: configs.hii_instance(p["n"], p["nH"], p["tstar"], p["Q"],
                                                                     nphotons=nphot_, precision=prec, seed=seed)

    def state(self):
        return None

    def cpu_fraction(self):
        return 100


def cpu_reference_batch(wl, nthreads, steps=1):
    """The oracle port on three batch64 instances (the smallest, the median
    and the largest grid), each measured on 1/100 of its step from its
    configured start: packets over time summed over the three."""
    _, par = wl.instances("fp64")
    order = sorted(range(len(par)), key=lambda k: par[k]["n"])
    pick = [order[0], order[len(order) // 2], order[-1]]
    pk, tt, ns = 0.0, 0.0, []
    for k in pick:
        iw = InstanceWorkload(par[k], wl.nphot)
        _, _, t_step, p_step = cpu_reference(iw, nthreads, steps=steps, warmup=1)
        pk += p_step
        tt += t_step
        ns.append(par[k]["n"])
    desc = (f"instances of {ns[0]}^3, {ns[1]}^3, {ns[2]}^3 from their configured start, each on 1/100 of a step "
            f"(stellar packets and every 100th leaf's thermal bisection), measured; {nthreads} threads")
    return pk / tt, desc, tt


def run_reference(args, wl):
    """--impl reference: the reference's algorithm (the oracle port) on the
    host cores, every step 1/f of the workload's step from the same analytic
    state the device steps start from, each step measured."""
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    nthreads = cpu_threads(wl)
    if wl.name == "batch64":
        value, desc, t_step = cpu_reference_batch(wl, nthreads, steps=args.steps)
        p_step = value * t_step
    else:
        value, desc, t_step, p_step = cpu_reference(wl, nthreads, steps=args.steps, warmup=args.warmup)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_step * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": config_of(wl),
            "sample": {"packets_per_step": p_step, "fraction_of_step": 1.0 / wl.cpu_fraction(),
                       "note": "each timed step is the stated fraction of the workload's step, measured (not scaled)"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": "port", "sample": desc},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def config_of(wl, nleaf=None):
    """The workload's identity, the same for the device arm and the
    reference arm."""
    cfg = {"workload": wl.name, "grid": grid_name(wl, nleaf), "stellar_packets_per_step": wl.nphot,
           "balance": "thermal" if wl.thermal else "ionisation, fixed T_e"}
    if wl.name == "batch64":
        cfg.update({"instances": wl.count, "state": "each instance's configured ionized start"})
    elif wl.state() is not None:
        cfg["state"] = ("from the analytic developed H II region of configs.prepared_state (the device iterates from "
                        "it; the reference's bisection costs the same from any start)")
    else:
        cfg["state"] = f"{wl.prep} preparation iterations from the configured start"
    return cfg


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mochii_b200")
    ap.add_argument("--workload", default="hii_metals128",
                    choices=["hii_metals128", "stromgren64", "clumpy_dusty", "batch64"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-converge", action="store_true", help="skip the time-to-converged comparison")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the dusty-octree and batched-nebulae figures the default run adds")
    ap.add_argument("--precision", default=None, choices=["fp64", "fp32"],
                    help="transport arithmetic (default: the workload's)")
    ap.add_argument("--solver", default="bracketed", choices=["bisection", "bracketed"],
                    help="cell solver: the reference's bisection or the bracketed roots")
    ap.add_argument("--cell-layout", default="lane", choices=["lane", "lockstep", "flow", "warp"],
                    help="thermal solve with metals: per-lane machines with the cache in shared memory, "
                         "lockstep nested loops, one flat machine per leaf, or one warp per leaf")
    ap.add_argument("--tally", default="fp64", choices=["fp64", "compensated"],
                    help="path tallies with FP32 segments: compensated FP32 pairs or FP64 atomics")
    ap.add_argument("--order", default=None, choices=["launch", "direction", "coherent"],
                    help="walk order of the stellar packets (default: the library's)")
    ap.add_argument("--grid", type=int, default=None, help="grid side of a Cartesian workload (default: its own)")
    ap.add_argument("--packets", type=int, default=None, help="stellar packets per pass (default: the workload's)")
    args = ap.parse_args()
    wl = Workload(args.workload, args.grid, args.packets)
    prec = args.precision or wl.default_precision
    if args.impl == "reference":
        return run_reference(args, wl)
    if wl.name == "batch64":
        return run_batch(args, wl, prec)

    rank, world, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    from mochii_b200 import Nebula, parse_namelist
    from mochii_b200.build import build
    if rank == 0 or not os.path.exists(os.path.join(ROOT, "mochii_b200", "libmochii_gpu.so")):
        build()
    if dist is not None:
        dist.barrier()

    order = f" par%packet_order = '{args.order}'\n" if args.order else ""
    par = parse_namelist(wl.make(wl.nphot, prec, 12345 + rank).replace(
        "/\n", f" par%thermal_solver = '{args.solver}'\n par%cell_layout = '{args.cell_layout}'\n"
              f" par%tally_precision = '{args.tally}'\n{order}/\n"))
    neb = Nebula(par)
    state0 = wl.state()
    if state0 is not None:
        set_state(neb, state0)
    else:
        prepare(neb, wl)
    tuning = neb.autotune(1 << 20)   # launch shape for this grid / precision / device

    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    if state0 is not None:   # the autotuner's trial passes and solves leave the start state in place
        set_state(neb, state0)
    for _ in range(args.warmup):
        neb.ionizing_field_and_rates()
        wl.balance(neb)
        neb.gas_opacity_fill()

    # ---- device-timed steps ---------------------------------------------
    pass_ms, kern_ms, bal_ms, segs, nact, npk, bcnt = [], [], [], [], [], [], []
    # each timed step's start state, kept on the host (untimed) so that the
    # end-to-end steps below redo exactly these steps from host buffers
    fields = ("x_HI", "x_HeI", "x_HeII", "n_e", "T_e")
    step_in = []
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        t_wall = time.perf_counter()
        torch.cuda.nvtx.range_push("timed")   # ncu --nvtx --nvtx-include "timed/" selects these launches
        for k in range(args.steps):
            step_in.append({f: neb.get(f) for f in fields})
            flush.zero_()
            torch.cuda.synchronize()
            st = neb.ionizing_field_and_rates()
            wl.balance(neb)
            neb.gas_opacity_fill()
            pass_ms.append(st.pass_ms)
            kern_ms.append(st.kernel_ms)
            bal_ms.append(neb.last_metrics.kernel_ms)
            lm = neb.last_metrics
            bcnt.append((lm.cells_solved, lm.rate_evaluations, lm.metal_sum_calls, lm.fixed_point_passes))
            segs.append(st.direct_segments)
            nact.append(st.metal_active)
            npk.append(st.packets)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        t_wall = time.perf_counter() - t_wall
    # Each API call synchronises its own stream and reports the device time
    # (CUDA events on the library's stream) of its work: the pass (tally
    # reset, transport, rate normalisation) and the balance (solve + opacity
    # refresh); a step is their sum.
    step_ms = [x + y for x, y in zip(pass_ms, bal_ms)]
    total_ms = sum(step_ms)
    packets = sum(npk)
    if dist is not None:
        t = torch.tensor([total_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        p = torch.tensor([float(packets)], device="cuda", dtype=torch.float64)
        dist.all_reduce(p, op=dist.ReduceOp.SUM)
        packets = int(p.item())
    value = packets / (total_ms * 1e-3)

    # ---- end-to-end through the C ABI with host buffers --------------------
    nleaf = neb.nleaf
    # step k's inputs: the start state of timed step k (every field of it)
    # from pinned host memory
    host_in = [{f.encode(): torch.from_numpy(np.ascontiguousarray(v, dtype=np.float64)).pin_memory()
                for f, v in src.items()} for src in step_in]
    del step_in
    x_out = torch.empty(nleaf, dtype=torch.float64).pin_memory()
    t_out = torch.empty(nleaf, dtype=torch.float64).pin_memory()
    g_out = torch.empty(nleaf, dtype=torch.float64).pin_memory()
    lib, ctx = neb.lib, neb.ctx
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    e_packets = 0
    e0 = time.perf_counter()
    for k in range(args.steps):
        rc = 0
        for f, hb in host_in[k].items():
            rc |= lib.mochii_set_field(ctx, f, hb.data_ptr(), nleaf)
        rc |= lib.mochii_opacity_fill(ctx)
        st = neb.ionizing_field_and_rates()
        e_packets += st.packets
        wl.balance(neb)
        rc |= lib.mochii_get_field(ctx, b"x_HI", x_out.data_ptr(), nleaf)
        rc |= lib.mochii_get_field(ctx, b"T_e", t_out.data_ptr(), nleaf)
        rc |= lib.mochii_get_field(ctx, b"gamma_HI", g_out.data_ptr(), nleaf)
        assert rc == 0
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - e0
    if dist is not None:
        t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
        p = torch.tensor([float(e_packets)], device="cuda", dtype=torch.float64)
        dist.all_reduce(p, op=dist.ReduceOp.SUM)
        e_packets = int(p.item())
    e2e_value = e_packets / e2e_s

    # ---- roofline of the transport kernels -----------------------------------
    peak, peak_kind = peaks()
    wbytes = 8 if prec == "fp64" else 4
    bseg = bytes_per_segment(wl, prec, args.tally)
    alg_bytes = float(np.mean([bseg * s_ + wbytes * a_ for s_, a_ in zip(segs, nact)]))
    mean_seg = float(np.mean(segs))
    mean_ms = float(np.mean(kern_ms))
    achieved = alg_bytes / (mean_ms * 1e-3) / 1e9
    traffic, traffic_kind = None, None
    if DRAM_BYTES_PER_SEGMENT.get(wl.name) and prec == "fp32" and args.tally == "fp64":   # the captured configuration
        b_, kind_ = DRAM_BYTES_PER_SEGMENT[wl.name]
        traffic, traffic_kind = b_ * mean_seg, kind_

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        nthreads = cpu_threads(wl)
        # the same start state as the device steps (octree: the configured start)
        v, desc, _, _ = cpu_reference(wl, nthreads, steps=2, warmup=1)
        cpu = {"value": v, "unit": UNIT, "cores": nthreads, "kind": "port", "sample": desc}

    conv = None
    if rank == 0 and not args.no_converge and wl.name == "hii_metals128":
        conv = time_to_converged()
    extras = None
    if rank == 0 and world == 1 and not args.no_extras and wl.name == "hii_metals128" and wl.grid == 128:
        extras = run_extras()
    # the thermal solve (the step's other kernel): leaves and net-rate
    # evaluations per second of its device time
    bm = np.mean(np.array(bcnt, dtype=float), axis=0)
    bal_s = float(np.mean(bal_ms)) * 1e-3
    balance = {"cells_per_s": bm[0] / bal_s, "net_rate_evaluations_per_s": bm[1] / bal_s,
               "evaluations_per_cell": bm[1] / max(bm[0], 1.0), "kernel_ms": bal_s * 1e3}
    if wl.name == "hii_metals128" and wl.thermal:
        fl = FP64_FLOP_PER_EVALUATION * bm[1] / bal_s
        balance["fp64"] = {"flop_per_evaluation": FP64_FLOP_PER_EVALUATION,
                           "flop_source": "ncu DADD + DMUL + 2 DFMA thread instructions of one 96^3 update over its "
                                          "counted evaluations",
                           "achieved_tflops": fl / 1e12, "peak_tflops": FP64_PEAK_TFLOPS,
                           "peak_kind": "nominal: 148 SMs x 64 FP64 FMA per clock x 2 x 1.965 GHz",
                           "frac": fl / 1e12 / FP64_PEAK_TFLOPS}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if prec == "fp64" else "f32+f64",
            "data": "synthetic",
            "config": config_of(wl, nleaf),
            "implementation": {"packets_per_step": packets / args.steps / world, "precision": prec,
                               "solver": args.solver, "cell_layout": args.cell_layout, "tallies": args.tally,
                               "packet_order": neb_order(neb), "l2": "flushed between steps (256 MiB write)",
                               "tuning": tuning, "parallelism": "replicas" if world > 1 else "single"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 8 * len(fields) * nleaf,
                    "d2h_bytes_per_step": 24 * nleaf},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": traffic, "traffic_kind": traffic_kind,
                         "kernel": ("transport pass: k_coherent_keys, key sort, k_launch, k_walk_coh (stellar "
                                    "chunks); k_diffuse_keys, key sort, k_launch_diffuse, k_walk_coh (diffuse "
                                    "chunks)"
                                    if neb_order(neb) == "coherent" else "transport pass: k_launch + k_walk_edge"),
                         "bytes_per_segment": alg_bytes / mean_seg, "segments_per_launch": mean_seg,
                         "kernel_ms": mean_ms},
            "cpu_baseline": cpu,
            "time_to_converged": conv,
            "clocks": clk.summary(),
            "gpu_launches": int(sum(launches_per_step(wl, n_ - wl.nphot, neb_order(neb) == "coherent" and wl.grid)
                                    for n_ in npk)),
            "breakdown_ms": {"transport": float(np.mean(pass_ms)), "balance": float(np.mean(bal_ms))},
            "balance_counts_per_step": dict(zip(("cells", "rate_evaluations", "metal_sums", "ne_evaluations"),
                                                (float(v) for v in bm))),
            "balance": balance,
            "wall_s": t_wall,
        }
        if extras:
            line["extras"] = extras
        print(json.dumps(line), flush=True)
    neb.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_batch(args, wl, prec):
    """batch64: the instances as one Batch (mochii_batch_*); a step is one
    iteration of every instance, timed by the library's CUDA events around
    the graph launch.  After the timed steps, one iteration per instance
    through the single-nebula calls gives the transport kernels' own time
    (roofline) and the unbatched step time for comparison."""
    rank, world, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    from mochii_b200 import Batch, Nebula, parse_namelist
    from mochii_b200.build import build
    if rank == 0 or not os.path.exists(os.path.join(ROOT, "mochii_b200", "libmochii_gpu.so")):
        build()
    if dist is not None:
        dist.barrier()
    extra = (f" par%thermal_solver = '{args.solver}'\n par%cell_layout = '{args.cell_layout}'\n"
             f" par%tally_precision = '{args.tally}'\n par%packet_chunk = 1048576\n")
    nls, par = wl.instances(prec, extra)
    t0 = time.perf_counter()
    nebs = [Nebula(parse_namelist(nl)) for nl in nls]
    tuned = {}
    for neb, p_ in zip(nebs, par):   # walk shape per grid size, before the graph is recorded
        tuned[p_["n"]] = neb.autotune(1 << 18)
    batch = Batch(nebs)
    t_setup = time.perf_counter() - t0
    nleaf = [neb.nleaf for neb in nebs]
    free, total = torch.cuda.mem_get_info()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    for _ in range(args.warmup):
        batch.iterate()

    ms_steps, packets, segs, nact, bcnt = [], 0, [], [], []
    # each timed step's start state of every instance, kept on the host
    # (untimed) so that the end-to-end steps below redo exactly these steps
    fields = ("x_HI", "x_HeI", "x_HeII", "n_e", "T_e")
    step_in = []
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        t_wall = time.perf_counter()
        for _ in range(args.steps):
            step_in.append([{f: torch.from_numpy(neb.get(f)).pin_memory() for f in fields} for neb in nebs])
            flush.zero_()
            torch.cuda.synchronize()
            st, m, ms = batch.iterate()
            ms_steps.append(ms)
            packets += sum(s_.packets for s_ in st)
            segs.append([s_.direct_segments for s_ in st])
            nact.append([s_.metal_active for s_ in st])
            bcnt.append([sum(getattr(x, f) for x in m)
                         for f in ("cells_solved", "rate_evaluations", "metal_sum_calls", "fixed_point_passes")])
        torch.cuda.synchronize()
        t_wall = time.perf_counter() - t_wall
    total_ms = sum(ms_steps)
    if dist is not None:
        t = torch.tensor([total_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        p = torch.tensor([float(packets)], device="cuda", dtype=torch.float64)
        dist.all_reduce(p, op=dist.ReduceOp.SUM)
        packets = int(p.item())
    value = packets / (total_ms * 1e-3)

    # ---- end-to-end: every instance's state of timed step k up from pinned
    # host buffers, the batch iteration, x_HI, T_e and Gamma_HI of every
    # instance back
    lib = nebs[0].lib
    outs = [[torch.empty(n, dtype=torch.float64).pin_memory() for _ in range(3)] for n in nleaf]
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    e_packets = 0
    e0 = time.perf_counter()
    for k in range(args.steps):
        rc = 0
        for neb, hin, n in zip(nebs, step_in[k], nleaf):
            for f, hb in hin.items():
                rc |= lib.mochii_set_field(neb.ctx, f.encode(), hb.data_ptr(), n)
            rc |= lib.mochii_opacity_fill(neb.ctx)
        st, _, _ = batch.iterate()
        e_packets += sum(s_.packets for s_ in st)
        for neb, o, n in zip(nebs, outs, nleaf):
            rc |= lib.mochii_get_field(neb.ctx, b"x_HI", o[0].data_ptr(), n)
            rc |= lib.mochii_get_field(neb.ctx, b"T_e", o[1].data_ptr(), n)
            rc |= lib.mochii_get_field(neb.ctx, b"gamma_HI", o[2].data_ptr(), n)
        assert rc == 0
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - e0
    if dist is not None:
        t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
        p = torch.tensor([float(e_packets)], device="cuda", dtype=torch.float64)
        dist.all_reduce(p, op=dist.ReduceOp.SUM)
        e_packets = int(p.item())
    e2e_value = e_packets / e2e_s

    # ---- one unbatched iteration: the transport kernels' own time and the
    # single-nebula step time
    kern_ms, pass_ms, bal_ms, useg, uact = 0.0, 0.0, 0.0, 0, 0
    for neb in nebs:
        s_ = neb.ionizing_field_and_rates()
        neb.gas_thermal_update()
        kern_ms += s_.kernel_ms
        pass_ms += s_.pass_ms
        bal_ms += neb.last_metrics.kernel_ms
        useg += s_.direct_segments
        uact += s_.metal_active
    batch.close()
    peak, peak_kind = peaks()
    w = 8 if prec == "fp64" else 4
    alg_bytes = bytes_per_segment(wl, prec) * useg + (w + 32) * uact
    achieved = alg_bytes / (kern_ms * 1e-3) / 1e9

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        nthreads = cpu_threads(wl)
        order = sorted(range(len(par)), key=lambda k: par[k]["n"])
        pick = [order[0], order[len(order) // 2], order[-1]]
        states = {k: {f: nebs[k].get(f) for f in ("x_HI", "x_HeI", "x_HeII", "n_e", "T_e")} for k in pick}
        v, desc, _ = cpu_reference_batch(wl, states, nthreads)
        cpu = {"value": v, "unit": UNIT, "cores": nthreads, "kind": "port", "sample": desc}
    for neb in nebs:
        neb.close()

    if rank == 0:
        n_all = int(sum(nleaf))
        chunks = sum(3 * -(-wl.nphot // 1048576) + 2 for _ in nebs)   # keys, launch, walk per chunk; rates
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if prec == "fp64" else "f32+f64",
            "data": "synthetic",
            "config": config_of(wl, n_all),
            "implementation": {"packets_per_step": packets / args.steps / world, "precision": prec,
                               "solver": args.solver, "cell_layout": args.cell_layout, "tallies": args.tally,
                               "metal_tallies": "exact", "packet_order": neb_order(nebs[0]),
                               "l2": "flushed between steps (256 MiB write)", "packet_chunk": 1048576,
                               "execution": "one CUDA graph per iteration (all passes, then one persistent thermal "
                                            "launch)",
                               "tuning": f"walk shape autotuned per grid size ({len(tuned)} sizes)",
                               "parallelism": "replicas" if world > 1 else "single"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 8 * len(fields) * n_all,
                    "d2h_bytes_per_step": 24 * n_all},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind, "traffic": None,
                         "kernel": "transport passes (keys, launch, walk; one unbatched iteration)",
                         "segments_per_step": useg, "kernel_ms": kern_ms},
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
            "gpu_launches": int(args.steps * (chunks + 1)),
            "unbatched_ms_per_step": {"transport": pass_ms, "balance": bal_ms, "total": pass_ms + bal_ms},
            "balance_counts_per_step": dict(zip(("cells", "rate_evaluations", "metal_sums", "ne_evaluations"),
                                                (float(v) for v in np.mean(np.array(bcnt, dtype=float), axis=0)))),
            "device_memory_gb": {"used": (total - free) / 1e9, "total": total / 1e9},
            "setup_s": t_setup, "wall_s": t_wall,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def solve_check(neb, sim, idx):
    """The device's next thermal update against the reference's bisection
    (the FP64 oracle) on the same inputs: the device state and rates before
    the update go to the oracle, which solves the leaves idx; returns a
    function that, called after the device update, gives the largest
    |dT_e| [K] and |dx_HII| over idx."""
    sim.set_state({f: neb.get(f) for f in ("x_HI", "x_HeI", "x_HeII", "n_e", "T_e")})
    for f in ("gamma_HI", "gamma_HeI", "gamma_HeII", "heat_HI", "heat_HeI", "heat_HeII", "gamma_metal", "heat_metal"):
        sim.set(f, np.ascontiguousarray(neb.get(f)).ravel())
    ref = sim.thermal_cells(idx)

    def after():
        T, x = neb.get("T_e")[idx], neb.get("x_HI")[idx]
        return float(np.max(np.abs(T - ref[:, 0]))), float(np.max(np.abs(x - ref[:, 1])))
    return after


def time_to_converged(n=64, nphot=1_000_000, iters=20, train_iters=10, seed_train=777, seed=12345, checks=(1, 10, 20),
                      nsample=3000):
    """Time to a converged nebula of the metals H II-region class (n^3, the
    128^3 workload's physics, FP32 transport) from its configured ionized
    start, `iters` transport + thermal iterations, three ways:
      plain      the reference's solver on the device (damped n_e fixed
                 point, bisection on log T over [te_min, te_max]);
      bracketed  the same roots by the bracketed search from the previous T_e;
      mlp        the bracketed search from the learned warm start: the MLP's
                 T_e is accepted where its net heating is below 1e-6 of
                 heating plus cooling, else it seeds a narrow first bracket.
    The MLP is trained first on the plain solver's (features, solved state)
    pairs of another nebula of the class (launch seed seed_train).  Device
    time from the library's CUDA events (the warm start's inference by host
    clock around its synchronous call).  Accuracy: at the iterations in
    `checks`, each arm's update of nsample leaves against the FP64 oracle's
    bisection on the same inputs (state and rates copied from the device).
    The final states of the arms are also compared with each other against
    the Monte Carlo noise of the iteration (the plain arm's last change)."""
    from oracle import pyorc
    from mochii_b200 import Nebula, configs, parse_namelist
    from mochii_b200.mlp import WarmStartMLP

    def nl_of(sd, prec="fp32"):
        return configs.hii_metals(nphotons=nphot, niter=iters, n=n, precision=prec, seed=sd)

    def neb_of(solver, sd):
        return Nebula(parse_namelist(nl_of(sd).replace("/\n", f" par%thermal_solver = '{solver}'\n/\n")))

    t0 = time.perf_counter()
    X, Y = [], []
    neb = neb_of("bisection", seed_train)
    for _ in range(train_iters):
        neb.ionizing_field_and_rates()
        X.append(WarmStartMLP.features(neb))
        neb.gas_thermal_update()
        Y.append(WarmStartMLP.targets(neb, X[-1]))
    neb.close()
    X, Y = np.concatenate(X), np.concatenate(Y)
    t_data = time.perf_counter() - t0
    mlp = WarmStartMLP(seed=1)
    t0 = time.perf_counter()
    losses = mlp.train(X, Y, epochs=20, batch=4096, lr=2e-3, seed=2)
    t_train = time.perf_counter() - t0
    sim = pyorc.Sim(nl_of(seed, "fp64"), nthreads=cpu_threads(Workload("hii_metals128", grid=n)))
    rng = np.random.default_rng(3)
    res = {}
    for mode in ("plain", "bracketed", "mlp"):
        neb = neb_of("bisection" if mode == "plain" else "bracketed", seed)
        ms, evals, accepted, acc, werr = 0.0, 0, 0, [], []
        prev_T = None
        for it in range(1, iters + 1):
            st = neb.ionizing_field_and_rates()
            ms += st.pass_ms
            check = None
            if it in checks:   # half the sample from the ionized leaves, where the solve iterates
                x = neb.get("x_HI")
                ion = np.flatnonzero(x < 0.9)
                k = min(nsample // 2, ion.size)
                idx = np.unique(np.concatenate([rng.choice(ion, k, replace=False) if k else ion[:0],
                                                rng.choice(x.size, nsample - k, replace=False)]))
                check = solve_check(neb, sim, idx)
            if mode == "mlp":
                e0 = time.perf_counter()
                mlp.warm_start(neb)          # synchronous: device features + inference
                ms += (time.perf_counter() - e0) * 1e3
                t_warm, t_prev = neb.get("T_warm"), neb.get("T_e")   # untimed: the start-point diagnostics
            if it == iters:
                prev_T = neb.get("T_e")
            neb.gas_thermal_update()
            ms += neb.last_metrics.kernel_ms
            evals += neb.last_metrics.rate_evaluations
            accepted += neb.last_metrics.warm_accepted
            if mode == "mlp":   # RMS distance in ln T of the solved T_e from the two possible starts
                t_new = neb.get("T_e")
                inner = (t_new > neb.par.te_min * (1 + 1e-9)) & (t_new < neb.par.te_max * (1 - 1e-9)) & (neb.get("nH") > 0)
                werr.append((float(np.sqrt(np.mean(np.log(t_new[inner] / t_warm[inner]) ** 2))),
                             float(np.sqrt(np.mean(np.log(t_new[inner] / t_prev[inner]) ** 2))),
                             neb.last_metrics.rate_evaluations))
            if check is not None:
                dT, dx = check()
                acc.append({"iteration": it, "leaves": int(idx.size), "max_dT_e_K": dT, "max_dx_HII": dx})
        res[mode] = dict(s=ms / 1e3, evals=evals, accepted=accepted, acc=acc, x=neb.get("x_HI"), T=neb.get("T_e"),
                         last_change=np.abs(neb.get("T_e") - prev_T), werr=werr)
        neb.close()
    mlp.close()

    def stats(d):
        return {"p50": float(np.percentile(d, 50)), "p99": float(np.percentile(d, 99)), "max": float(d.max())}

    def glob(r):
        x, T = r["x"], r["T"]
        return {"ionized_fraction": float(np.mean(1 - x)), "mean_T_e_ionized": float(np.mean(T[x < 0.5]))}
    ion = res["plain"]["x"] < 0.5
    worst = {m: {"max_dT_e_K": max(a["max_dT_e_K"] for a in r["acc"]), "max_dx_HII": max(a["max_dx_HII"] for a in r["acc"])}
             for m, r in res.items()}
    return {"config": f"hii_metals {n}^3, {nphot:.0e} packets, {iters} iterations from the configured ionized start, "
                      f"FP32 transport",
            "plain_s": res["plain"]["s"], "bracketed_s": res["bracketed"]["s"], "mlp_s": res["mlp"]["s"],
            "speedup_mlp_vs_plain": res["plain"]["s"] / res["mlp"]["s"],
            "speedup_bracketed_vs_plain": res["plain"]["s"] / res["bracketed"]["s"],
            "speedup_mlp_vs_bracketed": res["bracketed"]["s"] / res["mlp"]["s"],
            "net_rate_evaluations": {k: int(v["evals"]) for k, v in res.items()},
            "mlp_gate_accepted_leaves": int(res["mlp"]["accepted"]),
            "mlp_start_rms_ln": {"note": "per iteration: RMS over the solved leaves inside (te_min, te_max) of "
                                         "ln(T_e / start) for the MLP's start and for the previous T_e, and the "
                                         "update's net-rate evaluations",
                                 "mlp_start": [round(w[0], 5) for w in res["mlp"]["werr"]],
                                 "previous_T_e": [round(w[1], 5) for w in res["mlp"]["werr"]],
                                 "evaluations": [int(w[2]) for w in res["mlp"]["werr"]]},
            "solve_vs_fp64_oracle": {"bars": {"T_e_K": 20.0, "x_HII": 1e-3}, "worst": worst,
                                     "per_check": {k: v["acc"] for k, v in res.items()}},
            "final_state_between_arms": {
                "note": "the coupled iteration carries Monte Carlo noise: the diffuse packets relaunch from "
                        "different leaves as the state moves; compare with the plain arm's own last change",
                "plain_last_change_T_e_K_ionized": stats(res["plain"]["last_change"][ion]),
                "dT_e_K_ionized": {m: stats(np.abs(res[m]["T"] - res["plain"]["T"])[ion]) for m in ("bracketed", "mlp")},
                "global": {k: glob(v) for k, v in res.items()}},
            "training": {"pairs": int(len(X)), "data_s": t_data, "train_s": t_train, "epochs": 20,
                         "loss_first": float(losses[0]), "loss_last": float(losses[-1])}}


def run_extras(steps=2, warmup=3):
    """The other single-GPU configurations as extra keys of the headline
    line: the dusty clumpy nebula on the octree and the 64 batched H II
    regions, each this script in a child process (its own device memory),
    reduced to value, e2e, step time and roofline."""
    out = {}
    for name in ("clumpy_dusty", "batch64"):
        cmd = [sys.executable, os.path.abspath(__file__), "--workload", name, "--steps", str(steps), "--warmup",
               str(warmup), "--no-converge", "--no-cpu-baseline", "--no-extras"]
        try:
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=1500)
            d = json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][-1])
            out[name] = {k: d.get(k) for k in ("value", "unit", "ms_per_step", "steps", "warmup", "config",
                                               "implementation", "e2e", "clocks", "gpu_launches")}
            out[name]["roofline"] = {k: d["roofline"].get(k) for k in ("achieved", "peak", "frac", "kernel_ms")}
        except Exception as e:   # reported, not fatal: the headline stands on its own
            out[name] = {"error": f"{type(e).__name__}: {e}"[:300]}
    return out


def neb_order(neb):
    return {0: "launch", 1: "direction", 2: "coherent"}.get(int(neb.par.packet_order), "?")


def grid_name(wl, nleaf):
    if wl.name == "batch64":
        return f"{wl.count} instances, cubic grids 32^3..128^3, {nleaf or 'about 4.5e7'} leaves in all"
    return f"{wl.grid}^3" if wl.grid else f"octree, {nleaf or 'about 3e6'} leaves"


def launches_per_step(wl, diffuse_packets, coherent=True):
    """Kernels of this library per step: per chunk of up to 4 Mi stellar
    packets a launch and a walk (coherent order: also the key kernel; the
    sort is a library radix sort, not counted), the H/He rates (+ the metal
    rates), the balance; with the diffuse field the leaf luminosities and a
    launch and a walk per diffuse chunk (the prefix sum is a library scan, not
    counted)."""
    cap = 1 << 22
    n = (3 if coherent else 2) * -(-wl.nphot // cap) + 1 + 1
    if wl.name == "hii_metals128":
        n += 1 + 1 + 2 * -(-diffuse_packets // cap)
    return n


if __name__ == "__main__":
    sys.exit(main())
