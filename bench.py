#!/usr/bin/env python
"""Benchmark of the SPH-VE hydro step on B200: particle-steps/s of the whole step (domain sync, neighbour search,
VE chain, integration) on a Sedov blast of 128^3 = 2,097,152 particles.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--side S]

Prints one JSON line (rank 0). For N > 1 (torchrun) every rank runs an independent replica of the workload (the
path does not shard at one GPU), times are max-reduced over ranks and `value` is the whole-job
throughput. `--impl reference` times the reference's own OpenMP CPU implementation (oracle/_ref, compiled from the
reference sources) on this host's cores instead.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s per B200, mixed vs FP64 plain at stated err; adjoint/fwd time"
UNIT = "particle-steps/s"
#: algorithmic FP operations per neighbour pair of each J-loop (add/mul = 1, FMA = 2, table lookup = 6)
FLOPS_PER_PAIR = {"xmass": 18, "ve_def_gradh_eos": 31, "iad_divv_curlv": 88, "av_switches": 55,
                  "momentum_energy": 140}
KERNEL_STAGES = ("sync", "neighbors", "xmass", "ve_def_gradh_eos", "iad_divv_curlv", "av_switches",
                 "momentum_energy")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--side", type=int, default=128)
    ap.add_argument("--precision", choices=("mixed", "fp64"), default="mixed")
    ap.add_argument("--no-fp64-leg", action="store_true", help="skip the plain FP64 comparison leg")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def dist_info():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def workload_config(side, n, precision):
    return {"workload": f"sedov-{side}^3 VE hydro step ({n:,} particles, periodic box, ng0=100, ngmax=150)",
            "side": side, "n_particles": n, "precision": precision,
            "step": "sync(keys+sort+trees+gather) + neighbours(h-iter) + XMass + VeDefGradh/EOS + IAD/divv/curlv"
                    " + AVswitches + MomentumEnergy + conserved + integrate + h update",
            "l2": "no flush: per-step working set > 0.5 GB, larger than the 126 MB L2"}


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def run_ours(args, ws, rank, local):
    import numpy as np
    import torch

    from sphexa_b200 import ic as icm
    from sphexa_b200 import lib as L
    from sphexa_b200.ic import CONSERVED_FIELDS
    from sphexa_b200.simulation import Simulation

    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier_sync():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v: float) -> float:
        if dist is None:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    ic = icm.sedov(args.side, seed=rank)  # each replica its own seed
    n = ic["x"].size

    def timed_leg(precision: str, steps: int, warmup: int, with_e2e: bool, with_clocks: bool):
        sim = Simulation(ic, precision)
        stream = torch.cuda.ExternalStream(sim.lib.sphb_sim_stream(sim.h))
        for _ in range(warmup):
            sim.step()
        stage_sum = {k: 0.0 for k in sim.stage_times()}
        clocks = ClockSampler(local)
        barrier_sync()
        if with_clocks:
            clocks.start()
        launches0 = sim.kernel_launches()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            sim.step()
            for k, v in sim.stage_times().items():
                stage_sum[k] += v
        e1.record(stream)
        barrier_sync()
        clk = clocks.stop() if with_clocks else None
        launches = sim.kernel_launches() - launches0
        ms = e0.elapsed_time(e1)
        ms = max_over_ranks(ms)
        nc = sim.get("nc").astype(np.int64)
        pairs = int(np.minimum(nc - 1, int(ic["params"]["ngmax"])).sum())
        res = {"ms_total": ms, "stage_ms": {k: v / steps for k, v in stage_sum.items()}, "launches": launches,
               "pairs": pairs, "clocks": clk, "sim": sim}
        if with_e2e:
            # per step: host->device copy of the whole particle state from pinned memory, the step, and the
            # device->host copy of the updated state (the C-ABI round trip of a caller holding host buffers)
            host = [torch.empty(n, dtype=torch.float64, pin_memory=True) for _ in CONSERVED_FIELDS]
            hid = torch.empty(n, dtype=torch.int64, pin_memory=True)
            tbl_out = (C.c_void_p * len(host))(*[h.data_ptr() for h in host])
            L.check(sim.lib.sphb_sim_store_state(sim.h, tbl_out, C.c_void_p(hid.data_ptr()), 0), "store_state")
            tbl_in = (C.c_void_p * len(host))(*[h.data_ptr() for h in host])
            barrier_sync()
            e0.record(stream)
            for _ in range(steps):
                L.check(sim.lib.sphb_sim_load_state(sim.h, tbl_in, C.c_void_p(hid.data_ptr()), 0), "load_state")
                sim.step()
                L.check(sim.lib.sphb_sim_store_state(sim.h, tbl_out, C.c_void_p(hid.data_ptr()), 0),
                        "store_state")
            e1.record(stream)
            barrier_sync()
            res["e2e_ms"] = max_over_ranks(e0.elapsed_time(e1))
            res["h2d_bytes"] = (len(host) * 8 + 8) * n
            res["d2h_bytes"] = (len(host) * 8 + 8) * n
        return res

    main = timed_leg(args.precision, args.steps, args.warmup, with_e2e=True, with_clocks=True)
    fp64 = None
    if args.precision == "mixed" and not args.no_fp64_leg:
        fp64 = timed_leg("fp64", max(2, args.steps // 2), max(1, args.warmup), with_e2e=False, with_clocks=False)

    # roofline of the dominant kernel (stage times are CUDA events around each launch on the sim stream)
    stages = main["stage_ms"]
    dominant = max(KERNEL_STAGES, key=lambda k: stages.get(k, 0.0))
    which = 0 if args.precision == "mixed" else 1
    peak = C.c_double()
    L.check(L.load().sphb_probe_fma_peak(which, C.byref(peak)), "probe")
    roofline = None
    if dominant in FLOPS_PER_PAIR:
        flops = FLOPS_PER_PAIR[dominant] * main["pairs"]
        achieved = flops / (stages[dominant] * 1e-3) / 1e12
        roofline = {"bound": "fp32" if which == 0 else "fp64", "kernel": dominant, "achieved": achieved,
                    "peak": peak.value, "unit": "TFLOP/s", "frac": achieved / peak.value, "traffic": None,
                    "peak_source": "measured on this GPU by sphb_probe_fma_peak (register FMA loop, all SMs)",
                    "flops_per_launch": flops}
    else:
        roofline = {"bound": "latency", "kernel": dominant, "achieved": None, "peak": peak.value,
                    "unit": "TFLOP/s", "frac": None, "traffic": None}

    steps = args.steps
    value = n * ws * steps / (main["ms_total"] * 1e-3)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": steps, "warmup": args.warmup,
        "ms_per_step": main["ms_total"] / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if args.precision == "mixed" else "f64", "data": "synthetic",
        "precision": ("mixed: FP32 Kahan-compensated neighbour sums on FP64 relative coordinates; FP64 positions, "
                      "keys, integration, h update and reductions") if args.precision == "mixed" else "fp64",
        "config": workload_config(args.side, n, args.precision),
        "e2e": {"value": n * ws * steps / (main["e2e_ms"] * 1e-3), "unit": UNIT,
                "h2d_bytes_per_step": main["h2d_bytes"], "d2h_bytes_per_step": main["d2h_bytes"]},
        "gpu_launches": main["launches"],
        "stage_ms": {k: round(v, 4) for k, v in stages.items()},
        "neighbor_pairs_per_step": main["pairs"],
        "roofline": roofline,
        "clocks": main["clocks"],
    }
    if fp64 is not None:
        fsteps = max(2, args.steps // 2)
        v64 = n * ws * fsteps / (fp64["ms_total"] * 1e-3)
        line["fp64_plain"] = {"value": v64, "unit": UNIT, "ms_per_step": fp64["ms_total"] / fsteps,
                              "stage_ms": {k: round(v, 4) for k, v in fp64["stage_ms"].items()},
                              "mixed_over_fp64": value / v64}
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(ic, n)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_baseline(ic, n, steps=2, warmup=1, mixed=True):
    """Reference OpenMP CPU step (oracle/_ref, reference default types unless mixed=False) on this host."""
    os.environ.setdefault("OMP_NUM_THREADS", str(host_threads()))
    from oracle import refsim
    if not refsim.available(mixed):
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": "oracle/_ref not built"}
    r = refsim.RefSim(ic, mixed=mixed)
    for _ in range(warmup):
        r.step()
    t0 = time.perf_counter()
    for _ in range(steps):
        r.step()
    dt = time.perf_counter() - t0
    return {"value": n * steps / dt, "unit": UNIT, "cores": int(os.environ["OMP_NUM_THREADS"]),
            "kind": "reference",
            "sample": f"{steps} steps after {warmup} warm-up of the same Sedov workload ({n:,} particles), reference "
                      f"CPU code with its default types (f64 coordinates, f32 hydro fields), wall clock"}


def run_reference(args, ws, rank):
    if rank != 0:
        return
    os.environ.setdefault("OMP_NUM_THREADS", str(host_threads()))
    from sphexa_b200 import ic as icm
    ic = icm.sedov(args.side)
    n = ic["x"].size
    steps = min(args.steps, 3)
    warmup = min(args.warmup, 1)
    base = cpu_baseline(ic, n, steps=steps, warmup=warmup)
    v = base["value"]
    line = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": ws, "steps": steps,
            "warmup": warmup, "ms_per_step": (n / v * 1e3) if v else None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(args.side, n, "reference default types (f64 coordinates, f32 hydro)"),
            "cpu_baseline": base, "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0,
                                          "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    ws, rank, local = dist_info()
    if args.impl == "reference":
        run_reference(args, ws, rank)
        return
    run_ours(args, ws, rank, local)


if __name__ == "__main__":
    main()
