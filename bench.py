"""Benchmark of the Hallen MoM hot path on B200.

Workload (one "step" = one pass of the hot path over one batch): the
frequency sweep of a 5-element parallel-wire array in free space -- five
z-parallel wires of 51 segments (N = 255, S = 260) with seeded lengths
U(0.9, 1.1) * lambda/2 and gaps U(0.15, 0.25) * lambda at 14.2 MHz, radius
1 mm, a 1 V source on the centre segment of element 2, 201 linear
frequencies 13.0-15.5 MHz, and the 91 x 361 (1 degree) RP gain grid per
frequency.  Each frequency is one solve (fill + normal equations + GEPP +
feedpoint + pattern with its power integral).

  value     solves/s, inputs resident in HBM, CUDA events on the library's
            stream, max over ranks (weak scaling: every rank solves its own
            201-frequency sweep)
  e2e       the same through the C ABI with host buffers: pinned H2D of the
            batch tables, the run, D2H of currents/feeds/pattern per step
  roofline  the dominant phase, FP64-pipe bound, against the FP64 peak this
            script measures on the same GPU
  cpu_baseline  the CPU oracle (C restatement of the reference CPU path),
            one solve per host thread, on a bounded sample of the sweep

--impl reference times that CPU implementation alone on the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "fnec-rust_b200"))
sys.path.insert(0, ROOT)

METRIC = "solves/s & p50/p99 latency, mixed vs FP64 GPU at |ΔZin|/|Zin|≤1e-6"
C0 = 299792458.0


def sweep_workload(seed: int = 11):
    """5-wire array (lengths/gaps seeded), 201 frequencies, RP 91 x 361."""
    rng = np.random.default_rng(seed)
    f0 = 14.2e6
    lam = C0 / f0
    x = 0.0
    wires = []
    for t in range(5):
        L = rng.uniform(0.9, 1.1) * lam / 2
        wires.append((t + 1, 51, (x, 0.0, -L / 2), (x, 0.0, L / 2), 1e-3))
        x += rng.uniform(0.15, 0.25) * lam
    sources = [(2, 26, 1.0)]
    freqs = [13.0e6 + i * (15.5e6 - 13.0e6) / 200 for i in range(201)]
    rp = (91, 361, 0.0, 0.0, 1.0, 1.0)
    return wires, sources, freqs, rp


def algorithmic_flops(n: int, s: int, n_int: int, n_req: int, runs: int):
    """Per-unit algorithmic work of each phase (real flops; a complex
    multiply-add is 8: 4 multiplies + 4 adds)."""
    return {
        "gram": 8.0 * n * n * (n + 1),          # Z^H [Z | y]
        "factor": 8.0 * (s ** 3) / 3.0,         # GEPP trailing updates
        "farfield": 8.0 * (n_int + n_req) * n,  # Horner: 1 complex MAC / (direction, segment)
    }


def clock_sampler(device: int):
    q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    try:
        return subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "200",
                                 "-i", str(device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
    except OSError:
        return None


def clock_summary(proc):
    if proc is None:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
    proc.terminate()
    try:
        out, _ = proc.communicate(timeout=10)
    except subprocess.TimeoutExpired:
        proc.kill()
        out, _ = proc.communicate()
    rows = [r.split(",") for r in out.strip().splitlines() if r.count(",") >= 6]
    if not rows:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
    sm = [float(r[0]) for r in rows]
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    reasons = sorted({names[i] for r in rows for i in range(4) if "Active" in r[3 + i] and "Not" not in r[3 + i]})
    return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(rows[0][1]), "reasons": reasons,
            "samples": len(rows), "power_w_max": max(float(r[2]) for r in rows if r[2].strip()
                                                     .replace(".", "", 1).isdigit())}


def cpu_oracle_rate(wires, sources, freqs, rp, n_units: int, threads: int):
    """Solve n_units of the sweep with the CPU oracle on `threads` threads."""
    from oracle import oracle as O

    ow = O.wires_array(wires)
    osrc = O.sources_array(sources)
    pts = O.rp_card_points(*rp)
    idx = np.linspace(0, len(freqs) - 1, n_units).round().astype(int)
    probs = [O.Problem(ow, osrc, freqs[i], points=pts) for i in idx]
    t0 = time.perf_counter()
    O.solve_problems(probs, threads)
    dt = time.perf_counter() - t0
    assert all(p.status == 0 for p in probs)
    return n_units / dt, dt, probs, idx


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    wires, sources, freqs, rp = sweep_workload()
    threads = os.cpu_count() or 1
    n = max(threads, 1)
    for _ in range(args.warmup):
        cpu_oracle_rate(wires, sources, freqs, rp, min(n, 8), threads)
    times = []
    for _ in range(args.steps):
        r, dt, _, _ = cpu_oracle_rate(wires, sources, freqs, rp, n, threads)
        times.append(dt)
    rate = n * len(times) / sum(times)
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": "solves/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(times)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded 5-element array, seed 11)",
        "config": {"workload": "sweep5: 5-wire parallel array, N=255 (S=260), 201 freqs 13.0-15.5 MHz, "
                               "RP 91x361 per freq", "sample_units_per_step": n},
        "cpu_baseline": {"value": rate, "unit": "solves/s", "cores": threads, "kind": "port",
                         "sample": f"{n} of the 201 sweep frequencies per step (evenly spaced), one solve per "
                                   f"thread, CPU oracle (C restatement of the reference CPU path, -O2 "
                                   f"-ffp-contract=off); the Rust reference itself cannot be built here"},
        "e2e": {"value": rate, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    torch.cuda.set_device(local)
    import nec_accel as acc

    ctx = acc.Context(local)
    wires, sources, freqs, rp = sweep_workload()
    prec = acc.PRECISION_MIXED if args.precision == "mixed" else acc.PRECISION_FP64
    ant = acc.Antenna(acc.wires_array(wires), acc.sources_array(sources), freqs, acc.GROUND_FREE, rp)
    batch = acc.HallenBatch([ant], precision=prec, ctx=ctx)
    units = len(freqs)
    stream = torch.cuda.ExternalStream(acc.lib().fnec_ctx_stream(ctx.handle), device=local)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(local)

    # ---- device-resident timing ------------------------------------------
    for _ in range(args.warmup):
        batch.run()
    batch.sync()
    sampler = clock_sampler(local) if rank == 0 else None
    barrier()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    evs[0].record(stream)
    for k in range(args.steps):
        batch.run()
        evs[k + 1].record(stream)
    batch.sync()
    barrier()
    step_ms = np.array([evs[k].elapsed_time(evs[k + 1]) for k in range(args.steps)])
    total_ms = float(step_ms.sum())
    clocks = clock_summary(sampler) if rank == 0 else None
    launches = batch.kernel_launches * args.steps

    # ---- end to end through the C ABI, host buffers ----------------------
    batch.read_raw()
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        batch.upload()
        batch.run()
        batch.read_raw()  # synchronises: device -> pinned -> host arrays
    e1.record(stream)
    batch.sync()
    barrier()
    e2e_ms = e0.elapsed_time(e1)
    h2d = batch.h2d_bytes
    d2h = batch.d2h_bytes()

    # ---- per-phase times (profiled runs, after the timed regions) --------
    batch.set_profiling(True)
    phase = {k: 0.0 for k in batch.PHASES}
    reps = 3
    for _ in range(reps):
        batch.run()
        for k, v in batch.phase_ms().items():
            phase[k] += v / reps
    batch.set_profiling(False)

    # ---- max over ranks ---------------------------------------------------
    vals = torch.tensor([total_ms, e2e_ms], dtype=torch.float64, device=f"cuda:{local}")
    if dist is not None:
        dist.all_reduce(vals, op=dist.ReduceOp.MAX)
    total_ms, e2e_ms = vals.tolist()

    # ---- parity spot check of this run against the oracle -----------------
    res = batch.read()
    if rank == 0:
        fma_tf, muladd_tf = acc.measure_fp64_peak(local)
        n = 255
        s = 260
        flops = algorithmic_flops(n, s, 181 * 360, 91 * 361, 5)
        dom = max(("fill", "gram", "factor", "farfield"), key=lambda k: phase[k])
        dom_ms = phase[dom]
        if dom in flops:
            achieved = flops[dom] * units / (dom_ms * 1e-3) / 1e12
            peak = muladd_tf if dom in ("gram", "factor") else fma_tf
            roof = {"kernel": dom, "bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                    "frac": achieved / peak, "traffic": None,
                    "peak_source": "measured in this run by fnec_measure_fp64_peak ("
                                   + ("DMUL+DADD, the exact path issues no FMA" if peak == muladd_tf else "DFMA")
                                   + "); MEASURED_PEAKS.json holds no FP64 figure"}
        else:
            roof = {"kernel": dom, "bound": "fp64", "achieved": None, "peak": fma_tf, "unit": "TFLOP/s",
                    "frac": None, "traffic": None,
                    "note": "fill throughput is reported as G samples/s in phase_detail"}
        samples = units * (n * n * 8 - 4 * n)  # off-diagonal 8-point + self 4-point G samples
        line = {
            "metric": METRIC,
            "value": args.gpus * units * args.steps / (total_ms * 1e-3),
            "unit": "solves/s",
            "n_gpus": args.gpus,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64" if prec == acc.PRECISION_FP64 else "f32+f64",
            "data": "synthetic (seeded 5-element array, seed 11)",
            "config": {"workload": "sweep5: 5-wire parallel array, N=255 (S=260), 201 freqs 13.0-15.5 MHz, "
                                   "RP 91x361 per freq", "precision": args.precision, "units_per_step": units,
                       "l2": f"working set {batch.info.device_bytes / 1e9:.2f} GB per step > 126 MB L2 "
                             f"(no flush needed)", "parallelism": f"replicas x{args.gpus} (no collective)"},
            "latency_ms": {"p50": float(np.percentile(step_ms, 50)), "p99": float(np.percentile(step_ms, 99)),
                           "what": "batch (201-solve step) latency"},
            "e2e": {"value": args.gpus * units * args.steps / (e2e_ms * 1e-3), "unit": "solves/s",
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": int(launches),
            "roofline": roof,
            "phase_ms": {k: round(v, 4) for k, v in phase.items()},
            "phase_detail": {"fill_gsamples_per_s": samples / (phase["fill"] * 1e-3) / 1e9 if phase["fill"] else None,
                             "fp64_peak_tflops": {"dfma": fma_tf, "dmul_dadd": muladd_tf}},
            "clocks": clocks,
        }
        # CPU baseline (oracle, bounded sample) + parity of the sampled units
        if not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            n_units = min(units, max(threads, 4))
            rate, dt, probs, idx = cpu_oracle_rate(wires, sources, freqs, rp, n_units, threads)
            line["cpu_baseline"] = {"value": rate, "unit": "solves/s", "cores": threads, "kind": "port",
                                    "sample": f"{n_units} evenly spaced sweep frequencies, one per thread, "
                                              f"{dt:.1f} s wall"}
            dz = []
            for p, i in zip(probs, idx):
                zg = complex(res.feeds[i][0, 5], res.feeds[i][0, 6])
                dz.append(abs(zg - p.zin[0]) / abs(p.zin[0]))
            line["parity"] = {"units_checked": n_units, "max_rel_dzin_vs_oracle": float(max(dz))}
        print(json.dumps(line), flush=True)
    batch.close()
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
