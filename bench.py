"""Benchmark of the Hallen MoM hot path on B200.

Headline workload (one "step" = one pass of the hot path over one batch):
the uneven batch of 4096 random wire antennas -- 1-8 straight wires each
(count uniform), endpoints uniform in a 20 m cube, 11-101 segments per wire
(odd, uniform), radius log-uniform 0.5-5 mm, one 1 V source on the centre
segment of wire 1, one frequency log-uniform 3-30 MHz, free space or GN 1
with probability 1/2 -- filled, normal-equation formed, factored and solved
in one captured pipeline, in both forms: the mixed form (3xTF32 Gram, FP32
factor, FP64 GMRES refinement) and the plain FP64 form.

  value     solves/s of the chosen (mixed) form, inputs resident in HBM,
            CUDA events on the library's stream, max over ranks.  With N
            GPUs the job is N x 4096 antennas split across the ranks by the
            work model (nec_accel.shard), no collective on the data path
            (weak scaling); the feedpoint rows are gathered on rank 0 after
            the timed region.
  e2e       the same through the C ABI with host buffers: pinned H2D of the
            batch tables, the run, D2H of what the report prints per step
            (currents, feeds, status); e2e_with_planning also plans a new
            batch (topology, junctions, packing, device allocation) every
            step, as a call that brings new geometries must
  roofline  the dominant phase of the chosen form against the measured peak
            of the pipe that bounds it
  cpu_baseline  the CPU oracle (C restatement of the reference CPU path),
            one solve per host thread, on a bounded sample of the units;
            the same sample checks both forms' Zin and currents

The 5-wire frequency sweep (201 frequencies, 91 x 361 pattern each) is
measured after the headline and reported under the key "sweep5".
--workload selects another workload as the headline (sweep5, mesh, serve,
receive).  --impl reference times the CPU implementation alone.
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


def sweep_workload(seed: int = 11, n_freqs: int = 201):
    """5-wire array (lengths/gaps seeded), 201 frequencies, RP 91 x 361
    (n_freqs < 201 keeps an evenly spaced subset: small profiling cases)."""
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
    if n_freqs < 201:
        freqs = [freqs[i] for i in np.linspace(0, 200, n_freqs).round().astype(int)]
    rp = (91, 361, 0.0, 0.0, 1.0, 1.0)
    return wires, sources, freqs, rp


def receive_workload(n_theta: int = 37, n_phi: int = 72):
    """The 5-element array of the sweep as a receiving antenna: an EX 2 card
    (right elliptic, axial ratio 0.5, eta 20 degrees) whose n_theta x n_phi
    incidence directions in 5 degree steps are the receive sweep, at 13.0,
    14.2 and 15.5 MHz; no RP card."""
    wires, _, _, _ = sweep_workload()
    freqs = [13.0e6, 14.2e6, 15.5e6]
    card = (2, n_theta, n_phi, 0.0, 0.0, 20.0, 5.0, 5.0, 0.5)
    return wires, freqs, card


def receive_units(wires, freqs, card):
    """The receive sweep as (wires, sources, ground, freq, rp, wave) units:
    one per (frequency, direction), theta outer, phi inner."""
    t, nth, nph, th0, ph0, eta, dth, dph, ar = card
    out = []
    for f in freqs:
        for it in range(nth):
            for ip in range(nph):
                out.append((wires, [], 0, f, None, (t, th0 + it * dth, ph0 + ip * dph, eta, ar)))
    return out


def _seg_closest(p1, q1, p2, q2):
    """Closest distance and parameters between segments p1-q1 and p2-q2."""
    d1, d2, r = q1 - p1, q2 - p2, p1 - p2
    a, e, f = d1 @ d1, d2 @ d2, d2 @ r
    c, b = d1 @ r, d1 @ d2
    den = a * e - b * b
    sp = np.clip((b * f - c * e) / den, 0.0, 1.0) if den > 1e-300 else 0.0
    tp = (b * sp + f) / e
    if tp < 0.0:
        tp, sp = 0.0, np.clip(-c / a, 0.0, 1.0)
    elif tp > 1.0:
        tp, sp = 1.0, np.clip((b - c) / a, 0.0, 1.0)
    return float(np.linalg.norm((p1 + d1 * sp) - (p2 + d2 * tp))), sp, tp


def uneven_workload(n_ant: int = 4096, seed: int = 7):
    """Uneven batch: antennas of 1-8 straight wires (count uniform) with
    endpoints uniform in a 20 m cube (z in (0, 20]), 11-101 segments per wire
    (odd, uniform), radius log-uniform 0.5-5 mm, one 1 V source on the centre
    segment of wire 1, one frequency log-uniform 3-30 MHz, free space or GN 1
    with probability 1/2.  Geometries the CLI guards reject are resampled:
    crossing wire interiors (apps/nec-cli/src/geometry_validation.rs:14-45),
    a source segment shorter than 2 radii (:47-80), a wire touching the
    ground plane (:83-117)."""
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < n_ant:
        nw = int(rng.integers(1, 9))
        wires = []
        for t in range(nw):
            p0 = rng.uniform([-10.0, -10.0, 0.0], [10.0, 10.0, 20.0])
            p1 = rng.uniform([-10.0, -10.0, 0.0], [10.0, 10.0, 20.0])
            nseg = 2 * int(rng.integers(5, 51)) + 1
            rad = float(np.exp(rng.uniform(np.log(0.5e-3), np.log(5e-3))))
            wires.append((t + 1, nseg, tuple(p0), tuple(p1), rad))
        ground = int(rng.integers(0, 2))
        f = float(np.exp(rng.uniform(np.log(3e6), np.log(30e6))))
        ok = all(min(w[2][2], w[3][2]) > 1e-9 for w in wires)
        L1 = np.linalg.norm(np.subtract(wires[0][3], wires[0][2])) / wires[0][1]
        ok = ok and L1 / wires[0][4] >= 2.0
        for i in range(nw):
            for j in range(i + 1, nw):
                dist, sp, tp = _seg_closest(np.array(wires[i][2]), np.array(wires[i][3]),
                                            np.array(wires[j][2]), np.array(wires[j][3]))
                if dist <= 1e-7 and 1e-6 < sp < 1 - 1e-6 and 1e-6 < tp < 1 - 1e-6:
                    ok = False
        if not ok:
            continue
        out.append((wires, [(1, (wires[0][1] + 1) // 2, 1.0)], ground, f))
    return out


def uneven_desc(n):
    return (f"uneven: {n} random antennas of 1-8 wires, 11-101 segments per wire (N 11-808), "
            f"one frequency each (3-30 MHz), free space / GN 1, no pattern")


SERVE_RP = (91, 361, 0.0, 0.0, 1.0, 1.0)  # theta 0-90 x phi 0-360, 1 degree steps


def serve_requests(n_req: int, seed: int = 13, n_cap: int = 4096, sigma: float = 0.75):
    """Served request stream: each request is a random wire antenna like the
    uneven batch's (1-8 straight wires, endpoints in a 20 m cube, radius
    log-uniform 0.5-5 mm, one frequency log-uniform 3-30 MHz, free space or
    GN 1 with probability 1/2) whose total segment count N is drawn
    lognormal with median 150 (sigma 0.75, capped at n_cap) and split over
    the wires in odd counts of at least 3.  It carries 1-4 source positions
    (uniform): the centre segment of wire 1 and distinct random segments,
    each a separate right-hand side; half of the requests ask for the
    91 x 361 pattern.  The CLI guards of the uneven generator apply."""
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < n_req:
        n_tot = int(min(n_cap, max(11, round(float(np.exp(rng.normal(np.log(150.0), sigma)))))))
        nw = int(rng.integers(1, 9))
        nw = max(1, min(nw, n_tot // 3))
        share = rng.dirichlet(np.ones(nw))
        counts = [max(3, int(round(n_tot * f))) for f in share]
        counts = [c if c % 2 else c + 1 for c in counts]
        wires = []
        for t in range(nw):
            p0 = rng.uniform([-10.0, -10.0, 0.0], [10.0, 10.0, 20.0])
            p1 = rng.uniform([-10.0, -10.0, 0.0], [10.0, 10.0, 20.0])
            rad = float(np.exp(rng.uniform(np.log(0.5e-3), np.log(5e-3))))
            wires.append((t + 1, counts[t], tuple(p0), tuple(p1), rad))
        ground = int(rng.integers(0, 2))
        f = float(np.exp(rng.uniform(np.log(3e6), np.log(30e6))))
        n_src = int(rng.integers(1, 5))
        srcs = [(1, (wires[0][1] + 1) // 2)]
        while len(srcs) < n_src:
            t = int(rng.integers(0, nw))
            cand = (t + 1, int(rng.integers(1, wires[t][1] + 1)))
            if cand not in srcs:
                srcs.append(cand)
        ok = all(min(w[2][2], w[3][2]) > 1e-9 for w in wires)
        for tag, seg in srcs:
            w = wires[tag - 1]
            ok = ok and np.linalg.norm(np.subtract(w[3], w[2])) / w[1] / w[4] >= 2.0
        for i in range(nw):
            for j in range(i + 1, nw):
                dist, sp, tp = _seg_closest(np.array(wires[i][2]), np.array(wires[i][3]),
                                            np.array(wires[j][2]), np.array(wires[j][3]))
                if dist <= 1e-7 and 1e-6 < sp < 1 - 1e-6 and 1e-6 < tp < 1 - 1e-6:
                    ok = False
        if not ok:
            continue
        rp = SERVE_RP if rng.random() < 0.5 else None
        out.append((wires, [(tag, seg, 1.0) for tag, seg in srcs], ground, f, rp))
    return out


def mesh_workload(cells: int = 46, seed: int = 5, f0: float = 14.2e6):
    """Junctioned wire mesh over PEC ground: a square grid of cells x cells
    cells with edge 0.05 lambda in the plane z = 0.25 lambda, node positions
    jittered by a seeded +-1 % of the pitch, every cell edge a 2-segment wire
    of radius 1 mm (row edges first, then column edges, in tag order), and a
    1 V source on the first segment of the row edge nearest the grid centre.
    Every interior node joins four wire ends, so junction rows are pairwise
    (C(4,2) = 6 per interior node, geometry.rs:274-339)."""
    lam = C0 / f0
    pitch = 0.05 * lam
    rng = np.random.default_rng(seed)
    nn = cells + 1
    jit = rng.uniform(-0.01, 0.01, size=(nn, nn, 2)) * pitch
    node = np.zeros((nn, nn, 3))
    for i in range(nn):
        for j in range(nn):
            node[i, j] = (i * pitch + jit[i, j, 0], j * pitch + jit[i, j, 1], 0.25 * lam)
    wires = []
    tag = 1
    centre = None
    for j in range(nn):          # row edges: along x
        for i in range(cells):
            wires.append((tag, 2, tuple(node[i, j]), tuple(node[i + 1, j]), 1e-3))
            if j == nn // 2 and i == cells // 2:
                centre = tag
            tag += 1
    for i in range(nn):          # column edges: along y
        for j in range(cells):
            wires.append((tag, 2, tuple(node[i, j]), tuple(node[i, j + 1]), 1e-3))
            tag += 1
    return wires, [(centre, 1, 1.0)], f0


def algorithmic_flops(n, s, n_dir):
    """Algorithmic work of each phase summed over units (real flops; a
    complex multiply-add is 8: 4 multiplies + 4 adds).  n, s, n_dir are
    per-unit arrays: segments, unknowns, far-field directions (integration
    grid + requested points, 0 without a pattern)."""
    n = np.asarray(n, np.float64)
    s = np.asarray(s, np.float64)
    n_dir = np.asarray(n_dir, np.float64)
    return {
        "gram": float(np.sum(8.0 * n * n * (n + 1))),  # Z^H [Z | y]
        "factor": float(np.sum(8.0 * s ** 3 / 3.0)),  # GEPP trailing updates
        "farfield": float(np.sum(8.0 * n_dir * n)),   # Horner: 1 complex MAC / (direction, segment)
        "fill_samples": float(np.sum(n * n * 8 - 4 * n)),
    }


FILL_FLOPS_PER_SAMPLE = 60.0  # one G(R) sample: sqrt + sincos + 2 divisions + ~26 add/mul, in FP64 ops
SINCOS_FLOPS = 40.0           # one FP64 sincos, in FP64 ops


def measured_peaks():
    """HBM copy bandwidth and dense BF16 tensor throughput measured on this
    pool's B200s (MEASURED_PEAKS.json beside this file); TF32 tensor
    throughput is half the BF16 rate."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            m = json.load(fh)
        hbm = float(m.get("hbm_gbs"))
        bf16 = float(m.get("bf16_tflops"))
        src = "MEASURED_PEAKS.json"
    except Exception:
        hbm, bf16, src = 6650.0, 1590.0, "fallback (no MEASURED_PEAKS.json)"
    return {"hbm_gbs": hbm, "bf16_tflops": bf16, "tf32_tflops": bf16 / 2.0, "source": src}


def ff_directions(ground, rp):
    """Far-field directions evaluated per solve: the power-integration grid
    plus the requested points that do not coincide with one of its
    directions (theta 0, the last theta row, phi >= 360 are evaluated on
    their own)."""
    n_th, th_max = (91, 90.0) if ground == 1 else (181, 180.0)
    n_int = n_th * 360
    if rp is None:
        return n_int
    nt, nph, t0, p0, dt, dp = rp
    th = t0 + np.arange(nt) * dt
    ph = p0 + np.arange(nph) * dp
    step = th_max / (n_th - 1)
    on_t = (np.abs(th / step - np.round(th / step)) < 1e-12) & (th >= step) & (th <= th_max - step)
    if ground == 1:
        on_t &= th <= 90.0
    on_p = (np.abs(ph - np.round(ph)) < 1e-12) & (ph >= 0) & (ph < 360)
    below = (th > 90.0).sum() * nph if ground == 1 else 0
    return n_int + nt * nph - int(on_t.sum()) * int(on_p.sum()) - int(below)


def dram_traffic(phase, form, units, workload=None):
    """DRAM bytes of one run of a phase, scaled by units from the per-unit
    figure of an ncu capture committed under profiles/ (None if none): the
    capture of a smaller case of the same workload when there is one, else
    of the sweep workload."""
    key = {("solve", "mixed"): "solve_mixed", ("farfield", "mixed"): "farfield", ("farfield", "fp64"): "farfield",
           ("fill", "fp64"): "fill_fp64", ("fill", "mixed"): "fill_mixed"}.get((phase, form))
    try:
        with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "profiles", "traffic.json")) as fh:
            t = json.load(fh)
        e = t.get(f"{key}_{workload}") or t[key]
        return float(e["bytes_per_unit"]) * units, "profiles/" + e["capture"]
    except Exception:
        return None, None


def phase_rooflines(form, o, n, s, g, d, shapes, fma, muladd, ffma, peaks, runs):
    """Achieved rate and fraction of the measured peak of every phase.
    Work models (per unit): fill 60 FP64 ops per G(R) sample (8 N^2 - 4 N
    samples, doubled over GN 1); Gram 8 N^2 (N+1) flops (plain) or the
    3xTF32 tensor-core flops issued on the upper-triangle 128x128 tiles
    (mixed); factor (8/3) S^3 flops (GEPP) or (4/3) S^3 (the mixed form's
    Hermitian factor, lower triangle only); solve: plain back substitution 8 S^2
    flops on a serial chain, mixed GMRES HBM bytes: 16 N^2 per iteration
    (FP64 Z streamed once per apply of M^H M; one pass more for M^H y where
    the Gram phase does not form it) and (iterations + 1) x (8 S^2 + 512 S)
    (the FP32 factor and its diagonal blocks' inverses once per
    preconditioner apply); far
    field 8 N flops per direction (its sincos per wire run is not counted);
    antennas of z-parallel wires: 8 flops per (block row, segment) plus 8
    per (direction, run), the per-row path of the kernel."""
    ph = o["phase"]
    exact = form == "fp64"
    samples = float(np.sum((8 * n * n - 4 * n) * (1 + g)))
    res = {}

    def put(k, achieved, peak, unit, bound, src):
        ms = ph.get(k, 0.0)
        if not ms:
            res[k] = {"bound": bound, "achieved": None, "peak": peak, "unit": unit, "frac": None, "peak_source": src}
            return
        a = achieved / (ms * 1e-3)
        res[k] = {"bound": bound, "achieved": a, "peak": peak, "unit": unit, "frac": a / peak, "peak_source": src}

    p64 = (muladd, "DMUL+DADD measured by fnec_measure_fp64_peak (the exact path issues no FMA)") if exact else \
          (fma, "DFMA measured by fnec_measure_fp64_peak")
    put("fill", samples * FILL_FLOPS_PER_SAMPLE / 1e12, p64[0], "TFLOP/s", "fp64", p64[1])
    if exact:
        put("gram", float(np.sum(8 * n * n * (n + 1))) / 1e12, muladd, "TFLOP/s", "fp64", p64[1])
        put("factor", float(np.sum(8 * s ** 3 / 3)) / 1e12, muladd, "TFLOP/s", "fp64", p64[1])
        put("solve", float(np.sum(8 * s * s)) / 1e12, muladd, "TFLOP/s", "latency (serial chain)", p64[1])
    else:
        kb = np.ceil(n / 32)
        nt = np.ceil(2 * n / 128)
        tc = float(np.sum(nt * (nt + 1) / 2 * 128 * 128 * kb * 32 * 2 * 3))
        put("gram", tc / 1e12, peaks["tf32_tflops"], "TFLOP/s", "tensor (tf32)",
            "half the BF16 rate of " + peaks["source"])
        # the Hermitian factor (schedule factor_pivoting 0) updates only the
        # lower triangle: half of GEPP's (8/3) S^3
        sched = (o.get("schedule") or {}).get("schedule") or {}
        herm = int(sched.get("factor_pivoting", 0)) == 0
        put("factor", float(np.sum((4 if herm else 8) * s ** 3 / 3)) / 1e12, ffma, "TFLOP/s", "fp32",
            "FFMA measured by fnec_measure_fp32_peak")
        it = o.get("gmres_iters")
        n_s = np.array([u["n"] for u in shapes], np.float64)
        s_s = np.array([u["s"] for u in shapes], np.float64)
        its = it if it is not None and len(it) == len(n_s) else np.full(len(n_s), 5.0)
        # per iteration: Z once (16 N^2) for M^H M, the FP32 factor (8 S^2:
        # L below and U above the diagonal blocks) and the diagonal blocks'
        # FP32 inverses (two 32 x 32 complex64 blocks per 32 rows: 512 B per
        # row); plus the first preconditioner application, and one more Z
        # pass for M^H y unless the Gram phase formed it (systems of at most
        # 8 homogeneous columns and 4 right-hand sides)
        zpass = its + np.where(s_s - n_s <= 8, 0.0, 1.0)
        byt = float(np.sum(zpass * 16 * n_s * n_s + (its + 1) * (8 * s_s * s_s + 512 * s_s)))
        put("solve", byt / 1e9, peaks["hbm_gbs"], "GB/s", "hbm", peaks["source"])
    dd = np.asarray(d, np.float64)
    nr = np.asarray(runs, np.float64)
    # 8 flops (one complex multiply-add) per (direction, segment); the
    # per-(direction, wire run) sincos pairs are not counted as flops
    # antennas whose wires all run along z (runs[i] < 0 marks them, -runs[i]
    # wire runs) evaluate each run's Horner polynomial once per (block,
    # integration row): 8 flops per (row, segment), plus one complex
    # multiply-add per (direction, run) -- the far-field kernel's work for them
    vert = nr < 0
    nrun = np.abs(nr)
    pec = np.asarray(g, np.float64) > 0
    blocks = np.ceil(dd / 256.0)
    ff = np.where(vert, blocks * 2 * (1 + pec) * 8 * n + dd * (1 + pec) * 8 * nrun, dd * 8 * n)
    put("farfield", float(np.sum(ff)) / 1e12, fma, "TFLOP/s", "fp64",
        "DFMA measured by fnec_measure_fp64_peak")
    return res


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


def cpu_oracle_units(ref_units, n_units: int, threads: int):
    """Solve an evenly spaced sample of n_units workload units with the CPU
    oracle on `threads` threads; returns (solves/s, seconds, problems, idx)."""
    from oracle import oracle as O

    idx = np.linspace(0, len(ref_units) - 1, n_units).round().astype(int)
    probs = []
    for i in idx:
        w, src, g, f, rp = ref_units[i][:5]
        wave = O.wave(*ref_units[i][5]) if len(ref_units[i]) > 5 else None
        pts = O.rp_card_points(*rp) if rp is not None else None
        probs.append(O.Problem(O.wires_array(w), O.sources_array(src), f, ground=g, points=pts, wave=wave))
    t0 = time.perf_counter()
    O.solve_problems(probs, threads)
    dt = time.perf_counter() - t0
    assert all(p.status == 0 for p in probs)
    return n_units / dt, dt, probs, idx


def reference_units(args):
    """The workload's units as (wires, sources, ground, freq, rp) tuples."""
    if args.workload == "sweep5":
        wires, sources, freqs, rp = sweep_workload(n_freqs=args.freqs)
        return [(wires, sources, 0, f, rp) for f in freqs], "sweep5: 5-wire parallel array, N=255 (S=260), " \
            f"{len(freqs)} freqs 13.0-15.5 MHz, RP 91x361 per freq"
    if args.workload == "mesh":
        wl, src, f = mesh_workload(args.cells)
        return [(wl, src, 1, f, None)], f"mesh: {args.cells}x{args.cells} cells over PEC ground"
    if args.workload == "receive":
        wires, freqs, card = receive_workload(args.n_theta, args.n_phi)
        return receive_units(wires, freqs, card), RECEIVE_DESC(args.n_theta, args.n_phi)
    if args.workload == "serve":
        reqs = serve_requests(512, seed=13)
        return ([(w, [s], g, f, rp) for w, srcs, g, f, rp in reqs for s in srcs],
                "serve: random antennas, N lognormal (median 150), 1-4 source positions, half with 91x361 RP")
    wl = uneven_workload(args.antennas)
    return [(w, src, g, f, None) for w, src, g, f in wl], uneven_desc(len(wl))


def run_reference(args):
    """The CPU implementation of the path (the oracle restating the
    reference CPU code) on all host threads, on this workload."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    ref_units, desc = reference_units(args)
    threads = os.cpu_count() or 1
    n = min(len(ref_units), 2 * max(threads, 1))
    for _ in range(args.warmup):
        cpu_oracle_units(ref_units, min(n, 8), threads)
    times = []
    for _ in range(args.steps):
        _, dt, _, _ = cpu_oracle_units(ref_units, n, threads)
        times.append(dt)
    rate = n * len(times) / sum(times)
    metric = "receive solves/s (plane-wave incidence directions x frequencies)" if args.workload == "receive" \
        else METRIC
    line = {
        "impl": "reference", "metric": metric, "value": rate, "unit": "solves/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(times)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)",
        "config": {"workload": desc, "sample_units_per_step": n},
        "cpu_baseline": {"value": rate, "unit": "solves/s", "cores": threads, "kind": "port",
                         "sample": f"{n} evenly spaced units of the workload per step, one solve per thread, "
                                   f"CPU oracle (C restatement of the reference CPU path, -O2 -ffp-contract=off); "
                                   f"the Rust reference itself cannot be built here"},
        "e2e": {"value": rate, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def RECEIVE_DESC(nth, nph):
    return (f"receive: 5-wire parallel array (N=255, S=265), EX 2 plane wave, {nth}x{nph} incidence directions "
            f"x 3 freqs, each direction one right-hand side of its frequency's factorisation")


def run_receive(args, acc, ctx, rank, local, dist):
    """The plane-wave receive sweep (solve_session.rs:313-375): all
    incidence directions of all frequencies in one FP64 batch; a unit is one
    (frequency, direction) receive solve.  e2e uploads the batch tables,
    runs, and reads the receive pattern (3 doubles per unit)."""
    import torch

    wires, freqs, card = receive_workload(args.n_theta, args.n_phi)
    ant = acc.Antenna(acc.wires_array(wires), acc.sources_array([]), freqs, acc.GROUND_FREE, None, plane_wave=card)
    batch = acc.HallenBatch([ant], precision=acc.PRECISION_FP64, ctx=ctx)
    units = len(batch.units)
    stream = torch.cuda.ExternalStream(acc.lib().fnec_ctx_stream(ctx.handle), device=local)
    # schedule: the autotuner's pick, timed before and outside the timed region
    tune = None if args.no_tune else batch.tune(reps=args.tune_reps)
    if args.schedule:
        batch.schedule = json.loads(args.schedule)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(local)

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
    clocks = clock_summary(sampler) if sampler is not None else None
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record(stream)
    for _ in range(args.steps):
        batch.upload()
        batch.run()
        rec = batch.read_receive()  # synchronises: device peaks -> host, dB per unit
    e1.record(stream)
    batch.sync()
    barrier()
    e2e_ms = e0.elapsed_time(e1)
    batch.set_profiling(True)
    phase = {k: 0.0 for k in batch.PHASES}
    for _ in range(3):
        batch.run()
        for k, v in batch.phase_ms().items():
            phase[k] += v / 3
    batch.set_profiling(False)
    vals = torch.tensor([float(step_ms.sum()), e2e_ms], dtype=torch.float64, device=f"cuda:{local}")
    if dist is not None:
        dist.all_reduce(vals, op=dist.ReduceOp.MAX)
    total_ms, e2e_ms = vals.tolist()
    res = batch.read()
    launches = batch.kernel_launches * args.steps
    if rank == 0:
        _, muladd_tf = acc.measure_fp64_peak(local)
        n = 255.0
        s = n + 2 * len(wires)
        nsys = len(freqs)
        lw = [w[1] for w in wires]
        pairs = float(sum(L * L for L in lw))
        # work per phase (real FP64 ops): rhs 6 per (direction, same-wire
        # segment pair) + the per-system sin table; solve: Z^H y (8 N^2) and
        # the cos/sin columns (16 N) per extra direction, forward + back
        # substitution 8 S^2 per direction
        work = {"rhs": units * (6.0 * pairs + n * (8 + 2 * SINCOS_FLOPS)) + nsys * pairs * SINCOS_FLOPS,
                "gram": nsys * 8.0 * n * n * (n + 1), "factor": nsys * 8.0 * s ** 3 / 3,
                "solve": (units - nsys) * (8.0 * n * n + 16.0 * n) + units * 8.0 * s * s}
        dom = max(("rhs", "fill", "gram", "factor", "solve"), key=lambda k: phase[k])
        rr = {k: {"achieved": w / 1e12 / (phase[k] * 1e-3), "unit": "TFLOP/s", "bound": "fp64",
                  "peak": muladd_tf, "frac": w / 1e12 / (phase[k] * 1e-3) / muladd_tf}
              for k, w in work.items() if phase[k] > 0}
        roof = dict(rr.get(dom, {"bound": "fp64", "achieved": None, "peak": muladd_tf, "unit": "TFLOP/s",
                                 "frac": None}))
        roof.update({"kernel": dom, "traffic": None,
                     "peak_source": "DMUL+DADD measured by fnec_measure_fp64_peak (the exact path issues no FMA)"})
        line = {
            "metric": "receive solves/s (plane-wave incidence directions x frequencies)", "workload": "receive",
            "value": args.gpus * units * args.steps / (total_ms * 1e-3), "unit": "solves/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded 5-element array, seed 11)",
            "config": {"workload": RECEIVE_DESC(args.n_theta, args.n_phi), "units_per_step": units,
                       "precision": "fp64", "l2": "per-step working set ~60 MB (Z, factors, right-hand sides "
                                                  "of 3 systems): L2-resident, no flush",
                       "parallelism": f"replicas x{args.gpus} (no collective)"},
            "e2e": {"value": args.gpus * units * args.steps / (e2e_ms * 1e-3), "unit": "solves/s",
                    "h2d_bytes_per_step": int(batch.h2d_bytes), "d2h_bytes_per_step": 8 * units},
            "gpu_launches": int(launches), "roofline": roof, "phase_rooflines": rr,
            "phase_ms": {k: round(v, 4) for k, v in phase.items()}, "clocks": clocks,
            "receive_db_range": [float(np.min(rec[:, 2])), float(np.max(rec[:, 2]))],
            "schedule": {"schedule": batch.schedule,
                         "tune": None if tune is None else {k: tune[k] for k in ("candidates", "default_ms", "best_ms")}},
        }
        if not args.no_cpu_baseline:
            ref = receive_units(wires, freqs, card)
            threads = os.cpu_count() or 1
            n_units = max(threads, 8)
            rate, dt, probs, idx = cpu_oracle_units(ref, n_units, threads)
            line["cpu_baseline"] = {"value": rate, "unit": "solves/s", "cores": threads, "kind": "port",
                                    "sample": f"{n_units} evenly spaced (frequency, direction) receive solves, one "
                                              f"per thread, each a full solve as the reference re-solves every "
                                              f"direction, {dt:.1f} s wall"}
            dev = max(float(np.abs(res.currents[i] - p.currents).max() / max(np.abs(p.currents).max(), 1e-300))
                      for p, i in zip(probs, idx))
            line["parity"] = {"units_checked": n_units, "max_rel_current_vs_oracle": dev}
        print(json.dumps(line), flush=True)
    batch.close()


def run_serve(args, acc, ctx, rank, local, dist):
    """The served request stream: requests arrive as a Poisson process at
    each offered rate; the submitting loop replays the arrival times and the
    server (continuous batching over `lanes` streams, HBM-budget admission)
    returns each request's currents, feedpoints and pattern into host
    arrays.  Latency is submit -> results delivered, measured by the server.
    Every number here is end to end (host decks in, host arrays out)."""
    import torch

    rates = [float(r) for r in args.rates.split(",")]
    rng = np.random.default_rng(29)
    n_pool = int(min(4000, max(rates) * args.serve_seconds))
    pool = serve_requests(n_pool, seed=13)
    ants = [acc.Antenna(acc.wires_array(w), acc.sources_array(srcs), [f], g, rp, separate_sources=True)
            for w, srcs, g, f, rp in pool]
    warm = ants[: min(64, len(ants))]
    forms = {"mixed": acc.PRECISION_MIXED, "fp64": acc.PRECISION_FP64}
    if args.precision == "fp64":
        forms = {"fp64": acc.PRECISION_FP64}
    elif args.precision == "mixed-only":
        forms = {"mixed": acc.PRECISION_MIXED}
    res = {}
    feeds = {}
    clocks = None
    for name, prec in forms.items():
        srv = acc.Server(prec, lanes=args.lanes, hbm_budget_bytes=int(args.budget_gb * (1 << 30)), max_batch=256,
                         ctx=ctx)
        for _ in range(max(1, args.warmup)):
            for r in [srv.submit(a) for a in warm]:
                srv.wait(r)
                r.release()
        res[name] = []
        for k, rate in enumerate(rates):
            n = int(min(len(ants), max(8, rate * args.serve_seconds)))
            gaps = rng.exponential(1.0 / rate, size=n)
            arrive = np.cumsum(gaps) - gaps[0]
            srv.stats(reset=True)
            sampler = clock_sampler(local) if (name == "mixed" or len(forms) == 1) and k == len(rates) - 1 else None
            keep = k == len(rates) - 1
            last = [None] * n if keep else None
            t_done = [0.0]

            def consume():
                # a client thread: takes finished requests in completion order,
                # reads what it needs and releases them (their memory recycles)
                got = 0
                while got < n:
                    r = srv.next_done(5000.0)
                    if r is None:
                        raise RuntimeError("served request stream stalled")
                    if keep:
                        last[r.tag] = np.array(r.result()[1], copy=True)
                    r.release()
                    got += 1
                t_done[0] = time.perf_counter()

            import threading
            th = threading.Thread(target=consume)
            th.start()
            t0 = time.perf_counter()
            for i in range(n):
                while time.perf_counter() - t0 < arrive[i]:
                    pass
                srv.submit(ants[i], tag=i)
            t_sub = time.perf_counter() - t0
            th.join()
            wall = t_done[0] - t0
            if sampler is not None:
                clocks = clock_summary(sampler)
            st = srv.stats()
            res[name].append({"offered_req_per_s": rate, "requests": n,
                              "achieved_submit_req_per_s": n / t_sub if t_sub > 0 else None,
                              "solves": int(st["solves"]), "wall_s": wall,
                              "solves_per_s": st["solves"] / wall, "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"],
                              "mean_ms": st["mean_ms"], "batches": int(st["batches"]),
                              "max_batch": int(st["max_batch"]), "peak_in_flight_gb": st["peak_in_flight_bytes"] / 1e9,
                              "kernel_launches": int(st["kernel_launches"]), "h2d": int(st["h2d_bytes"]),
                              "d2h": int(st["d2h_bytes"]), "failed": int(st["failed"]),
                              "loop_host_ms": {"plan": st["plan_ms"], "alloc": st["alloc_ms"],
                                               "alloc_device": st["alloc_device_ms"],
                                               "alloc_upload": st["alloc_upload_ms"],
                                               "alloc_pinned": st["alloc_pinned_ms"],
                                               "alloc_mixed": st["alloc_mixed_ms"],
                                               "launch": st["launch_ms"], "collect": st["collect_ms"]}})
            if last is not None:
                feeds[name] = last
        srv.close()
    if rank != 0:
        return
    gate = None
    if "mixed" in feeds and "fp64" in feeds:
        dz = 0.0
        for a, b in zip(feeds["mixed"], feeds["fp64"]):
            zm = a[:, 5] + 1j * a[:, 6]
            zp = b[:, 5] + 1j * b[:, 6]
            dz = max(dz, float(np.max(np.abs(zm - zp) / np.abs(zp))))
        gate = {"max_rel_dzin_mixed_vs_fp64_gpu": dz, "gate": 1e-6, "passed": bool(dz <= 1e-6)}
    head = "mixed" if ("mixed" in res and (gate is None or gate["passed"])) else "fp64"
    H = res[head][-1]
    line = {
        "metric": METRIC, "value": H["solves_per_s"] * args.gpus, "unit": "solves/s", "n_gpus": args.gpus,
        "steps": H["requests"], "warmup": max(1, args.warmup) * len(warm), "ms_per_step": 1e3 * H["wall_s"] / H["requests"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if head == "fp64" else "f32+f64",
        "data": "synthetic (seeded served request stream, seed 13; Poisson arrivals, seed 29)",
        "config": {"workload": f"serve: Poisson requests at {rates} req/s, random antennas (N lognormal median 150, "
                               f"cap 4096), 1-4 source positions each, half with a 91x361 pattern",
                   "precision": head, "lanes": args.lanes, "hbm_budget_gb": args.budget_gb,
                   "step": "one request", "l2": "per-batch working sets differ; no flush between requests",
                   "parallelism": f"replicas x{args.gpus} (no collective)"},
        "latency_ms": {"p50": H["p50_ms"], "p99": H["p99_ms"], "what": "request submit -> results in host arrays",
                       "offered_req_per_s": H["offered_req_per_s"]},
        "e2e": {"value": H["solves_per_s"] * args.gpus, "unit": "solves/s",
                "h2d_bytes_per_step": int(H["h2d"] / max(H["requests"], 1)),
                "d2h_bytes_per_step": int(H["d2h"] / max(H["requests"], 1))},
        "gpu_launches": H["kernel_launches"],
        "roofline": {"kernel": None, "bound": None, "achieved": None, "peak": None, "unit": None, "frac": None,
                     "traffic": None, "note": "the served stream runs the batch kernels; their rooflines are "
                                              "reported by --workload uneven and sweep5"},
        "clocks": clocks,
        "rates": res,
    }
    if gate is not None:
        line["mixed_gate"] = gate
        line["mixed_vs_fp64"] = res["mixed"][-1]["solves_per_s"] / res["fp64"][-1]["solves_per_s"]
    if not args.no_cpu_baseline:
        ref_units, _ = reference_units(args)
        threads = os.cpu_count() or 1
        n_units = min(len(ref_units), max(threads, 4))
        rate, dt, _, _ = cpu_oracle_units(ref_units, n_units, threads)
        line["cpu_baseline"] = {"value": rate, "unit": "solves/s", "cores": threads, "kind": "port",
                                "sample": f"{n_units} single-source decks of the request stream, one per thread, "
                                          f"{dt:.1f} s wall"}
    print(json.dumps(line), flush=True)


def rank_workload(args, acc, world, rank):
    """This rank's antennas of a batch workload.  The uneven batch is a job
    of world x `antennas` random antennas split across ranks by the work
    model (nec_accel.shard.partition_antennas: largest first onto the least
    loaded rank); sweep5 and the mesh run as replicas (one sweep or one mesh
    per rank).  Returns (antennas, reference units, job indices of this
    rank's units, job size, description, data)."""
    from nec_accel import shard

    if args.workload == "sweep5":
        wires, sources, freqs, rp = sweep_workload(n_freqs=args.freqs)
        ants = [acc.Antenna(acc.wires_array(wires), acc.sources_array(sources), freqs, acc.GROUND_FREE, rp)]
        desc = (f"sweep5: 5-wire parallel array, N=255 (S=260), {len(freqs)} freqs 13.0-15.5 MHz, "
                f"RP 91x361 per freq")
        ref = [(wires, sources, acc.GROUND_FREE, f, rp) for f in freqs]
        return ants, ref, list(range(len(ref))), len(ref) * world, desc, \
            "synthetic (seeded 5-element array, seed 11)", f"replicas x{world} (no collective)"
    if args.workload == "mesh":
        wl, src, f = mesh_workload(args.cells)
        ants = [acc.Antenna(acc.wires_array(wl), acc.sources_array(src), [f], acc.GROUND_PEC, None)]
        desc = (f"mesh: {args.cells}x{args.cells} cells of 2-segment wires over PEC ground (GN 1), N={2 * len(wl)}, "
                f"W={len(wl)}, one frequency 14.2 MHz, no pattern")
        return ants, [(wl, src, acc.GROUND_PEC, f, None)], [0], world, desc, \
            "synthetic (seeded jittered mesh, seed 5)", f"replicas x{world} (one solve; no distributed LU)"
    wl = uneven_workload(args.antennas * world)
    all_ants = [acc.Antenna(acc.wires_array(w), acc.sources_array(src), [f], g, None) for w, src, g, f in wl]
    parts = shard.partition_antennas(all_ants, world, mixed=args.precision != "fp64")
    mine = parts[rank]
    desc = uneven_desc(len(wl))
    if world > 1:
        desc += f"; {len(mine)} on this rank (work-balanced shard {rank}/{world})"
    ref = [(wl[i][0], wl[i][1], wl[i][2], wl[i][3], None) for i in mine]
    par = "1 GPU" if world == 1 else f"sharded x{world}: work-balanced partition of the antennas, no collective"
    return [all_ants[i] for i in mine], ref, mine, len(wl), desc, "synthetic (seeded random antennas, seed 7)", par


def current_err(a, b):
    """Normwise relative difference of two current vectors (2-norm)."""
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def gain_err(pa, pb):
    """Largest |difference| in dB of the three gain columns over the points
    where the reference value is printed (above -999.99 dB)."""
    g = pb[:, :3]
    ok = g > -900
    if not np.any(ok):
        return 0.0
    return float(np.max(np.abs(pa[:, :3][ok] - g[ok])))


def measure_batch(args, acc, batch, stream, rank, local, dist, steps, warmup, with_clocks):
    """Device-timed steps with inputs resident, then the same steps end to
    end through the C ABI with host buffers, then per-phase times."""
    import torch

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(local)

    for _ in range(warmup):
        batch.run()
    batch.sync()
    sampler = clock_sampler(local) if (rank == 0 and with_clocks) else None
    barrier()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    evs[0].record(stream)
    for k in range(steps):
        batch.run()
        evs[k + 1].record(stream)
    batch.sync()
    barrier()
    step_ms = np.array([evs[k].elapsed_time(evs[k + 1]) for k in range(steps)])
    clocks = clock_summary(sampler) if sampler is not None else None
    launches = batch.kernel_launches * steps
    # end to end through the C ABI with host buffers
    batch.read_raw()
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        batch.upload()
        batch.run_report()  # the pattern columns stream out chunk by chunk behind the far field
        batch.read_report(pattern=False)  # synchronises; currents, feeds, status
    e1.record(stream)
    batch.sync()
    barrier()
    e2e_ms = e0.elapsed_time(e1)
    # per-phase times (profiled runs, outside the timed regions)
    batch.set_profiling(True)
    phase = {k: 0.0 for k in batch.PHASES}
    for _ in range(3):
        batch.run()
        for k, v in batch.phase_ms().items():
            phase[k] += v / 3
    batch.set_profiling(False)
    vals = torch.tensor([float(step_ms.sum()), e2e_ms], dtype=torch.float64, device=f"cuda:{local}")
    if dist is not None:
        dist.all_reduce(vals, op=dist.ReduceOp.MAX)
    total_ms, e2e_ms = vals.tolist()
    return {"step_ms": step_ms, "total_ms": total_ms, "e2e_ms": e2e_ms, "clocks": clocks,
            "launches": int(launches), "h2d": batch.h2d_bytes, "d2h": batch.d2h_report_bytes(), "phase": phase,
            "res": batch.read()}


def measure_followup(acc, batch, stream, local, dist, steps):
    """Follow-up requests on the resident factorisations: new voltage
    sources for the sweep (the source moved along element 2, alternating
    between two positions), then every frequency solved again on the stored
    factor (fnec_batch_set_sources + fnec_batch_resolve: right-hand sides,
    substitution or refinement, feedpoints, pattern; no fill, Gram or
    factorisation).  CUDA events on the batch's stream; max over ranks."""
    import torch

    srcs = [[(2, 20, 1.0)], [(2, 32, 1.0)]]
    batch.set_sources(0, srcs[0])
    batch.resolve(read=False)
    batch.sync()
    if dist is not None:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(steps):
        batch.set_sources(0, srcs[k % 2])
        batch.resolve(read=False)
    e1.record(stream)
    batch.sync()
    ms = e0.elapsed_time(e1)
    vals = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{local}")
    if dist is not None:
        dist.all_reduce(vals, op=dist.ReduceOp.MAX)
    batch.set_sources(0, [(2, 26, 1.0)])  # the workload's own source again
    return {"ms_per_step": vals.item() / steps, "steps": steps}


def measure_with_planning(acc, ants, prec, ctx, stream, local, dist, steps):
    """End to end per call when every call brings new geometries: the C
    ABI's batch planning (topology, junctions, constraint rows, packing,
    device allocation), upload, run, the report's results to host memory and
    the batch's release, timed by the host clock between device
    synchronisations (max over ranks)."""
    import torch

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(local)

    b = acc.HallenBatch(ants, precision=prec, ctx=ctx)  # warm-up: caches, allocator
    b.run()
    b.read_report()
    b.close()
    barrier()
    t0 = time.perf_counter()
    plan = 0.0
    for _ in range(steps):
        p0 = time.perf_counter()
        b = acc.HallenBatch(ants, precision=prec, ctx=ctx)  # plans and uploads
        plan += time.perf_counter() - p0
        b.run()
        b.read_report()
        b.close()
    barrier()
    ms = 1e3 * (time.perf_counter() - t0)
    vals = torch.tensor([ms, 1e3 * plan], dtype=torch.float64, device=f"cuda:{local}")
    if dist is not None:
        dist.all_reduce(vals, op=dist.ReduceOp.MAX)
    return vals.tolist()


def run_batch_workload(args, acc, ctx, rank, local, dist, world, steps, warmup, oracle_units=0,
                       with_planning=False):
    """Both forms of one batch workload; rank 0 returns the JSON line."""
    import torch

    ants, ref_units, job_index, job_units, desc, data, parallelism = rank_workload(args, acc, world, rank)
    units_local = len(ref_units)
    stream = torch.cuda.ExternalStream(acc.lib().fnec_ctx_stream(ctx.handle), device=local)
    forms = {"mixed": ["mixed", "fp64"], "fp64": ["fp64"], "mixed-only": ["mixed"]}[args.precision]
    out = {}
    for form in forms:
        prec = acc.PRECISION_MIXED if form == "mixed" else acc.PRECISION_FP64
        batch = acc.HallenBatch(ants, precision=prec, ctx=ctx)
        shapes = batch.units
        # schedule: the autotuner's pick (timed before, outside the timed region)
        tune = None if args.no_tune else batch.tune(reps=args.tune_reps)
        if args.schedule and form == "mixed":
            batch.schedule = json.loads(args.schedule)
        out[form] = measure_batch(args, acc, batch, stream, rank, local, dist, steps, warmup,
                                  with_clocks=(form == forms[0]))
        st, nodes = batch.graph_state()
        out[form]["schedule"] = {"schedule": batch.schedule,
                                 "graph": {1: "replayed", 0: "eager", -1: "capture refused"}[st],
                                 "graph_kernels": nodes}
        if tune is not None:
            out[form]["schedule"]["tune"] = {k: tune[k] for k in ("candidates", "default_ms", "best_ms", "key")}
        if args.workload == "sweep5":
            out[form]["followup"] = measure_followup(acc, batch, stream, local, dist, steps)
        if form == "mixed":
            it, rs = batch.refinement_stats()
            out[form]["gmres"] = {"iters_mean": float(it.mean()), "iters_max": int(it.max()),
                                  "resid_max": float(rs.max())}
            out[form]["gmres_iters"] = it.astype(np.float64)
        batch.close()
        if with_planning:
            ms, plan_ms = measure_with_planning(acc, ants, prec, ctx, stream, local, dist, max(1, min(steps, 3)))
            out[form]["planning"] = {"ms": ms / max(1, min(steps, 3)), "plan_ms": plan_ms / max(1, min(steps, 3)),
                                     "steps": max(1, min(steps, 3))}

    # results of this rank's units gathered on rank 0 in job order (feedpoint
    # rows: 7 doubles per row)
    gathered = None
    if dist is not None and args.workload == "uneven":
        from nec_accel import shard

        got = shard.gather_units([f.copy() for f in out[forms[0]]["res"].feeds], job_index, job_units, dst=0)
        if rank == 0:
            gathered = {"units": len(got), "all_present": bool(all(g is not None for g in got))}
    if rank != 0:
        return None
    fma_tf, muladd_tf = acc.measure_fp64_peak(local)
    ffma_tf = acc.measure_fp32_peak(local)
    peaks = measured_peaks()
    n_u = np.array([u["n"] for u in shapes], np.float64)
    s_u = np.array([u["s"] for u in shapes], np.float64)
    g_u = np.array([ref_units[i][2] if i < len(ref_units) else 0 for i in range(len(shapes))], np.float64)
    d_u = [ff_directions(ref_units[i][2], ref_units[i][4]) if u["n_points"] else 0 for i, u in enumerate(shapes)]
    flops = algorithmic_flops(n_u, s_u, d_u)
    def wire_runs(u):
        # -W for antennas whose wires all run along z (the far field's per-row path), else W
        wl = ref_units[u][0] if u < len(ref_units) else []
        if not wl:
            return 1
        z_par = all(w[2][0] == w[3][0] and w[2][1] == w[3][1] for w in wl)
        return -len(wl) if z_par else len(wl)

    w_u = [wire_runs(i) for i in range(len(shapes))]
    rr = {form: phase_rooflines(form, out[form], n_u, s_u, g_u, d_u, shapes, fma_tf, muladd_tf, ffma_tf, peaks,
                                w_u) for form in forms}
    # accuracy of the chosen form against the plain FP64 GPU path (all units)
    gate = None
    if "mixed" in out and "fp64" in out:
        rm, rp_ = out["mixed"]["res"], out["fp64"]["res"]
        dz = max(abs(complex(*a[0, 5:7]) - complex(*b[0, 5:7])) / abs(complex(*b[0, 5:7]))
                 for a, b in zip(rm.feeds, rp_.feeds))
        di = max(current_err(a, b) for a, b in zip(rm.currents, rp_.currents))
        gate = {"max_rel_dzin_mixed_vs_fp64_gpu": dz, "gate": 1e-6, "passed": bool(dz <= 1e-6),
                "max_rel_current_mixed_vs_fp64_gpu": di, "units": len(rm.feeds)}
        if any(len(p) for p in rm.pattern):
            gate["max_abs_gain_db_mixed_vs_fp64_gpu"] = max(gain_err(a, b) for a, b in zip(rm.pattern, rp_.pattern)
                                                            if len(b))
    headline = forms[0] if (gate is None or gate["passed"]) else "fp64"
    H = out[headline]
    phase = H["phase"]
    dom = max(("fill", "gram", "factor", "solve", "farfield"), key=lambda k: phase[k])
    roof = dict(rr[headline][dom])
    roof["kernel"] = dom
    roof["traffic"], roof["traffic_source"] = dram_traffic(dom, headline, units_local, args.workload)
    samples = flops["fill_samples"]
    per_step_units = job_units
    line = {
        "metric": METRIC,
        "value": per_step_units * steps / (H["total_ms"] * 1e-3),
        "unit": "solves/s",
        "n_gpus": args.gpus,
        "steps": steps,
        "warmup": warmup,
        "ms_per_step": H["total_ms"] / steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if headline == "fp64" else "f32+f64",
        "data": data,
        "config": {"workload": desc, "precision": headline, "units_per_step": per_step_units,
                   "units_this_rank": units_local,
                   "l2": "working set > 0.9 GB per step > 126 MB L2 (no flush needed)",
                   "parallelism": parallelism},
        "latency_ms": {"p50": float(np.percentile(H["step_ms"], 50)),
                       "p99": float(np.percentile(H["step_ms"], 99)),
                       "what": f"batch ({units_local}-solve step) latency"},
        "e2e": {"value": per_step_units * steps / (H["e2e_ms"] * 1e-3), "unit": "solves/s",
                "h2d_bytes_per_step": int(H["h2d"]), "d2h_bytes_per_step": int(H["d2h"])},
        "gpu_launches": int(sum(o["launches"] for o in out.values())),
        "roofline": roof,
        "phase_ms": {k: round(v, 4) for k, v in phase.items()},
        "phase_detail": {"fill_gsamples_per_s": samples / (phase["fill"] * 1e-3) / 1e9
                         if phase["fill"] else None,
                         "measured_peaks": {"fp64_dfma_tflops": fma_tf, "fp64_dmul_dadd_tflops": muladd_tf,
                                            "fp32_ffma_tflops": ffma_tf, **peaks}},
        "phase_rooflines": rr,
        "clocks": out[forms[0]]["clocks"],
    }
    if gathered is not None:
        line["gathered_on_rank0"] = gathered
    for form in forms:
        o = out[form]
        line[f"form_{form}"] = {"value": per_step_units * steps / (o["total_ms"] * 1e-3),
                                "ms_per_step": o["total_ms"] / steps,
                                "e2e_value": per_step_units * steps / (o["e2e_ms"] * 1e-3),
                                "phase_ms": {k: round(v, 4) for k, v in o["phase"].items()}}
        if "gmres" in o:
            line[f"form_{form}"]["gmres"] = o["gmres"]
        if "followup" in o:
            fu = o["followup"]
            line[f"form_{form}"]["followup_resident"] = {
                "value": per_step_units / (fu["ms_per_step"] * 1e-3), "unit": "solves/s",
                "ms_per_step": fu["ms_per_step"],
                "what": "new source position on every frequency, solved on the resident factorisations "
                        "(fnec_batch_set_sources + fnec_batch_resolve): right-hand sides, substitution or "
                        "refinement, feedpoints, the 91x361 pattern; device time"}
        if "planning" in o:
            pl = o["planning"]
            line[f"form_{form}"]["e2e_with_planning"] = {
                "value": per_step_units / (pl["ms"] * 1e-3), "unit": "solves/s", "ms_per_step": pl["ms"],
                "planning_ms_per_step": pl["plan_ms"], "steps": pl["steps"],
                "what": "every step plans a new batch through the C ABI (topology, junctions, constraint rows, "
                        "packing, device allocation), uploads, runs, reads the results and frees the batch; "
                        "host clock between device synchronisations"}
        line[f"form_{form}"]["schedule"] = o["schedule"]
    if "planning" in H:
        line["e2e_with_planning"] = line[f"form_{headline}"]["e2e_with_planning"]
    if gate is not None:
        line["mixed_gate"] = gate
        line["mixed_vs_fp64"] = line["form_mixed"]["value"] / line["form_fp64"]["value"]
        line["mixed_vs_fp64_e2e"] = line["form_mixed"]["e2e_value"] / line["form_fp64"]["e2e_value"]
    if args.workload == "mesh" and args.cells > 12:
        line["cpu_baseline"] = {"value": None, "unit": "solves/s", "cores": os.cpu_count() or 1, "kind": "port",
                                "sample": "not run: the faithful single-threaded CPU solve of this mesh takes "
                                          "hours (2.9e13 flops of naive Gram + 5.8e12 of GEPP)"}
    elif oracle_units:
        threads = os.cpu_count() or 1
        n_units = min(units_local, oracle_units)
        rate, dt, probs, idx = cpu_oracle_units(ref_units, n_units, threads)
        line["cpu_baseline"] = {"value": rate, "unit": "solves/s", "cores": threads, "kind": "port",
                                "sample": f"{n_units} evenly spaced units of the workload, one per thread, "
                                          f"{dt:.1f} s wall"}
        par = {"units_checked": n_units, "unit_index": [int(i) for i in idx]}
        for form in forms:
            rr_ = out[form]["res"]
            par[f"max_rel_dzin_{form}_vs_oracle"] = float(max(
                abs(complex(*rr_.feeds[i][0, 5:7]) - p.zin[0]) / abs(p.zin[0]) for p, i in zip(probs, idx)))
            par[f"max_rel_current_{form}_vs_oracle"] = float(max(
                current_err(rr_.currents[i], p.currents) for p, i in zip(probs, idx)))
            if any(len(rr_.pattern[i]) for i in idx):
                par[f"max_abs_gain_db_{form}_vs_oracle"] = float(max(
                    gain_err(rr_.pattern[i], p.pattern) for p, i in zip(probs, idx) if len(rr_.pattern[i])))
        line["parity"] = par
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed", "mixed-only"],
                    help="mixed: time the chosen form and the plain FP64 form; fp64: plain only; "
                         "mixed-only: the chosen form alone, no accuracy gate (for profiling)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--freqs", type=int, default=201, help="sweep points (201 = the workload; fewer = profiling)")
    ap.add_argument("--workload", default="uneven", choices=["sweep5", "uneven", "mesh", "serve", "receive"],
                    help="uneven: 4096 random antennas of uneven N in one batch (headline); sweep5: the 5-wire "
                         "frequency sweep; mesh: the junctioned wire mesh over ground (one large solve); serve: "
                         "a Poisson request stream through the continuous-batching server; receive: the "
                         "plane-wave receive sweep")
    ap.add_argument("--no-extra", action="store_true",
                    help="uneven: skip the extra sweep5 measurement reported under the key 'sweep5'")
    ap.add_argument("--extra-steps", type=int, default=10, help="timed steps of the extra sweep5 measurement")
    ap.add_argument("--rates", default="100,1000,5000,20000", help="serve: offered request rates (req/s)")
    ap.add_argument("--serve-seconds", type=float, default=2.0, help="serve: arrival window per rate")
    ap.add_argument("--lanes", type=int, default=4, help="serve: concurrent batches")
    ap.add_argument("--budget-gb", type=float, default=64.0, help="serve: HBM budget of the batches in flight")
    ap.add_argument("--cells", type=int, default=46, help="mesh workload size (cells per side)")
    ap.add_argument("--n-theta", type=int, default=37, help="receive: incidence directions in theta")
    ap.add_argument("--n-phi", type=int, default=72, help="receive: incidence directions in phi")
    ap.add_argument("--antennas", type=int, default=4096, help="uneven workload size (per GPU)")
    ap.add_argument("--no-tune", action="store_true",
                    help="skip the autotuner (default schedule; the pipeline is still graph-captured)")
    ap.add_argument("--tune-reps", type=int, default=2, help="timed runs per candidate schedule")
    ap.add_argument("--schedule", default="",
                    help='schedule fields set on the (mixed) batch after tuning, JSON, e.g. \'{"tensor_trailing": 1}\'')
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
    if args.workload in ("serve", "receive"):
        (run_serve if args.workload == "serve" else run_receive)(args, acc, ctx, rank, local, dist)
    else:
        threads = os.cpu_count() or 1
        line = run_batch_workload(args, acc, ctx, rank, local, dist, world, args.steps, args.warmup,
                                  oracle_units=0 if args.no_cpu_baseline else max(threads, 4),
                                  with_planning=args.workload == "uneven")
        if args.workload == "uneven" and not args.no_extra:
            # the 5-wire sweep (201 frequencies, 91 x 361 pattern each), kept
            # beside the headline: its far field is the dominant kernel there;
            # the oracle checks 4 of its frequencies (Zin, currents, gains)
            sub = argparse.Namespace(**vars(args))
            sub.workload, sub.freqs = "sweep5", 201
            extra = run_batch_workload(sub, acc, ctx, rank, local, dist, world, args.extra_steps,
                                       max(3, args.warmup), oracle_units=0 if args.no_cpu_baseline else 4)
            if rank == 0:
                keep = ("value", "ms_per_step", "e2e", "roofline", "phase_ms", "mixed_gate", "mixed_vs_fp64",
                        "mixed_vs_fp64_e2e", "parity", "form_mixed", "form_fp64", "config", "steps", "warmup",
                        "gpu_launches")
                line["sweep5"] = {k: extra[k] for k in keep if k in extra}
                line["gpu_launches"] += extra["gpu_launches"]
        if rank == 0:
            print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
