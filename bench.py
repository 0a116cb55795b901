#!/usr/bin/env python3
"""Benchmark of the PO diffraction hot path (one JSON line on rank 0).

Workload: the orientation-averaged hexagonal column of the reference's
headline configuration: --particle 1 100 40 (D = 40 um, L = 100 um),
m = 1.3116 + 1e-9 i, 4 reflections, 16,384 Owen-Sobol orientations (seed 42),
zenith 0..180 deg in 0.1 deg steps x 48 azimuth bins (86,448 directions).
Beams come from the reference's own host tracer (libmbs_host.so, compiled
from the reference sources); they are synthetic only in that no measured
data set is involved.

A step = one pass of the hot path over the whole batch: diffraction of every
(orientation, beam, direction), coherent Jones sums, Mueller conversion and
the orientation average, in the FP32-compensated precision.
  value : orientations/s with the batch resident in HBM (device timing).
  e2e   : the same through the public C-ABI call mbs_po_diffract with pinned
          host buffers: H2D of the beam arrays, kernels, D2H of the Mueller
          grid, every step.
  roofline : algorithmic flop / the diffraction kernel's CUDA-event time
          against the measured FFMA peak (and the nominal one); the plain
          FP64 kernel against the measured DFMA peak.
  parity_vs_reference : FP64 and FP32C through the C ABI against the
          reference's own CPU result on the cpu_baseline sample (M11, the
          normalised elements, C_sca, g, C_ext).
  reference_gpu : the reference's own CUDA build against the drop-in binary
          on the same box, kernels and whole calls.
The FP64 path runs once on the whole batch as the error reference and the
plain FP64 batched path's time.

--impl reference times the reference's own CPU implementation of the path
(HandlerPO::HandleBeamsToLocal + AddToMuellerLocal under OpenMP, built from
the reference sources into oracle/_ref, its tracer and PrepareBeams making
the beams) on a bounded sample of the same orientations, with every host
thread.  --gpus N without a torchrun environment starts N ranks itself.
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

METRIC = "PO orientations/s and beam·dir evals/s at stated M11 error vs plain FP64 path"
WORKLOAD = "orientation-averaged hexagonal column D=40um L=100um, m=1.3116+1e-9i, 4 reflections, " \
           "16384 Sobol orientations, theta 0-180 deg step 0.1 x 48 phi"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--orient", type=int, default=16384)
    ap.add_argument("--n-phi", type=int, default=48)
    ap.add_argument("--n-theta", type=int, default=1800)
    ap.add_argument("--cpu-sample", type=int, default=48, help="orientations in the CPU baseline sample")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 error reference")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-refgpu", action="store_true",
                    help="skip the same-box comparison with the reference's CUDA build")
    ap.add_argument("--refgpu-orient", type=int, default=1024,
                    help="orientations of the same-box comparison with the reference's CUDA build")
    ap.add_argument("--no-autotune", action="store_true",
                    help="skip the launch-shape autotuner (the default shapes run; for launch lists "
                         "under a profiler, whose serialised launches reorder close shapes)")
    ap.add_argument("--launch-selftest", action="store_true",
                    help="ranks only exchange one gloo all-reduce (tests the --gpus N launcher on the CPU)")
    ap.add_argument("--proposal-epochs", type=int, default=200,
                    help="training epochs of the proposal network (workload proposal)")
    ap.add_argument("--proposal-pilot", type=int, default=2048,
                    help="plain Sobol pilot orientations of the proposal (workload proposal)")
    ap.add_argument("--aggregate-distinct", type=int, default=512,
                    help="distinct traced orientations of the aggregate workload, cycled to --orient")
    ap.add_argument("--proposal-rows", default="all", choices=["all", "backscatter"],
                    help="zenith rows whose errors the proposal network targets (workload proposal)")
    ap.add_argument("--proposal-pilot-rows", default="target", choices=["target", "full"],
                    help="rows of the pilot run: the target rows alone (thinned to at most about "
                         "200), or the whole grid (workload proposal)")
    ap.add_argument("--proposal-batch", type=int, default=256,
                    help="training minibatch of the proposal network (workload proposal)")
    ap.add_argument("--workload", default="column", choices=["column", "proposal", "aggregate", "refgpu", "mlp", "fftphi",
                                                          "sizescan"],
                    help="column: the headline line (default); proposal: the learned "
                         "orientation proposal against plain Sobol at equal error; aggregate: "
                         "the non-convex 8-column aggregate (thousands of beams per "
                         "orientation), one graph-captured step per precision; refgpu: the "
                         "reference's own CUDA build against the drop-in binary, same CLI run; mlp: "
                         "training and inference of the proposal network alone; fftphi: the FFT-phi "
                         "azimuth interpolation path against the direct evaluation; sizescan: 16 "
                         "sizes of one traced batch in one launch")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def build_inputs(args, rank, world):
    from mbs_fast_b200 import beams as B, workloads as W
    cfg = W.COLUMN_40x100
    if world > 1:
        # ranks share the host cores (torchrun also sets OMP_NUM_THREADS=1)
        import dataclasses
        cfg = dataclasses.replace(cfg, n_threads=max(1, (os.cpu_count() or 1) // world))
    bs, gs, _ = B.symmetry(cfg)
    # weak scaling: the job averages args.orient x world Sobol orientations
    # and every rank owns a contiguous shard of args.orient of them
    # (TracerPOTotal.cpp:5715-5718 splits ranks the same way); rank 0's
    # shard is the one-GPU workload
    beta, gamma, w = B.sobol_orientations(args.orient * world, bs, gs, 42)
    if world > 1:
        n = args.orient
        beta, gamma, w = beta[rank * n:(rank + 1) * n], gamma[rank * n:(rank + 1) * n], w[rank * n:(rank + 1) * n]
    batch = B.trace(cfg, beta, gamma, w)
    grid = B.grid(0.0, 180.0, args.n_phi, args.n_theta)
    wave = B.wave(cfg)
    return cfg, batch, grid, wave, (beta, gamma, w)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=5)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(mx)) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def algorithmic_flops(batch, n_dirs: int) -> float:
    """F = 12*nv + 168 flops per beam-direction, +100 per orientation-direction
    (the per-unit work definition of the PO path)."""
    return float((12.0 * batch.n_verts + 168.0 * batch.n_beams) * n_dirs
                 + 100.0 * batch.n_orient * n_dirs)


def measured_peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


def reference_sample(cfg, batch, args):
    """The reference's CPU path (oracle/_ref, all host threads) on a bounded
    sample of the batch: the first --cpu-sample orientations on the full grid.
    Returns (cpu_baseline dict, the reference's Mueller grid, its C_ext per
    orientation, the sample), or the restatement's figures when the
    reference library is absent."""
    import oracle
    n = min(args.cpu_sample, batch.n_orient)
    sample = batch.select(0, n)
    spec = (0.0, 180.0, args.n_phi, args.n_theta)
    if oracle.have_reference():
        M_ref, _, cext_ref, sec = oracle.ref_batch(cfg, spec, sample, n_threads=0)
        kind = "reference"
    else:
        from mbs_fast_b200 import beams as B
        t0 = time.perf_counter()
        M_ref = oracle.po_diffract(sample, B.grid(*spec), B.wave(cfg), n_threads=0)
        sec = time.perf_counter() - t0
        cext_ref = oracle.po_extinction(sample, B.wave(cfg))
        kind = "port"
    base = {"value": n / sec, "unit": "orientations/s", "cores": os.cpu_count(), "kind": kind,
            "sample": f"{n} of the {batch.n_orient} orientations on the full "
                      f"{args.n_phi}x{args.n_theta + 1} grid ({sec:.2f} s)",
            "beam_dir_evals_per_s": sample.n_beams * args.n_phi * (args.n_theta + 1) / sec}
    return base, M_ref, cext_ref, sample


def parity_vs_reference(h, sample, M_ref, cext_ref) -> dict:
    """FP64 and FP32C results of the reference's sample, diffracted through
    the C ABI, against the reference's own CPU result of the same
    orientations: M11, the normalised elements, C_sca, g and C_ext (device
    extinction kernel against the reference's ComputeForwardExtinctionOt)."""
    from mbs_fast_b200 import abi, metrics
    out = {"orientations": sample.n_orient}
    cext = h.extinction(sample)
    for prec, name in ((abi.FP64, "fp64"), (abi.FP32C, "fp32c")):
        M = h.new_mueller()
        h.handle_orientations_to_local_gpu(sample, M, precision=prec)
        out[name] = metrics.compare(h, M, M_ref, cext, cext_ref)
    return out


def run_reference(args):
    """The reference's own CPU implementation of the path on the host cores:
    its tracer and PrepareBeams build the orientations' beams (untimed), its
    OpenMP HandleBeamsToLocal + AddToMuellerLocal loop is timed, every host
    thread, on a bounded sample of the headline workload's orientations."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import oracle
    from mbs_fast_b200 import workloads as W
    cfg = W.COLUMN_40x100
    n = max(1, args.cpu_sample)
    spec = (0.0, 180.0, args.n_phi, args.n_theta)
    kind = "reference" if oracle.have_reference() else "port"
    if kind == "reference":
        beta, gamma, w = oracle.ref_orientations(cfg, args.orient, 42)
        beta, gamma, w = beta[:n], gamma[:n], w[:n]
        for _ in range(min(args.warmup, 1)):
            oracle.ref_run(cfg, spec, beta[:2], gamma[:2], w[:2])
        times = []
        for _ in range(args.steps):
            _, _, _, _, td = oracle.ref_run(cfg, spec, beta, gamma, w)
            times.append(td)
        n_beams = None
    else:
        from mbs_fast_b200 import beams as B
        bs, gs, _ = B.symmetry(cfg)
        beta, gamma, w = B.sobol_orientations(args.orient, bs, gs, 42)
        sample = B.trace(cfg, beta[:n], gamma[:n], w[:n])
        grid, wave = B.grid(*spec), B.wave(cfg)
        times = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            oracle.po_diffract(sample, grid, wave, n_threads=0)
            times.append(time.perf_counter() - t0)
        n_beams = sample.n_beams
    sec = float(np.mean(times))
    v = n / sec
    line = {"metric": METRIC, "value": v, "unit": "orientations/s", "n_gpus": 0, "impl": "reference",
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (beams from the reference's own tracer and PrepareBeams)",
            "config": {"workload": WORKLOAD, "sample_orientations": n},
            "cpu_baseline": {"value": v, "unit": "orientations/s", "cores": os.cpu_count(),
                             "kind": kind,
                             "sample": f"the first {n} of the {args.orient} Sobol orientations per "
                                       f"step on the full {args.n_phi}x{args.n_theta + 1} grid; "
                                       "diffraction phase timed"},
            "e2e": {"value": v, "unit": "orientations/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    if n_beams:
        line["beam_dir_evals_per_s"] = n_beams * args.n_phi * (args.n_theta + 1) / sec
    print(json.dumps(line), flush=True)


def run_proposal(args):
    """Learned orientation proposal against plain Sobol on the headline
    column and grid (D=40 um, L=100 um, 0.1 deg zenith rows x 48 azimuth
    bins).  Errors of the azimuth-averaged rows against a 65,536-orientation
    plain FP64 Sobol reference, over all rows (0.5-179.5 deg) and over the
    backscattering rows (170-179.5 deg): RMS relative error of M11 and RMS
    absolute error of -M12/M11.  At N = 1024..8192 orientations (four
    scrambles each): plain FP64 Sobol (the plain FP64 batched path), plain
    FP32C Sobol, the learned FP32C proposal alone and combined with its pilot
    by the balance heuristic.  A power law fitted to each error against N
    gives the orientations to 1 % on M11 and on -M12/M11 (both: the larger);
    the wall time to 1 % is that count times the measured wall time per
    orientation of the whole average with host tracing overlapped (the
    pipeline of the headline line), plus the pilot and the training for the
    learned estimates (16,384 orientations timed per precision).  The network
    is trained on the rows of --proposal-rows."""
    import torch
    from mbs_fast_b200 import abi, beams as B, proposal as PR, workloads as W
    from mbs_fast_b200.handler import GpuHandlerPO
    from mbs_fast_b200.pipeline import orientation_average
    torch.cuda.set_device(0)
    cfg = W.COLUMN_40x100
    bs, gs, _ = B.symmetry(cfg)
    grid = B.grid(0.0, 180.0, args.n_phi, args.n_theta)
    h = GpuHandlerPO(grid, B.wave(cfg))
    th = np.rad2deg(grid.theta)
    regions = {"all": (th > 0.5) & (th < 179.5), "backscatter": (th >= 170) & (th < 179.5)}
    st_best = {}
    for prec, name in ((abi.FP32C, "fp32c"), (abi.FP64, "fp64")):
        bb, gg, ww = B.sobol_orientations(256, bs, gs, 42)
        stg = h.stage(B.trace(cfg, bb, gg, ww))
        st_best[name] = h.autotune(stg, prec, max_orient=256)[0]
        stg.free()

    def rows_of(u, v, w, prec):
        b = PR.orientation_sample_batch(cfg, u, v, w, bs, gs)
        return PR.averaged_rows(h, b, prec)[0]

    # wall time per orientation of the whole average (host tracing
    # overlapped with the device), per precision, on 16,384 orientations
    # (the headline line's pipeline)
    per_orient = {}
    bq, gq, wq = B.sobol_orientations(16384, bs, gs, 7)
    for prec, name in ((abi.FP64, "fp64"), (abi.FP32C, "fp32c")):
        orientation_average(h, cfg, bq[:2048], gq[:2048], wq[:2048], precision=prec, batch=1024)
        walls = sorted(orientation_average(h, cfg, bq, gq, wq, precision=prec, batch=1024)[2]["wall_s"]
                       for _ in range(3))
        per_orient[name] = walls[1] / len(bq)          # the median of three passes

    t0 = time.perf_counter()
    ref = rows_of(*PR.plain_sobol(65536, seed=4242), abi.FP64)
    t_ref = time.perf_counter() - t0
    n_pilot = args.proposal_pilot
    target = regions[args.proposal_rows]
    pilot_th = None
    if args.proposal_pilot_rows == "target":
        pilot_th = PR.pilot_theta_rows(th, target, every=max(1, int(target.sum()) // 192))
    # one untimed fit first: the network library's module load and first
    # launches are not part of a proposal's cost
    PR.train_proposal_with_pilot(h, cfg, 256, rows_mask=target, epochs=2,
                                 batch=args.proposal_batch, pilot_theta_deg=pilot_th)
    # the pilot and fit three times (same seeds, the same proposal): the
    # median time, as the shared host's load shows in single runs
    runs = [PR.train_proposal_with_pilot(h, cfg, n_pilot, rows_mask=target,
                                         epochs=args.proposal_epochs, batch=args.proposal_batch,
                                         pilot_theta_deg=pilot_th) for _ in range(3)]
    order = sorted(range(3), key=lambda i: runs[i].pilot_s + runs[i].fit_s)
    tp = runs[order[1]]
    prop, r2 = tp.proposal, tp.fit_r2
    t_train = tp.pilot_s + tp.fit_s
    train_runs_s = [round(r.pilot_s + r.fit_s, 4) for r in runs]
    Ns = [1024, 2048, 4096, 8192]
    modes = ("plain_fp64", "plain_fp32c", "learned_fp32c", "learned_fp32c_with_pilot")
    if tp.pilot_rows is None:      # the pilot's rows are not the grid's: nothing to reuse
        modes = modes[:3]
    metrics_ = ("M11_rms_rel", "P_rms_abs")
    err = {m: {k: {q: [] for q in metrics_} for k in regions} for m in modes}
    for N in Ns:
        acc = {m: {k: {q: [] for q in metrics_} for k in regions} for m in modes}
        for seed in (1, 2, 3, 4):
            u, v, w = prop.sample(N, seed=seed)
            wp, wm = PR.balance_weights(prop, n_pilot, (tp.pilot_u, tp.pilot_v), (u, v))
            plain = PR.plain_sobol(N, seed=seed)
            for m, (uu, vv, ww), prec in (("plain_fp64", plain, abi.FP64),
                                          ("plain_fp32c", plain, abi.FP32C),
                                          ("learned_fp32c", (u, v, w), abi.FP32C),
                                          ("learned_fp32c_with_pilot", (u, v, wm), abi.FP32C)):
                if m not in modes:
                    continue
                r = rows_of(uu, vv, ww, prec)
                if m == "learned_fp32c_with_pilot":
                    r = r + np.tensordot(wp, tp.pilot_rows, axes=1)
                for k, mask in regions.items():
                    e = PR.row_errors(r, ref, mask)
                    for q in metrics_:
                        acc[m][k][q].append(e[q])
        for m in modes:
            for k in regions:
                for q in metrics_:
                    err[m][k][q].append(float(np.sqrt(np.mean(np.square(acc[m][k][q])))))

    def to_1pct(errs):
        b, a = np.polyfit(np.log(Ns), np.log(errs), 1)
        return (float(np.exp((np.log(0.01) - a) / b)) if b < 0 else float("inf")), float(b)

    proj = {}
    for k in regions:
        proj[k] = {}
        for m in modes:
            prec = "fp64" if m == "plain_fp64" else "fp32c"
            d = {}
            for q in metrics_:
                d[q + "_orientations_to_1pct"], d[q + "_slope"] = to_1pct(err[m][k][q])
            n_both = max(d["M11_rms_rel_orientations_to_1pct"], d["P_rms_abs_orientations_to_1pct"])
            extra = t_train if m.startswith("learned") else 0.0
            d["orientations_to_1pct_both"] = n_both
            d["wall_s_to_1pct_both"] = n_both * per_orient[prec] + extra
            proj[k][m] = d
        base = proj[k]["plain_fp64"]["wall_s_to_1pct_both"]
        for m in modes[1:]:
            proj[k]["speedup_" + m] = base / proj[k][m]["wall_s_to_1pct_both"]
    out = {"metric": "wall time to 1% on orientation-averaged M11 (RMS relative) and -M12/M11 "
                     "(RMS absolute), learned FP32C proposal vs plain FP64 Sobol",
           "unit": "s", "higher_is_better": False, "impl": "b200", "n_gpus": 1,
           "value": min(proj[args.proposal_rows][m]["wall_s_to_1pct_both"] for m in modes[2:]),
           "config": {"workload": "hexagonal column D=40um L=100um m=1.3116+1e-9i, 4 reflections; "
                                  "theta 0-180 step %.3g deg x %d phi; learned proposal (MLP "
                                  "4-128-128-128-1, BF16 tensor-core training) on the %s rows; "
                                  "4 scrambles per N" % (180.0 / args.n_theta, args.n_phi,
                                                         args.proposal_rows),
                      "orientations": Ns, "reference_orientations": 65536,
                      "pilot_orientations": n_pilot, "epochs": args.proposal_epochs,
                      "batch": args.proposal_batch,
                      "pilot_rows": (len(pilot_th) if pilot_th is not None else int(grid.n_zen + 1)),
                      "launch_shapes": st_best},
           "fit_r2": r2, "proposal_train_s": t_train, "pilot_s": tp.pilot_s, "fit_s": tp.fit_s,
           "proposal_parts_s": tp.parts,
           "proposal_train_runs_s": train_runs_s,
           "proposal_learned": bool(prop.learned),
           "predicted_variance_ratio": tp.variance_ratio,
           "reference_s": t_ref,
           "wall_s_per_orientation_with_tracing": per_orient,
           "errors": err, "to_1pct": proj}
    h.close()
    print(json.dumps(out), flush=True)


def run_aggregate(args):
    """Non-convex aggregate of 8 touching hexagonal columns (D=20 um, L=60 um,
    seed-drawn orientations), 6 reflections, importance cutoffs of 1e-4
    (tracing) and 1e-3 (beams) over the fast profile, 32,768 Sobol
    orientation evaluations per step on the headline grid in ONE persistent
    graph-captured diffraction launch, FP32C and FP64.  Host tracing of
    32,768 distinct aggregate orientations takes minutes on the host cores,
    so --aggregate-distinct Sobol orientations are traced and staged once
    and the step's orientation table (mbs_po_stage_repeat) cycles over them
    with weight 1/N each: the device does the work of N orientations with the
    distinct orientations' beam counts."""
    import dataclasses
    import tempfile
    import torch
    from mbs_fast_b200 import abi, beams as B, metrics, workloads as W
    from mbs_fast_b200.handler import GpuHandlerPO
    torch.cuda.set_device(0)
    n = args.orient if args.orient != 16384 else 32768
    distinct = min(n, args.aggregate_distinct)
    path = os.path.join(tempfile.mkdtemp(), "agg8.particle")
    cfg = dataclasses.replace(W.aggregate_config(path), trace_cutoff_importance=1e-4,
                              beam_cutoff_importance=1e-3)
    bs, gs, _ = B.symmetry(cfg)
    beta, gamma, w = B.sobol_orientations(n, bs, gs, 42)
    t0 = time.perf_counter()
    batch = B.trace(cfg, beta[:distinct], gamma[:distinct], w[:distinct])
    t_trace = time.perf_counter() - t0
    grid = B.grid(0.0, 180.0, args.n_phi, args.n_theta)
    G = grid.n_dirs
    h = GpuHandlerPO(grid, B.wave(cfg))
    src = h.stage(batch)
    idx = np.arange(n) % distinct
    st = h.stage_repeat(src, idx, np.full(n, 1.0 / n))
    bpo = np.diff(batch.beam_offsets)
    beam_dirs = float(bpo[idx].sum()) * G
    acc = torch.zeros(G * 16, dtype=torch.float64, device="cuda:0")
    s = torch.cuda.Stream()
    out, planes = {}, {}
    for prec, name, steps in ((abi.FP32C, "fp32c", args.steps), (abi.FP64, "fp64", 1)):
        best, ms = h.autotune(src, prec, max_orient=min(64, distinct))
        with torch.cuda.stream(s):
            h.diffract_staged(st, acc.data_ptr(), precision=prec, stream=s.cuda_stream, stats=False)
        s.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            acc.zero_()
            h.diffract_staged(st, acc.data_ptr(), precision=prec, stream=s.cuda_stream, stats=False)
        g.replay()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            g.replay()
        e1.record()
        torch.cuda.synchronize()
        ms_step = e0.elapsed_time(e1) / steps
        planes[name] = acc.cpu().numpy().reshape(grid.n_az, grid.n_zen + 1, 16)
        out[name] = {"ms_per_step": ms_step, "steps": steps,
                     "orientations_per_s": n / (ms_step * 1e-3),
                     "beam_dir_evals_per_s": beam_dirs / (ms_step * 1e-3),
                     "autotune": {"variant": best, "ms_per_variant": [round(m, 3) for m in ms]}}
        del g
    errs = metrics.compare(h, planes["fp32c"], planes["fp64"])
    st.free()
    src.free()
    h.close()
    line = {"metric": METRIC, "value": out["fp32c"]["orientations_per_s"], "unit": "orientations/s",
            "impl": "b200", "n_gpus": 1, "steps": args.steps, "warmup": 1,
            "higher_is_better": True, "dtype": "f32+f64", "data": "synthetic (reference tracer)",
            "config": {"workload": "non-convex aggregate of 8 hexagonal columns D=20um L=60um, "
                                   "m=1.3116, 6 reflections, cutoff profile fast with importance "
                                   "cutoffs 1e-4 (trace) / 1e-3 (beams), %d Sobol orientation "
                                   "evaluations per step (%d distinct traced orientations cycled), "
                                   "theta 0-180 step %.3g x %d phi; one graph-captured persistent "
                                   "launch per step" % (n, distinct, 180.0 / args.n_theta, args.n_phi),
                       "beams_per_orientation": [int(bpo.min()), int(bpo.max()), float(bpo.mean())],
                       "trace_seconds": t_trace, "distinct_orientations": distinct},
            "fp32c": out["fp32c"], "fp64": out["fp64"],
            "fp32c_speedup_vs_fp64": out["fp64"]["ms_per_step"] / out["fp32c"]["ms_per_step"],
            "fp32c_error_vs_fp64": errs,
            "host_trace_orientations_per_s": distinct / t_trace}
    print(json.dumps(line), flush=True)


def run_fftphi(args):
    """FFT-phi path on the headline column and grid: the direct evaluation on
    n_phi / factor azimuth bins plus the device interpolation to n_phi bins,
    against the direct evaluation on n_phi bins, both FP32C with
    device-resident inputs (2048 Sobol orientations unless --orient is
    given).  Reports the time per step of each and the interpolation error
    of the azimuth-averaged rows and of the grid against the direct result."""
    import torch
    from mbs_fast_b200 import abi, beams as B
    from mbs_fast_b200 import metrics, workloads as W
    from mbs_fast_b200.handler import GpuHandlerPO
    torch.cuda.set_device(0)
    n = args.orient if args.orient != 16384 else 2048
    cfg = W.COLUMN_40x100
    bs, gs, _ = B.symmetry(cfg)
    beta, gamma, w = B.sobol_orientations(n, bs, gs, 42)
    batch = B.trace(cfg, beta, gamma, w)
    full = B.grid(0.0, 180.0, args.n_phi, args.n_theta)
    factor = GpuHandlerPO.fft_phi_factor(full.n_az)
    n_low = max(full.n_az // factor, min(full.n_az, 16))
    low = full.with_azimuths(n_low)
    rows = full.n_zen + 1
    hf, hl = GpuHandlerPO(full, B.wave(cfg)), GpuHandlerPO(low, B.wave(cfg))
    sf, sl = hf.stage(batch), hl.stage(batch)
    acc_f = torch.zeros(full.n_dirs * 16, dtype=torch.float64, device="cuda:0")
    acc_l = torch.zeros(low.n_dirs * 16, dtype=torch.float64, device="cuda:0")
    acc_i = torch.zeros_like(acc_f)
    hf.autotune(sf, abi.FP32C)
    hl.autotune(sl, abi.FP32C)

    def direct():
        acc_f.zero_()
        hf.diffract_staged(sf, acc_f.data_ptr(), precision=abi.FP32C, stats=False)

    def fft():
        acc_l.zero_()
        acc_i.zero_()
        hl.diffract_staged(sl, acc_l.data_ptr(), precision=abi.FP32C, stats=False)
        hl.phi_interpolate(acc_l.data_ptr(), n_low, rows, acc_i.data_ptr(), full.n_az)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / args.steps

    ms_direct, ms_fft = timed(direct), timed(fft)
    Md = acc_f.cpu().numpy().reshape(full.n_az, rows, 16)
    Mi = acc_i.cpu().numpy().reshape(full.n_az, rows, 16)
    errs = metrics.compare(hf, Mi, Md)
    errs["L2_grid"] = float(np.sqrt(np.sum((Mi - Md) ** 2) / max(np.sum(Md ** 2), 1e-300)))
    for s_ in (sf, sl):
        s_.free()
    hf.close()
    hl.close()
    line = {"metric": METRIC, "value": n / (ms_fft * 1e-3), "unit": "orientations/s",
            "impl": "b200", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "dtype": "f32+f64", "data": "synthetic (reference tracer)",
            "config": {"workload": WORKLOAD.replace("16384", str(n)) + "; FFT-phi: direct on %d "
                                   "azimuth bins, interpolated to %d" % (n_low, full.n_az),
                       "factor": factor},
            "fft_phi_ms_per_step": ms_fft, "direct_ms_per_step": ms_direct,
            "speedup_vs_direct": ms_direct / ms_fft,
            "interpolation_error_vs_direct": errs}
    print(json.dumps(line), flush=True)


def run_sizescan(args):
    """Size scan on the device (the multi-size path): 16 plates L = 0.2 D, D
    log-spaced 10-200 um, m = 1.3116, 4 reflections, Sobol orientations
    traced once at D = 10 um and rescaled on the device for every size, on
    the non-uniform zenith grid (0.05 deg to 10 deg, 0.5 deg beyond: 541
    rows) x 48 azimuth bins; one launch for all sizes per step, FP32C and
    FP64, device-resident inputs (4096 orientations unless --orient is
    given).  Reports (size, orientation) pairs per second and the FP32C
    error against FP64 on the largest size."""
    import torch
    from mbs_fast_b200 import abi, beams as B
    from mbs_fast_b200 import metrics, workloads as W
    from mbs_fast_b200.handler import GpuHandlerPO
    torch.cuda.set_device(0)
    n = args.orient if args.orient != 16384 else 4096
    cfg = W.PLATE_D10
    bs, gs, _ = B.symmetry(cfg)
    beta, gamma, w = B.sobol_orientations(n, bs, gs, 42)
    batch = B.trace(cfg, beta, gamma, w)
    grid = B.grid(0.0, 180.0, args.n_phi, 0, theta_deg=W.size_scan_theta_deg())
    scales = W.size_scan_diameters() / 10.0
    h = GpuHandlerPO(grid, B.wave(cfg))
    st = h.stage_multisize(batch, scales)
    plane = grid.n_dirs * 16
    acc = torch.zeros(len(scales) * plane, dtype=torch.float64, device="cuda:0")
    out = {}
    planes = {}
    for prec, name in ((abi.FP32C, "fp32c"), (abi.FP64, "fp64")):
        best, ms = h.autotune(st, prec, max_orient=min(256, n))
        for _ in range(args.warmup):
            acc.zero_()
            h.diffract_staged(st, acc.data_ptr(), precision=prec, stats=False)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            acc.zero_()
            h.diffract_staged(st, acc.data_ptr(), precision=prec, stats=False)
        e1.record()
        torch.cuda.synchronize()
        ms_step = e0.elapsed_time(e1) / args.steps
        pairs = n * len(scales)
        out[name] = {"ms_per_step": ms_step, "size_orientations_per_s": pairs / (ms_step * 1e-3),
                     "beam_dir_evals_per_s": batch.n_beams * len(scales) * grid.n_dirs / (ms_step * 1e-3),
                     "autotune": {"variant": best, "ms_per_variant": [round(m, 3) for m in ms]}}
        planes[name] = acc.cpu().numpy().reshape(len(scales), grid.n_az, grid.n_zen + 1, 16)
    errs = metrics.compare(h, planes["fp32c"][-1], planes["fp64"][-1])
    st.free()
    h.close()
    line = {"metric": METRIC, "value": out["fp32c"]["size_orientations_per_s"],
            "unit": "(size, orientation) pairs/s", "impl": "b200", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "dtype": "f32+f64", "data": "synthetic (reference tracer)",
            "config": {"workload": "size scan: 16 plates L=0.2D, D 10-200 um log-spaced, m=1.3116, "
                                   "4 reflections, %d Sobol orientations traced at D=10 um and "
                                   "rescaled per size, 541 zenith rows (0.05 deg to 10, 0.5 deg "
                                   "beyond) x %d phi; one launch per step" % (n, args.n_phi),
                       "beams_per_size": batch.n_beams, "directions": grid.n_dirs},
            "fp32c": out["fp32c"], "fp64": out["fp64"],
            "fp32c_error_vs_fp64_largest_size": errs}
    print(json.dumps(line), flush=True)


REFGPU_BINARIES = {
    "reference_fp64": ("oracle/_ref/mbs_po_gpu_ref_fp64", {}),
    "reference_fp32": ("oracle/_ref/mbs_po_gpu_ref_fp32", {}),
    "b200_fp64": ("mbs_fast_b200/_lib/mbs_po_b200", {"MBS_B200_PRECISION": "fp64"}),
    "b200_fp32c": ("mbs_fast_b200/_lib/mbs_po_b200", {"MBS_B200_PRECISION": "fp32c"}),
}


def reference_gpu_compare(n: int, n_phi: int, n_theta: int, warm: bool = True) -> dict:
    """Same-box GPU comparison at the CLI: the reference's own CUDA build
    (its GpuDiffraction.cu for sm_100, FP64 and FP32) against the drop-in
    binary (the same CLI with this library underneath, FP64 and FP32C), on
    the D=40 um, L=100 um column with n Sobol orientations.  Per binary: the
    sums of the "GPU timing diffract" lines (MBS_GPU_TIMING=1) of a run,
    kernels and whole calls (packing, copies, kernels, accumulation), and the
    process wall time, each the median of three runs; with `warm`, after one
    untimed run (the first process on a fresh device pays one-off costs)."""
    import re
    import tempfile
    cli = ["--method", "po", "--particle", "1", "100", "40", "--refractive-index", "1.3116", "1e-9",
           "--wavelength-um", "0.532", "--max-reflections", "4", "--sobol", str(n),
           "--scattering-grid", "0", "180", str(n_phi), str(n_theta), "--close",
           "--backend", "gpu"]
    out = {}
    for name, (rel, env_extra) in REFGPU_BINARIES.items():
        binary = os.path.join(ROOT, rel)
        if not os.path.exists(binary):
            out[name] = {"unavailable": "not built"}
            continue
        env = dict(os.environ, MBS_GPU_TIMING="1", **env_extra)
        if warm:
            subprocess.run([binary] + cli + ["--output", os.path.join(tempfile.mkdtemp(), "w")],
                           capture_output=True, text=True, env=env, timeout=1800)
        # three timed runs, the median of each figure: single runs on the
        # shared host show stalls of hundreds of ms in either binary
        runs = []
        for _ in range(3):
            d = tempfile.mkdtemp()
            t0 = time.perf_counter()
            r = subprocess.run([binary] + cli + ["--output", os.path.join(d, "o")], capture_output=True,
                               text=True, env=env, timeout=1800)
            wall = time.perf_counter() - t0
            text = r.stdout + r.stderr
            lines = [ln for ln in text.splitlines() if "GPU timing diffract" in ln]
            kern = sum(float(m) for ln in lines for m in re.findall(r"kernels=([0-9.]+)ms", ln))
            tot = sum(float(m) for ln in lines for m in re.findall(r"total=([0-9.]+)ms", ln))
            runs.append((r.returncode, len(lines), kern, tot, wall))
        out[name] = {"rc": max(x[0] for x in runs), "calls": runs[0][1],
                     "kernel_ms": float(np.median([x[2] for x in runs])),
                     "call_ms": float(np.median([x[3] for x in runs])),
                     "process_wall_s": float(np.median([x[4] for x in runs])),
                     "runs": 3}
    for prec, ref, mine in (("fp64", "reference_fp64", "b200_fp64"), ("fp32", "reference_fp32", "b200_fp32c")):
        a, b = out.get(ref, {}), out.get(mine, {})
        if a.get("kernel_ms") and b.get("kernel_ms"):
            out[prec + "_kernel_speedup"] = a["kernel_ms"] / b["kernel_ms"]
        if a.get("call_ms") and b.get("call_ms"):
            out[prec + "_call_speedup"] = a["call_ms"] / b["call_ms"]
        if a.get("process_wall_s") and b.get("process_wall_s"):
            out[prec + "_process_speedup"] = a["process_wall_s"] / b["process_wall_s"]
    return out


def run_refgpu(args):
    """reference_gpu_compare as its own workload (2048 orientations unless
    --orient is given)."""
    n = args.orient if args.orient != 16384 else 2048
    line = {"metric": METRIC, "unit": "orientations/s", "impl": "b200-vs-reference-gpu",
            "config": {"workload": WORKLOAD.replace("16384", str(n)), "orientations": n},
            "runs": reference_gpu_compare(n, args.n_phi, args.n_theta)}
    print(json.dumps(line), flush=True)


def run_mlp(args):
    """The proposal network's kernels alone: Adam training on 8192 seeded unit
    quaternions (2 epochs, batches of 2048) and one forward pass over them."""
    from mbs_fast_b200.mlp import ProposalNet
    rng = np.random.default_rng(0)
    q = rng.normal(size=(8192, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    t = np.sin(3 * q[:, 0]) + q[:, 1] * q[:, 2]
    net = ProposalNet(seed=1)
    t0 = time.perf_counter()
    loss = net.train(q, t, epochs=2, batch=2048, lr=2e-3)
    t1 = time.perf_counter()
    net.forward(q)
    t2 = time.perf_counter()
    net.close()
    print(json.dumps({"workload": "proposal network 4-128-128-128-1, BF16 tcgen05", "train_s": t1 - t0,
                      "forward_s": t2 - t1, "loss": loss}), flush=True)


# DRAM bytes (ncu dram__bytes_read.sum + dram__bytes_write.sum) of one
# full-size FP32C diffraction launch of the headline workload (16,384
# orientations), from the capture summarised in
# profiles/po_diffract_kernel_f32_traffic_hexcol40x100_16384orient.md
FP32C_LAUNCH_DRAM_BYTES = 1_571_426_560 + 2_719_601_664


def nominal_peaks(clock_mhz: float | None) -> dict:
    """B200 nominal FP32 and FP64 FMA peaks at the given SM clock: 148 SMs x
    128 FP32 lanes (64 FP64 lanes) x 2 flop."""
    f = (clock_mhz or 1965.0) * 1e6
    return {"fp32_tflops": 148 * 128 * 2 * f / 1e12, "fp64_tflops": 148 * 64 * 2 * f / 1e12,
            "sm_mhz": clock_mhz or 1965.0}


def launch_ranks(args) -> int:
    """--gpus N without a torchrun environment: run this script once per GPU
    under torch.distributed.run (one process per GPU, rendezvous on
    127.0.0.1) with the same arguments; rank 0 prints the line."""
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={args.gpus}", "--master-addr=127.0.0.1", f"--master-port={port}",
           os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def run_launch_selftest(args):
    """Ranks started by launch_ranks check their environment and exchange one
    all-reduce (gloo on the CPU): the multi-process plumbing of --gpus N
    without a GPU."""
    import datetime
    import torch
    import torch.distributed as dist
    rank, world, local = dist_env()
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    t = torch.tensor([float(rank + 1)])
    dist.all_reduce(t)
    mx = torch.tensor([float(rank)])
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    dist.destroy_process_group()
    if rank == 0:
        print(json.dumps({"launch_selftest": True, "world": world, "sum": float(t.item()),
                          "max_rank": float(mx.item()), "gpus_arg": args.gpus}), flush=True)


def main():
    args = parse()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(launch_ranks(args))
    if args.launch_selftest:
        run_launch_selftest(args)
        return
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload == "proposal":
        run_proposal(args)
        return
    if args.workload == "aggregate":
        run_aggregate(args)
        return
    if args.workload == "sizescan":
        run_sizescan(args)
        return
    if args.workload == "fftphi":
        run_fftphi(args)
        return
    if args.workload == "refgpu":
        run_refgpu(args)
        return
    if args.workload == "mlp":
        run_mlp(args)
        return
    rank, world, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from mbs_fast_b200 import abi, metrics
    from mbs_fast_b200.handler import GpuHandlerPO

    t0 = time.perf_counter()
    cfg, batch, grid, wave, orients = build_inputs(args, rank, world)
    t_trace = time.perf_counter() - t0
    G = grid.n_dirs
    h = GpuHandlerPO(grid, wave, device=local)
    staged = h.stage(batch)
    acc = torch.zeros(G * 16, dtype=torch.float64, device=f"cuda:{local}")
    stream = torch.cuda.current_stream().cuda_stream

    # launch-shape autotuner on a slice of the batch (untimed)
    tuned = {}
    for prec, name in ((abi.FP32C, "fp32c"), (abi.FP64, "fp64")):
        if args.no_autotune:
            tuned[name] = {"variant": 0, "ms_per_variant": None}
            continue
        best, ms = h.autotune(staged, prec, max_orient=min(256, batch.n_orient))
        tuned[name] = {"variant": best, "ms_per_variant": [round(m, 3) for m in ms]}
    # plain FP64 batched path: the error reference and the denominator of
    # the wall-time comparison (one full pass, device-timed)
    fp64_ms = fp64_kernel_ms = None
    M64 = None
    if not args.no_fp64:
        ref = torch.zeros_like(acc)
        st = abi.Stats()
        h.diffract_staged(staged, ref.data_ptr(), precision=abi.FP64, stream=stream, stats=st)
        if world > 1:        # the whole job's sums, like the FP32C steps'
            torch.distributed.all_reduce(ref)
        torch.cuda.synchronize()
        fp64_ms = st.kernel_ms + st.reduce_ms
        fp64_kernel_ms = st.kernel_ms
        M64 = ref.cpu().numpy().reshape(grid.n_az, grid.n_zen + 1, 16)
        del ref

    stats = abi.Stats()
    for _ in range(args.warmup):
        acc.zero_()
        h.diffract_staged(staged, acc.data_ptr(), precision=abi.FP32C, stream=stream, stats=stats)
    torch.cuda.synchronize()

    # ---- timed region: device-resident (value) ----
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    kernel_ms = []
    launches = 0
    ev0.record()
    for _ in range(args.steps):
        acc.zero_()
        h.diffract_staged(staged, acc.data_ptr(), precision=abi.FP32C, stream=stream, stats=stats)
        kernel_ms.append(stats.kernel_ms)
        launches += stats.launches + 1      # diffraction + reduce (+ pole rows), + the accumulator clear
        if world > 1:
            # the path's one exchange: the sum of the ranks' Mueller accumulators
            torch.distributed.all_reduce(acc)
    ev1.record()
    torch.cuda.synchronize()
    step_ms = ev0.elapsed_time(ev1) / args.steps
    clocks = sampler.stop()
    if world > 1:
        t = torch.tensor([step_ms], device=f"cuda:{local}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        step_ms = float(t.item())
    M32 = acc.cpu().numpy().reshape(grid.n_az, grid.n_zen + 1, 16)

    # ---- timed region: end-to-end through the public C ABI, every step ----
    pinned = pin_batch(batch)
    Mh = np.zeros((grid.n_az, grid.n_zen + 1, 16))
    h.handle_orientations_to_local_gpu(pinned, Mh, precision=abi.FP32C)   # warm
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    e2e_t = []
    for _ in range(args.steps):
        Mh[:] = 0.0
        t1 = time.perf_counter()
        h.handle_orientations_to_local_gpu(pinned, Mh, precision=abi.FP32C)
        if world > 1:
            # the ranks' host sums, added over NCCL (up and back down)
            red = torch.from_numpy(Mh).to(f"cuda:{local}")
            torch.distributed.all_reduce(red)
            Mh[...] = red.cpu().numpy()
        e2e_t.append(time.perf_counter() - t1)
    e2e_s = float(np.mean(e2e_t))
    if world > 1:
        t = torch.tensor([e2e_s], device=f"cuda:{local}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_s = float(t.item())
    h2d_bytes = int(sum(a.nbytes for a in (pinned.beam_offsets, pinned.orient_weight,
                                          pinned.vert_offsets, pinned.vx, pinned.vy,
                                          pinned.slope_yx, pinned.slope_xy, pinned.edge_flags,
                                          pinned.beam_geom, pinned.beam_flags)))
    d2h_bytes = G * 16 * 8
    if world > 1:              # the reduction's round trip
        h2d_bytes += G * 16 * 8
        d2h_bytes += G * 16 * 8

    # ---- the whole orientation average: host tracing overlapped with the device ----
    from mbs_fast_b200.pipeline import orientation_average
    beta_o, gamma_o, w_o = orients
    # one short untimed pass first (thread pools, pinned buffers), then the
    # whole average in batches of 1024
    orientation_average(h, cfg, beta_o[:2048], gamma_o[:2048], w_o[:2048], precision=abi.FP32C,
                        batch=1024)
    # five passes, the median wall time: single passes on the shared host
    # showed stalls of up to a second while the tracer's time was unchanged
    passes = [orientation_average(h, cfg, beta_o, gamma_o, w_o, precision=abi.FP32C, batch=1024)[2]
              for _ in range(5)]
    tp = sorted(passes, key=lambda x: x["wall_s"])[2]
    trace_wall = tp["wall_s"]
    if world > 1:
        t = torch.tensor([trace_wall], device=f"cuda:{local}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        trace_wall = float(t.item())

    # ---- error of FP32C against the plain FP64 path on the same orientations ----
    m11_err = metrics.compare(h, M32, M64) if M64 is not None else None

    flops = algorithmic_flops(batch, G)
    kern_s = float(np.mean(kernel_ms)) * 1e-3
    peak = h.probe_fp32_peak()
    peak64 = h.probe_fp64_peak()
    nom = nominal_peaks(clocks.get("sm_mhz"))
    achieved = flops / kern_s / 1e12
    total_orient = batch.n_orient * world
    value = total_orient / (step_ms * 1e-3)
    # the capture's figure holds for the headline batch only
    traffic = FP32C_LAUNCH_DRAM_BYTES if (batch.n_orient == 16384 and G == 48 * 1801) else None
    roofline = {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak if peak else None,
                "traffic": traffic,
                "traffic_unit": "bytes per launch (ncu DRAM read + write)",
                "algorithmic_bytes": int(batch.n_beams * 432 + batch.n_verts * 48 + G * 16 * 8),
                "peak_source": "measured FFMA probe of this device (MEASURED_PEAKS.json has no FP32 entry)",
                "nominal_peak": nom["fp32_tflops"], "frac_of_nominal": achieved / nom["fp32_tflops"],
                "work": "12*nv+168 flop per beam-direction + 100 per orientation-direction"}
    if fp64_kernel_ms:
        a64 = flops / (fp64_kernel_ms * 1e-3) / 1e12
        roofline["fp64"] = {"kernel": "po_diffract_kernel<double> (plain FP64 path)", "achieved": a64,
                            "peak": peak64, "frac": a64 / peak64 if peak64 else None,
                            "nominal_peak": nom["fp64_tflops"],
                            "frac_of_nominal": a64 / nom["fp64_tflops"],
                            "peak_source": "measured DFMA probe of this device"}
    line = {
        "metric": METRIC, "value": value, "unit": "orientations/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic (beams from the reference's own tracer, no data set)",
        "config": {"workload": WORKLOAD, "orientations_per_gpu": batch.n_orient,
                   "beams": batch.n_beams, "vertices": batch.n_verts, "directions": G,
                   "precision": "fp32c (FP32 trig/MAC, FP64 phase+reduction, Kahan Jones sums)",
                   "l2": "inputs larger than L2 (%.0f MB resident)" % ((batch.n_beams * 288 + batch.n_verts * 32) / 1e6),
                   "trace_seconds": t_trace},
        "beam_dir_evals_per_s": batch.n_beams * world * G / (step_ms * 1e-3),
        "m11_error_vs_fp64": m11_err,
        "fp64_ms_per_step": fp64_ms,
        "fp64_orientations_per_s": (batch.n_orient / (fp64_ms * 1e-3)) if fp64_ms else None,
        "fp32c_speedup_vs_fp64": (fp64_ms / step_ms) if fp64_ms else None,
        "e2e": {"value": total_orient / e2e_s, "unit": "orientations/s",
                "h2d_bytes_per_step": h2d_bytes, "d2h_bytes_per_step": d2h_bytes,
                "timed_calls": len(e2e_t)},
        "e2e_with_tracing": {"value": total_orient / trace_wall, "unit": "orientations/s",
                             "wall_s": trace_wall, "host_trace_s": tp["trace_s"],
                             "passes_wall_s": [round(x["wall_s"], 4) for x in passes],
                             "what": "reference tracer and restated PrepareBeams on all host "
                                     "cores but one (which stages the batches), batches of 1024, "
                                     "overlapped with FP32C diffraction on the device; the median "
                                     "of five passes"},
        "gpu_launches": launches,
        "autotune": tuned,
        "roofline": roofline,
        "clocks": clocks,
    }
    if rank == 0 and not args.no_cpu:
        base, M_ref, cext_ref, sample = reference_sample(cfg, batch, args)
        line["cpu_baseline"] = base
        line["parity_vs_reference"] = parity_vs_reference(h, sample, M_ref, cext_ref)
    staged.free()
    h.close()
    # the reference's CUDA CLI splits a call over every visible device: only
    # the one-GPU line compares with it
    if rank == 0 and world == 1 and not args.no_refgpu:
        line["reference_gpu"] = reference_gpu_compare(args.refgpu_orient, args.n_phi, args.n_theta)
    if world > 1:
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def pin_batch(batch):
    """Copy the batch's arrays into page-locked host memory."""
    import torch
    from mbs_fast_b200.beams import BeamBatch

    def pin(a):
        t = torch.empty(a.shape, dtype=getattr(torch, str(a.dtype)), pin_memory=True)
        n = t.numpy()
        n[...] = a
        return n
    return BeamBatch(beam_offsets=pin(batch.beam_offsets), orient_weight=pin(batch.orient_weight),
                     vert_offsets=pin(batch.vert_offsets), vx=pin(batch.vx), vy=pin(batch.vy),
                     slope_yx=pin(batch.slope_yx), slope_xy=pin(batch.slope_xy),
                     edge_flags=pin(batch.edge_flags), beam_geom=pin(batch.beam_geom),
                     beam_flags=pin(batch.beam_flags))


if __name__ == "__main__":
    main()
