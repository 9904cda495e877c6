"""Benchmark: ms per UPDC iteration on the 8 x 2048^2 -> 4096^2 workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload c1] [--form fp32|fp64|fp32-kahan|fp32-reference]

A step is one iteration of the solver (updc/c_core/updc_core.c:1410-1456) on
the workload's synthetic inputs, with everything already resident on the GPU.
``value`` is the device time per iteration (CUDA events on the engine's
stream, max over ranks), ``e2e`` the same through the public C ABI with the
estimate uploaded from and read back to host memory every step.  The per-stage
event timing pass gives the dominant kernel's roofline.  ``--impl reference``
times the reference core itself (compiled from its sources with the FFTW-API
shim, oracle/_ref) on the host cores for the same workload.
Under torchrun (N > 1) the field's exposures are split over the ranks: each
rank computes the partial correction of its exposures, one NCCL all-reduce
sums them and every rank applies the same update (strong scaling; --replicas
runs N independent copies instead).  ``--workload c2`` runs 64 batched
cutout fields, every stage one persistent launch over all fields.
``--workload pre`` times the per-exposure weight preprocessing (sigma-clipped
sky, weights, pedestals, WHT; updc/_engine.py:287-408) of the c1 exposures.
"""
from __future__ import annotations

import argparse
import csv
import json
import math
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))


# ----------------------------------------------------------------------------- helpers
def env_rank():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.is_file():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def stage_bytes(w, fw, fh, links, tlinks, dtype_bytes=4):
    """Algorithmic bytes of each kernel of one iteration (each input read once,
    each output written once; complex = 2 x dtype_bytes)."""
    N, W, H, nin, nout = w.nexp, w.W, w.H, w.iw * w.ih, w.W * w.H
    M1 = fw // 2 + 1
    c = 2 * dtype_bytes
    spec_h = M1 * H * c          # a row-pass intermediate (u-major, H rows)
    spec_f = M1 * fh * c         # a full spectrum (PSF OTF)
    r = dtype_bytes
    link_bytes = sum(4 * (nin + 1) + (4 * nin + 2 * L + (2 * L) % 4 if enc == 2 else 4 * L) + 4 * L
                     for L, enc in links)
    tmap_bytes = sum(4 * (nout + 1) + 8 * L for L in tlinks)
    return {
        "estimate_x_pass": nout * r + spec_h,
        "forward_y_passes": spec_h + N * spec_f + N * spec_h,
        "forward_x_pass": N * spec_h + N * nout * r,
        "detector": link_bytes + N * (nin * r * 3 + nin * 2) + N * nout * r,
        "adjoint_gather": tmap_bytes + N * nin * r + N * nout * r,
        "scatter_x_pass": N * (nout * r + spec_h),
        "adjoint_y_x_passes": N * spec_h + N * spec_f + spec_h + spec_h + nout * r,
        "update": 4 * nout * r,
    }


def model_bytes(w, fw, fh, links, dtype_bytes=4):
    """Algorithmic bytes of each stage under the path's stated model: every
    2-D FFT is two passes, each reading and writing the full FH x (FW/2+1)
    spectrum Sc (so 2 Sc per pass), an OTF read is Sc, the cross-exposure
    accumulator is read and written once per exposure (2 Sc), the detector
    loop reads its LinkMap, SCI, W, the mask and blur_k, and the scatter plane
    is written once (St).  The engine itself moves fewer bytes (the zero
    padding of the passes is never stored, the accumulator stays on chip or in
    L2): `stage_bytes` is that tighter count."""
    N, nin, nout = w.nexp, w.iw * w.ih, w.W * w.H
    c, r = 2 * dtype_bytes, dtype_bytes
    Sc = (fw // 2 + 1) * fh * c
    St, Sd = nout * r, nin * r
    link_bytes = sum(4 * (nin + 1) + (4 * nin + 2 * L + (2 * L) % 4 if enc == 2 else 4 * L) + 4 * L
                     for L, enc in links)
    return {
        "estimate_x_pass": 2 * Sc,
        "forward_y_passes": 2 * Sc + N * 3 * Sc,
        "forward_x_pass": N * 2 * Sc,
        "detector": link_bytes + N * (2 * Sd + nin + St),
        "adjoint_gather": N * St,
        "scatter_x_pass": N * 2 * Sc,
        "adjoint_y_x_passes": N * 5 * Sc + 4 * Sc,
        "update": 4 * St,
    }


# DRAM bytes (read + write) over the bytes each kernel must move, per
# stage, from the full-set ncu capture of the same kernels on the c1
# geometry with 2 exposures (profiles/kernels_c1x2_fp32_fullset.md): the
# kernels' traffic grows in proportion to the rows, columns and exposures
# they process, so this ratio carries the small case to the benchmark.
TRAFFIC_RATIO_C1X2 = {"estimate_x_pass": 120.8 / 149.7, "forward_y_passes": 514.8 / 451.0,
                      "forward_x_pass": 263.1 / 299.4, "detector": 759.5 / 771.6,
                      "gather_scatter_x_pass": 949.9 / 936.8,
                      "adjoint_y_x_passes": (620.8 + 114.0) / (451.0 + 149.7), "update": 214.2 / 268.4}

STAGES = ["estimate_x_pass", "forward_y_passes", "forward_x_pass", "detector", "adjoint_gather",
          "scatter_x_pass", "adjoint_y_x_passes", "update"]
STAGE_LAUNCHES = {"estimate_x_pass": 1, "forward_y_passes": 1, "forward_x_pass": 1, "detector": 1,
                  "adjoint_gather": 1, "scatter_x_pass": None, "adjoint_y_x_passes": 2, "update": 2}


# ----------------------------------------------------------------------------- reference arm
def reference_arm(args, rank, world):
    if rank != 0:
        return 0
    if args.workload == "pre":
        cpu = preprocess_cpu_sample(_pre_exposures(), limit_s=40.0)
        print(json.dumps({"impl": "reference", "metric": "ms/exposure (weight preprocessing)", "value": cpu["value"],
                          "unit": "ms", "higher_is_better": False, "n_gpus": world, "steps": args.steps,
                          "warmup": args.warmup, "config": {"workload": "pre", "shape": list(PRE_SHAPE)},
                          "cpu_baseline": cpu, "e2e": {"value": cpu["value"], "unit": "ms",
                                                       "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return 0
    from oracle import oracle as O
    from updc_b200 import synth
    if not O.REF_BINARY.is_file():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/updc_jwst_c was not built"}))
        return 0
    cores = os.cpu_count() or 1
    w = synth.WORKLOADS[args.workload]
    workdir = Path(tempfile.mkdtemp(prefix="updc_bench_ref_"))
    try:
        ds = synth.generate(w.name, workdir)
        # bounded sample: time one iteration first, then as many as fit ~150 s
        fftw = max(1, cores // w.nexp)
        def run(iters, prefix):
            a = ds.engine_args(iterations=iters, prefix=prefix, fft_workers=fftw, exposure_workers=w.nexp,
                               preprocess_workers=w.nexp).argv()
            t0 = time.time()
            r = subprocess.run([str(O.REF_BINARY), *a], capture_output=True, text=True,
                               env={**os.environ, "UPDC_PERSIST_CACHE": "1"})
            if r.returncode:
                raise RuntimeError(r.stderr[-400:])
            rows = list(csv.reader(open(f"{ds.directory}/{prefix}_timing.csv")))
            its = [float(v) for k, v in rows[1:] if k.endswith("_total") and k.startswith("iteration_")]
            return its, time.time() - t0
        first, wall = run(1, "probe")       # also fills the reference's persistent caches
        per = first[0]
        total = args.warmup + args.steps
        budget = max(1, int(150.0 / max(per, 1e-3)))
        n = min(total, budget)
        its, wall2 = run(n, "ref")
        timed = its[min(args.warmup, n - 1):] if n > 1 else its
        ms = 1000.0 * sum(timed) / len(timed)
        sample = (f"{len(timed)} timed of {n} reference-core iterations on {args.workload} "
                  f"({w.nexp}x{w.iw}x{w.ih} -> {w.W}x{w.H}), warm cache, fft_workers={fftw}, "
                  f"exposure_workers={w.nexp}; FFT = project FFTW-API shim (FFTW3f absent)")
        line = {"metric": "ms/iteration", "value": round(ms, 3), "unit": "ms", "n_gpus": world,
                "steps": len(timed), "warmup": args.warmup, "ms_per_step": round(ms, 3),
                "higher_is_better": False, "impl": "reference", "dtype": "f32", "data": "synthetic",
                "config": {"workload": args.workload, "target": [w.W, w.H], "exposures": w.nexp,
                           "detector": [w.iw, w.ih], "psf": w.psf_size},
                "cpu_baseline": {"value": round(ms, 3), "unit": "ms", "cores": cores, "kind": "reference",
                                 "sample": sample},
                "e2e": {"value": round(ms, 3), "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
    finally:
        shutil.rmtree(workdir, ignore_errors=True)
    return 0


# ----------------------------------------------------------------------------- b200 arm
def cufft_reference(torch, w, fw, fh, reps=5):
    """Device time of cuFFT (torch.fft) for one padded R2C of a W x H plane and
    one C2R with crop, on the FFT grid the engine uses."""
    x = torch.randn((w.H, w.W), device="cuda", dtype=torch.float32)
    pad = torch.zeros((fh, fw), device="cuda", dtype=torch.float32)
    spec = torch.fft.rfft2(pad)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    for _ in range(2):
        pad[:w.H, :w.W] = x
        spec = torch.fft.rfft2(pad)
        _ = torch.fft.irfft2(spec, s=(fh, fw))[:w.H, :w.W].contiguous()
    torch.cuda.synchronize()
    ev[0].record()
    for _ in range(reps):
        pad[:w.H, :w.W] = x
        spec = torch.fft.rfft2(pad)
    ev[1].record()
    for _ in range(reps):
        _ = torch.fft.irfft2(spec, s=(fh, fw))[:w.H, :w.W].contiguous()
    ev[2].record()
    torch.cuda.synchronize()
    r2c = ev[0].elapsed_time(ev[1]) / reps
    c2r = ev[1].elapsed_time(ev[2]) / reps
    del x, pad, spec
    torch.cuda.empty_cache()
    return {"r2c_ms": round(r2c, 4), "c2r_crop_ms": round(c2r, 4), "grid": [fw, fh],
            "note": "torch.fft (cuFFT) on the same padded grid; comparison only"}


def cpu_baseline_sample(ds, w):
    """One iteration of the reference core on the same inputs (rank 0, N=1)."""
    from oracle import oracle as O
    if not O.REF_BINARY.is_file():
        return None
    cores = os.cpu_count() or 1
    fftw = max(1, cores // w.nexp)
    a = ds.engine_args(iterations=1, prefix="cpubase", fft_workers=fftw, exposure_workers=w.nexp,
                       preprocess_workers=w.nexp).argv()
    r = subprocess.run([str(O.REF_BINARY), *a], capture_output=True, text=True,
                       env={**os.environ, "UPDC_PERSIST_CACHE": "1"}, timeout=900)
    if r.returncode:
        return {"value": None, "unit": "ms", "cores": cores, "kind": "reference", "sample": r.stderr[-200:]}
    rows = list(csv.reader(open(f"{ds.directory}/cpubase_timing.csv")))
    its = [float(v) for k, v in rows[1:] if k.startswith("iteration_") and k.endswith("_total")]
    return {"value": round(1000.0 * its[0], 1), "unit": "ms", "cores": cores, "kind": "reference",
            "sample": f"1 iteration of the reference core on the same {w.name} inputs "
                      f"(fft_workers={fftw}, exposure_workers={w.nexp}, FFTW-API shim FFT)"}


def reference_check(ds, w, form, device, **engine_kw):
    """The metric's accuracy side against the reference itself: a fresh engine
    of the timed form and the reference core (oracle/_ref, on this machine's
    host cores, warm caches) both run the workload's full iteration count on
    the same files; reported are the relative RMS and the largest relative
    error of the final x against the reference's, the per-iteration FreezeMu
    count rows that differ from the reference's freeze CSV
    (updc_core.c:1425-1431), the largest relative difference of min raw_mu,
    and the reference's own per-iteration times (the CPU baseline)."""
    import numpy as np
    from oracle import oracle as O
    from updc_b200.engine import Engine
    if not O.REF_BINARY.is_file():
        return None
    cores = os.cpu_count() or 1
    fftw = max(1, cores // w.nexp)
    e = Engine(form=form, device=device, **engine_kw)
    e.load(str(ds.manifest), w.W, w.H, w.iw, w.ih, w.nexp).setup()
    st = e.iterate(w.iterations, check_each=False)
    x = e.plane("estimate", as_double=True)
    mine = [(int(s.new_frozen[k]), int(s.total_frozen[k]), float(s.min_raw_mu[k])) for s in st for k in range(w.nexp)]
    e.close()
    a = ds.engine_args(iterations=w.iterations, prefix="refcheck", fft_workers=fftw, exposure_workers=w.nexp,
                       preprocess_workers=w.nexp).argv()
    t0 = time.time()
    r = subprocess.run([str(O.REF_BINARY), *a], capture_output=True, text=True,
                       env={**os.environ, "UPDC_PERSIST_CACHE": "1"}, timeout=3600)
    wall = time.time() - t0
    if r.returncode:
        return {"error": r.stderr[-300:]}
    xr = np.fromfile(f"{ds.directory}/refcheck_{w.iterations:02d}.bin", np.float32).reshape(w.H, w.W).astype(np.float64)
    d = x - xr
    mask = np.abs(xr) > 1e-8 * np.abs(xr).max()
    with open(f"{ds.directory}/refcheck_mufreeze.csv") as f:
        rows = list(csv.DictReader(f))
    count_mismatch = sum(1 for (a1, b1, _), q in zip(mine, rows)
                         if (a1, b1) != (int(q["n_new_frozen"]), int(q["n_total_frozen"])))
    mu_rel = max((abs(m - float(q["min_raw_mu"])) / max(abs(float(q["min_raw_mu"])), 1e-30)
                  for (_, _, m), q in zip(mine, rows)), default=0.0)
    trow = list(csv.reader(open(f"{ds.directory}/refcheck_timing.csv")))
    its = [float(v) for k, v in trow[1:] if k.startswith("iteration_") and k.endswith("_total")]
    return {"form": form, "iterations": w.iterations,
            "rel_rms": float(np.sqrt(np.mean(d * d) / np.mean(xr * xr))),
            "max_rel_masked": float(np.max(np.abs(d[mask]) / np.abs(xr[mask]))),
            "freeze_rows": len(rows), "freeze_count_rows_differing": count_mismatch,
            "frozen_total_reference": int(sum(int(q["n_new_frozen"]) for q in rows)),
            "min_raw_mu_max_rel_diff": mu_rel, "reference_wall_s": round(wall, 1),
            "reference_iteration_ms": [round(1000.0 * v, 1) for v in its], "cores": cores, "fft_workers": fftw}


def fp64_comparison(eng, ds, w, args, device, **engine_kw):
    """The metric's accuracy side: run the FP64 form (the GPU oracle) on the
    same inputs to the workload's full iteration count, bring the timed engine
    to the same count, and report the relative RMS of x, the FreezeMu masks
    that differ, and the FP64 form's own device ms/iteration.  The other FP32
    forms (Kahan-compensated sums; the reference's plain FP32 arithmetic) run
    the same count on the same FFT plans and are compared with it the same
    way (`forms`)."""
    import numpy as np
    from updc_b200.engine import Engine
    done = eng.iterations_done
    target = max(w.iterations, done)
    if target > done:
        eng.iterate(target - done, check_each=False)
    ref = Engine(form="fp64", device=device)
    ref.load(str(ds.manifest), w.W, w.H, w.iw, w.ih, w.nexp).setup()
    warm = 3
    st = ref.iterate(target, check_each=False)
    ms64 = 1000.0 * sum(s.seconds for s in st[warm:]) / max(1, target - warm)
    x64 = ref.plane("estimate", as_double=True)
    mask = np.abs(x64) > 1e-8 * np.abs(x64).max()
    frozen64 = [ref.plane("frozen", k) for k in range(w.nexp)]
    ref.close()

    def against_fp64(e):
        d = e.plane("estimate", as_double=True) - x64
        mism = sum(int(np.count_nonzero(e.plane("frozen", k) != frozen64[k])) for k in range(w.nexp))
        return {"rel_rms": float(np.sqrt(np.mean(d * d) / np.mean(x64 * x64))),
                "max_rel_masked": float(np.max(np.abs(d[mask]) / np.abs(x64[mask]))), "frozen_mismatch": mism}

    out = {"iterations": target, **against_fp64(eng), "fp64_ms_per_iteration": round(ms64, 4), "forms": {}}
    for form in ("fp32", "fp32-kahan", "fp32-reference"):
        if form == args.form:
            continue
        e = Engine(form=form, device=device, **engine_kw)
        e.load(str(ds.manifest), w.W, w.H, w.iw, w.ih, w.nexp).setup()
        st = e.iterate(target, check_each=False)
        out["forms"][form] = {**against_fp64(e),
                              "ms_per_iteration": round(1000.0 * sum(s.seconds for s in st[warm:]) / max(1, target - warm), 4)}
        e.close()
    return out


def batch_arm(args, rank, world, local_rank):
    """Batched cutouts: 64 fields of uneven size and exposure count, every
    stage one persistent launch over all fields, the loop one CUDA graph.
    A step is one iteration of every field; beside it, the same fields
    solved one after another by their own engines (graph per iteration)."""
    import torch
    from updc_b200 import synth
    from updc_b200.batch import Batch
    from updc_b200.engine import Engine
    torch.cuda.set_device(local_rank)
    workdir = Path(args.data_dir or tempfile.mkdtemp(prefix=f"updc_bench_batch_r{rank}_"))
    t0 = time.time()
    data = synth.generate_batch(workdir, n_fields=args.fields)
    gen_s = time.time() - t0
    b = Batch(form=args.form, device=local_rank, autotune=not args.no_autotune, tune_cache_dir=workdir)
    for ds in data:
        w = ds.workload
        b.add_field(ds.manifest, w.W, w.H, w.iw, w.ih, w.nexp)
    t0 = time.time()
    b.setup()
    setup_s = time.time() - t0
    b.iterate(args.warmup)
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clocks:
        recs = b.iterate(args.steps)
        torch.cuda.synchronize()
    ms = 1000.0 * sum(r["seconds"] for r in recs) / len(recs)
    # the same fields, one engine each, run one after another
    seq_ms = 0.0
    for ds in data:
        w = ds.workload
        e = Engine(form=args.form, device=local_rank, autotune=not args.no_autotune, tune_cache_dir=workdir)
        e.load(str(ds.manifest), w.W, w.H, w.iw, w.ih, w.nexp).setup()
        e.iterate(args.warmup, check_each=False)
        st = e.iterate(args.steps, check_each=False)
        seq_ms += 1000.0 * sum(x.seconds for x in st) / len(st)
        e.close()
    # e2e: upload every field's estimate from pinned host memory, one batch
    # iteration, read every estimate back
    hosts = []
    for i in range(b.fields):
        f = b.field(i)
        hosts.append(torch.empty((f.H, f.W), dtype=torch.float64 if args.form == "fp64" else torch.float32,
                                 pin_memory=True).numpy())
        f.read_plane_into("estimate", hosts[-1])
    e2e_steps = max(2, min(args.steps, 5))
    t0 = time.time()
    for _ in range(e2e_steps):
        for i in range(b.fields):
            b.field(i).set_plane("estimate", hosts[i])
        b.iterate(1, check_each=True)
        for i in range(b.fields):
            b.field(i).read_plane_into("estimate", hosts[i])
    e2e_ms = 1000.0 * (time.time() - t0) / e2e_steps
    nbytes = sum(h.nbytes for h in hosts)
    result = {
        "metric": "ms/iteration (all fields)", "value": round(ms, 4), "unit": "ms", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.form == "fp64" else "f32", "data": "synthetic",
        "config": {"workload": "c2", "fields": b.fields, "exposures": int(sum(d.workload.nexp for d in data)),
                   "grids": sorted({d.workload.W for d in data}), "form": args.form,
                   "units": {s: b.units(i) for i, s in enumerate(["estimate_rows", "columns", "forward_rows",
                                                                   "detector", "adjoint_gather", "scatter_rows",
                                                                   "update", "adjoint_rows"])},
                   "graph": "whole loop of --steps iterations", "l2": "per-field planes re-read each stage"},
        "sequential_single_field_ms": round(seq_ms, 4),
        "speedup_vs_sequential": round(seq_ms / ms, 3),
        "setup_s": round(setup_s, 2), "generate_s": round(gen_s, 1),
        "e2e": {"value": round(e2e_ms, 3), "unit": "ms", "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes},
        "gpu_launches": 11 * args.steps,
        "clocks": clocks.summary(),
    }
    if rank == 0:
        print(json.dumps(result))
    b.close()
    if not args.data_dir:
        shutil.rmtree(workdir, ignore_errors=True)
    return 0


PRE_SHAPE, PRE_EXPOSURES = (2048, 2048), 8
PRE_BYTES_PER_PIXEL = 4 + 4 + 8 + 8 + 8 + 4  # SCI, DQ, three variances read once; WHT written once


def _pre_exposures():
    from updc_b200 import synth
    return [synth.level2_exposure(PRE_SHAPE, "sources", 100 + k) for k in range(PRE_EXPOSURES)]


def _pre_planes(d):
    import numpy as np
    return (d["SCI"], d["DQ"], d["VAR_POISSON"].astype(np.float64), d["VAR_RNOISE"].astype(np.float64),
            d["VAR_FLAT"].astype(np.float64))


def preprocess_cpu_sample(exposures, limit_s=20.0):
    """The oracle's restatement of the reference's NumPy preprocessing on as
    many exposures as fit about `limit_s` seconds (at least one)."""
    from oracle import preprocess as OP
    t0 = time.time()
    done = 0
    for d in exposures:
        OP.prepare_exposure(*_pre_planes(d), "rnoise-sky", 1, 0.0, "bench")
        done += 1
        if time.time() - t0 > limit_s:
            break
    ms = 1000.0 * (time.time() - t0) / done
    return {"value": round(ms, 2), "unit": "ms", "cores": 1, "kind": "port",
            "sample": f"{done} of {len(exposures)} exposures of {PRE_SHAPE[0]}x{PRE_SHAPE[1]} (NumPy, one thread)"}


def preprocess_arm(args, rank, world, local_rank):
    """Per-exposure weight preprocessing of the c1 exposures (8 x 2048^2
    Level-2 planes): a step prepares every exposure; value = ms per exposure
    with the planes resident on the device, e2e = the same through pinned
    host arrays (planes copied in, WHT copied out)."""
    import numpy as np
    import torch
    from updc_b200 import preprocess as P
    torch.cuda.set_device(local_rank)
    exps = _pre_exposures()

    def pinned(a):
        t = torch.empty(a.shape, dtype=getattr(torch, a.dtype.name), pin_memory=True)
        t.numpy()[...] = a
        return t.numpy()
    host = [tuple(pinned(np.ascontiguousarray(a)) for a in _pre_planes(d)) for d in exps]
    dev = []
    for planes in host:
        t = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in planes]
        t[1] = t[1].view(torch.int32)
        dev.append(t)
    metrics = []
    for _ in range(args.warmup):
        for t in dev:
            P.prepare_exposure(*t, "rnoise-sky", 1, 0.0, "bench")
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clocks:
        start.record()
        for _ in range(args.steps):
            for t in dev:
                _w, m, _s = P.prepare_exposure(*t, "rnoise-sky", 1, 0.0, "bench")
                metrics.append(m)
        stop.record()
        torch.cuda.synchronize()
    ms = start.elapsed_time(stop) / (args.steps * len(dev))
    if world > 1:
        tt = torch.tensor([ms], device="cuda")
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        ms = float(tt.item())
    t0 = time.time()
    e2e_steps = max(1, min(args.steps, 3))
    for _ in range(e2e_steps):
        for planes in host:
            P.prepare_exposure(*planes, "rnoise-sky", 1, 0.0, "bench")
    e2e_ms = 1000.0 * (time.time() - t0) / (e2e_steps * len(host))
    npix = PRE_SHAPE[0] * PRE_SHAPE[1]
    peak, peak_kind = measured_peaks()
    achieved = PRE_BYTES_PER_PIXEL * npix / (ms * 1e-3) / 1e9
    cpu = preprocess_cpu_sample(exps) if rank == 0 and world == 1 and not args.no_cpu_baseline else None
    passes = statistics.mean(m["clip_passes"] for m in metrics)
    result = {
        "metric": "ms/exposure (weight preprocessing)", "value": round(ms, 4), "unit": "ms", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms * len(dev), 4),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic",
        "config": {"workload": "pre", "exposures": len(dev), "shape": list(PRE_SHAPE), "weight_mode": "rnoise-sky",
                   "clip_passes_mean": passes,
                   "l2": "each exposure's planes (151 MB) exceed the 126 MB L2; 8 exposures cycle"},
        "roofline": {"bound": "hbm", "kernel": "whole exposure (passes, sorts, host checks)",
                     "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "peak_kind": peak_kind, "algorithmic_bytes": PRE_BYTES_PER_PIXEL * npix, "traffic": None},
        "cpu_baseline": cpu,
        "e2e": {"value": round(e2e_ms, 3), "unit": "ms", "h2d_bytes_per_step": 32 * npix, "d2h_bytes_per_step": 4 * npix},
        # per exposure: k_pre_valid, k_pre_clip, k_pre_sky, k_pre_weight, two
        # radix selects (1 + 2 x 8 and 1 + 2 x 4 launches); a standard-deviation
        # fallback adds eight (the sort of SCI is CUB's)
        "gpu_launches": int(sum(31 + 8 * m["std_fallbacks"] for m in metrics)),
        "clocks": clocks.summary(),
    }
    if rank == 0:
        print(json.dumps(result))
    return 0


def sharded_arm(args, rank, world, local_rank):
    """N > 1: one field, its exposures split over the ranks (contiguous
    shares), every rank set up on its own share (the setup's cross-exposure
    sums all-reduced once); per iteration each rank
    computes the partial correction of its exposures, one NCCL all-reduce
    sums them, and every rank applies the same update.  Total work is fixed
    (strong scaling); time is the max over ranks of the device-timed loop."""
    import datetime
    import torch
    import torch.distributed as dist
    from updc_b200 import synth
    from updc_b200.sharded import ShardedSolver, open_engine_shard
    torch.cuda.set_device(local_rank)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                            device_id=torch.device("cuda", local_rank))
    w = synth.WORKLOADS[args.workload]
    workdir = Path(args.data_dir or tempfile.mkdtemp(prefix=f"updc_bench_shard_r{rank}_"))
    try:
        ds = synth.generate(w.name, workdir, use_torch=True)
        t0 = time.time()
        shard = open_engine_shard(str(ds.manifest), w.W, w.H, w.iw, w.ih, w.nexp, rank, world, form=args.form,
                                  device=local_rank, dist=dist)
        solver = ShardedSolver(shard, dist)
        setup_s = time.time() - t0
        solver.iterate(args.warmup)
        # one iteration (partial correction, NCCL all-reduce of the engine's
        # own correction plane, update) as a CUDA graph on the engine's stream
        solver.capture()
        dist.barrier()
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        with ClockSampler(local_rank) as clocks:
            ev[0].record(shard.stream)
            recs = solver.iterate(args.steps, records=False)
            ev[1].record(shard.stream)
            torch.cuda.synchronize()
        t = torch.tensor([ev[0].elapsed_time(ev[1]) / args.steps], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        # e2e: every step the estimate comes from pinned host memory and goes back
        eng = shard.engine
        x = torch.empty((w.H, w.W), dtype=torch.float64 if args.form == "fp64" else torch.float32,
                        pin_memory=True).numpy()
        eng.read_plane_into("estimate", x)
        e2e_steps = max(2, min(args.steps, 5))
        dist.barrier()
        t0 = time.time()
        for _ in range(e2e_steps):
            eng.set_plane("estimate", x)
            solver.iterate(1)
            eng.read_plane_into("estimate", x)
        te = torch.tensor([1000.0 * (time.time() - t0) / e2e_steps], device="cuda")
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
        solver.release()  # the graph holds an NCCL call: released before the group is destroyed
        first, count = shard.first, shard.count
        result = {
            "metric": "ms/iteration", "value": round(ms, 4), "unit": "ms", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": False, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64" if args.form == "fp64" else "f32", "data": "synthetic",
            "config": {"workload": args.workload, "form": args.form, "target": [w.W, w.H], "exposures": w.nexp,
                       "detector": [w.iw, w.ih], "psf": w.psf_size, "fft": list(eng.fft_shape),
                       "parallelism": f"exposure shards over {world} ranks, NCCL all-reduce of the correction plane "
                                      "in place on the engine's stream, one CUDA graph per iteration",
                       "rank0_exposures": [first, first + count],
                       "l2": "working set >> 126 MB L2; no flush needed"},
            "setup_s": round(setup_s, 2),
            "signed_sum_last": recs[-1]["signed_sum"],
            "e2e": {"value": round(float(te.item()), 3), "unit": "ms", "h2d_bytes_per_step": x.nbytes,
                    "d2h_bytes_per_step": x.nbytes},
            "gpu_launches": (7 if eng.kernel_variants["fused_gather"] else 8) * args.steps,
            "clocks": clocks.summary(),
        }
        if rank == 0:
            print(json.dumps(result))
        eng.close()
        dist.barrier()
    finally:
        dist.destroy_process_group()
        if not args.data_dir:
            shutil.rmtree(workdir, ignore_errors=True)
    return 0


def b200_arm(args, rank, world, local_rank):
    import numpy as np
    import torch
    from updc_b200 import synth
    from updc_b200.engine import Engine

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local_rank))
    w = synth.WORKLOADS[args.workload]
    if args.exposures:
        # the workload's geometry with fewer (or more) exposures: a smaller
        # case of the same kernels for profiler captures
        import dataclasses
        w = dataclasses.replace(w, name=f"{w.name}x{args.exposures}", nexp=args.exposures)
    workdir = Path(args.data_dir or tempfile.mkdtemp(prefix=f"updc_bench_r{rank}_"))
    ds = synth.generate(w, workdir, use_torch=True)
    tune_dir = args.tune_cache or workdir
    if args.tune_cache:
        Path(tune_dir).mkdir(parents=True, exist_ok=True)
    eng = Engine(form=args.form, device=local_rank, autotune=not args.no_autotune and not args.fft_shape,
                 tune_cache_dir=str(tune_dir), fft_shape=tuple(args.fft_shape) if args.fft_shape else None)
    eng.load(str(ds.manifest), w.W, w.H, w.iw, w.ih, w.nexp)
    t0 = time.time()
    eng.setup()
    setup_s = time.time() - t0
    fw, fh = eng.fft_shape
    eng.iterate(args.warmup, check_each=False)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clocks:
        t0 = time.time()
        stats = eng.iterate(args.steps, check_each=False)
        torch.cuda.synchronize()
        wall = time.time() - t0
    ms = 1000.0 * sum(s.seconds for s in stats) / len(stats)
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    # per-stage pass (eager launches with events between stages)
    eng.set_stage_timing(True)
    st = eng.iterate(max(3, min(args.steps, 5)), check_each=False)
    eng.set_stage_timing(False)
    stage_ms = {name: 1000.0 * statistics.mean(s.stage_seconds[i] for s in st) for i, name in enumerate(STAGES)}
    links = [(eng.link_count(k), eng.link_encoding(k)) for k in range(w.nexp)]
    sb = stage_bytes(w, fw, fh, links, [L for L, _ in links], 8 if args.form == "fp64" else 4)
    mb = model_bytes(w, fw, fh, links, 8 if args.form == "fp64" else 4)
    variants = eng.kernel_variants
    stages = list(STAGES)
    if variants["fused_gather"]:
        # one kernel gathers S^T(wr) into the scatter row transform: the two
        # stages are timed as one, and the scatter plane's write and re-read
        # (2 x 4 B per target and exposure) no longer exist
        fused = "gather_scatter_x_pass"
        stage_ms[fused] = stage_ms.pop("adjoint_gather") + stage_ms.pop("scatter_x_pass")
        sb[fused] = sb.pop("adjoint_gather") + sb.pop("scatter_x_pass") - 2 * w.nexp * w.W * w.H * (8 if args.form == "fp64" else 4)
        mb[fused] = mb.pop("adjoint_gather") + mb.pop("scatter_x_pass")
        i = stages.index("adjoint_gather")
        stages[i:i + 2] = [fused]
    dom = max(stage_ms, key=stage_ms.get)
    peak, peak_kind = measured_peaks()
    achieved = mb[dom] / (stage_ms[dom] * 1e-3) / 1e9
    achieved_pruned = sb[dom] / (stage_ms[dom] * 1e-3) / 1e9
    iter_gbs = sum(mb.values()) / (ms * 1e-3) / 1e9
    # cuFFT (through torch) on the same padded grid, for comparison only: one
    # zero-padded 2-D R2C of the 4096^2 plane and one C2R + crop, as our
    # estimate/forward passes do them (not used by the solver)
    cufft = cufft_reference(torch, w, fw, fh)
    # e2e through the C ABI with pinned host buffers: upload x, one iteration, read x back
    xdt = torch.float64 if args.form == "fp64" else torch.float32
    x = torch.empty((w.H, w.W), dtype=xdt, pin_memory=True).numpy()
    eng.read_plane_into("estimate", x)
    e2e_steps = max(2, min(args.steps, 5))
    t0 = time.time()
    for _ in range(e2e_steps):
        eng.set_plane("estimate", x)
        eng.iterate(1, check_each=True)
        eng.read_plane_into("estimate", x)
    e2e_ms = 1000.0 * (time.time() - t0) / e2e_steps
    nout = w.W * w.H
    fp64 = None
    if args.form != "fp64" and not args.no_fp64_check:
        fp64 = fp64_comparison(eng, ds, w, args, local_rank, autotune=not args.no_autotune and not args.fft_shape,
                               fft_shape=tuple(args.fft_shape) if args.fft_shape else None, tune_cache_dir=str(tune_dir))
    cpu = None
    refcheck = None
    if rank == 0 and world == 1 and not args.no_reference_check:
        refcheck = reference_check(ds, w, args.form, local_rank, autotune=not args.no_autotune and not args.fft_shape,
                                   fft_shape=tuple(args.fft_shape) if args.fft_shape else None,
                                   tune_cache_dir=str(tune_dir))
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        its = (refcheck or {}).get("reference_iteration_ms")
        if its and len(its) > 1:
            # the reference run of the accuracy check is the CPU baseline sample
            timed = its[1:]
            cpu = {"value": round(statistics.mean(timed), 1), "unit": "ms", "cores": refcheck["cores"],
                   "kind": "reference",
                   "sample": f"iterations 2-{len(its)} of the reference core's {len(its)}-iteration run on the same "
                             f"{w.name} inputs (fft_workers={refcheck['fft_workers']}, exposure_workers={w.nexp}, "
                             f"warm caches, FFTW-API shim FFT)"}
        else:
            cpu = cpu_baseline_sample(ds, w)
    # estimate R2C, column forward, forward C2R (all exposures), detector,
    # adjoint gather and scatter R2C (one kernel when fused), column adjoint,
    # adjoint C2R, update (with its reduction)
    launches_per_iter = 7 if variants["fused_gather"] else 8
    result = {
        "metric": "ms/iteration", "value": round(ms, 4), "unit": "ms", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": False,
        # one fixed field at every N: strong, unless N independent replicas run
        "scaling": "weak" if world > 1 else "strong", "vs_baseline": None,
        "dtype": "f64" if args.form == "fp64" else "f32",
        "data": "synthetic",
        "config": {"workload": args.workload, "form": args.form, "target": [w.W, w.H], "exposures": w.nexp,
                   "detector": [w.iw, w.ih], "psf": w.psf_size, "fft": [fw, fh],
                   "fft_radices": {"rows": eng.fft_radices(0), "columns": eng.fft_radices(1)},
                   "autotune": None if args.no_autotune else eng.autotune_info,
                   "parallelism": "replicas" if world > 1 else "single",
                   "l2": "working set ~%.1f GB >> 126 MB L2; no flush needed" % (eng.device_bytes / 1e9)},
        "wall_ms_per_step": round(1000.0 * wall / args.steps, 4),
        "setup_s": round(setup_s, 2),
        "stage_ms": {k: round(v, 4) for k, v in stage_ms.items()},
        "stage_gbs": {k: round(mb[k] / (stage_ms[k] * 1e-3) / 1e9, 1) for k in stages},
        "stage_gbs_pruned": {k: round(sb[k] / (stage_ms[k] * 1e-3) / 1e9, 1) for k in stages},
        "kernel_variants": variants,
        "iteration_model": {"bytes": sum(mb.values()), "achieved_gbs": round(iter_gbs, 1),
                            "frac": round(iter_gbs / peak, 4)},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak,
                     "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                     "algorithmic_bytes": mb[dom],
                     "pruned_bytes": sb[dom], "achieved_pruned": round(achieved_pruned, 1),
                     "frac_pruned": round(achieved_pruned / peak, 4),
                     "traffic": round(sb[dom] * TRAFFIC_RATIO_C1X2[dom]) if dom in TRAFFIC_RATIO_C1X2 else None,
                     "traffic_source": "ncu dram__bytes_read+write of the same kernel on the c1 geometry with 2 "
                                       "exposures, scaled by the units processed"},
        "cpu_baseline": cpu,
        "e2e": {"value": round(e2e_ms, 3), "unit": "ms", "h2d_bytes_per_step": x.itemsize * nout,
                "d2h_bytes_per_step": x.itemsize * nout},
        "cufft_reference": cufft,
        "fp64_check": fp64,
        "reference_check": refcheck,
        "speedup_vs_fp64": round(fp64["fp64_ms_per_iteration"] / ms, 3) if fp64 else None,
        "gpu_launches": launches_per_iter * args.steps,
        "clocks": clocks.summary(),
    }
    if rank == 0:
        print(json.dumps(result))
    eng.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if not args.data_dir:
        shutil.rmtree(workdir, ignore_errors=True)
    return 0


def main():
    p = argparse.ArgumentParser(description=__doc__)
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--workload", default="c1")
    p.add_argument("--form", default="fp32", choices=["fp32", "fp64", "fp32-kahan", "fp32-reference"])
    p.add_argument("--data-dir", default=None)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--replicas", action="store_true",
                   help="with N > 1: N independent replicas instead of exposure shards of one field")
    p.add_argument("--fields", type=int, default=64, help="fields of the batched workload (c2)")
    p.add_argument("--tune-cache", default=None,
                   help="directory of the FFT autotuner's cache (a profiled rerun then uses the same plans)")
    p.add_argument("--no-autotune", action="store_true",
                   help="smallest 7-smooth FFT shape and greedy radix splits instead of the device autotuner")
    p.add_argument("--no-fp64-check", action="store_true",
                   help="skip the FP64-form run that gives the metric's accuracy side")
    p.add_argument("--exposures", type=int, default=0,
                   help="run the workload's geometry with this many exposures (a smaller case for profiling)")
    p.add_argument("--fft-shape", type=int, nargs=2, default=None, metavar=("FW", "FH"),
                   help="fixed FFT shape instead of the autotuner's (catalog radix splits where the shape has them)")
    p.add_argument("--no-reference-check", action="store_true",
                   help="skip the full-length run of the reference core that the final x is compared with")
    args = p.parse_args()
    rank, world, local_rank = env_rank()
    if args.impl == "reference":
        return reference_arm(args, rank, world)
    if args.workload == "c2":
        return batch_arm(args, rank, world, local_rank)
    if args.workload == "pre":
        return preprocess_arm(args, rank, world, local_rank)
    if world > 1 and not args.replicas:
        return sharded_arm(args, rank, world, local_rank)
    return b200_arm(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
