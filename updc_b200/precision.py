"""Precision forms compared with the FP64 GPU form, iteration by iteration.

    python -m updc_b200.precision --workload c1 --iterations 39 [--forms fp32,fp32-kahan,fp32-reference]

The FP64 form (everything in double) is the GPU oracle.  Each FP32 form runs
in lockstep with it on the same inputs; after every iteration the estimates
are compared (relative RMS and maximum relative error over pixels with
|x| > 1e-8 max|x|, the masked-relative measure of the reference's
tools/compare_fits.py:10-29) and the FreezeMu masks are compared pixel by
pixel (the count of mask entries that differ).  Device ms/iteration of each
form is reported.
"""
from __future__ import annotations

import argparse
import json
import sys
import tempfile
import time
from pathlib import Path
from typing import Dict, List

import numpy as np

from .engine import Engine


def compare(x: np.ndarray, ref: np.ndarray) -> Dict[str, float]:
    x = x.astype(np.float64)
    ref = ref.astype(np.float64)
    d = x - ref
    rms = float(np.sqrt(np.mean(d * d) / max(np.mean(ref * ref), 1e-300)))
    mask = np.abs(ref) > 1e-8 * np.abs(ref).max()
    max_rel = float(np.max(np.abs(d[mask]) / np.abs(ref[mask]))) if mask.any() else 0.0
    return {"rel_rms": rms, "max_rel": max_rel, "max_abs": float(np.abs(d).max())}


def run_forms(manifest: str, W: int, H: int, iw: int, ih: int, nexp: int, iterations: int,
              forms: List[str], device: int = 0) -> Dict[str, list]:
    """Returns {form: [per-iteration record]} with errors against the FP64 form."""
    out: Dict[str, list] = {}
    for form in forms:
        # the FP32 form first: its one-time FP64 denominator needs transient
        # memory that must not coincide with the FP64 engine's planes (c4
        # holds ~150 GB with both engines alive)
        eng = Engine(form=form, device=device)
        eng.load(manifest, W, H, iw, ih, nexp).setup()
        ref = Engine(form="fp64", device=device)
        ref.load(manifest, W, H, iw, ih, nexp).setup()
        recs = []
        for it in range(1, iterations + 1):
            sr = ref.iterate(1)[0]
            se = eng.iterate(1)[0]
            rec = {"iteration": it, "ms": 1000.0 * se.seconds, "ms_fp64": 1000.0 * sr.seconds}
            rec.update(compare(eng.plane("estimate", as_double=True), ref.plane("estimate", as_double=True)))
            mism = 0
            for k in range(nexp):
                mism += int(np.count_nonzero(eng.plane("frozen", k) != ref.plane("frozen", k)))
            rec["frozen_mismatch"] = mism
            rec["frozen_total"] = int(se.total_frozen.sum())
            recs.append(rec)
        out[form] = recs
        eng.close()
        ref.close()
    return out


def summary(results: Dict[str, list]) -> Dict[str, dict]:
    s = {}
    for form, recs in results.items():
        last = recs[-1]
        s[form] = {"final_rel_rms": last["rel_rms"], "final_max_rel": last["max_rel"],
                   "worst_rel_rms": max(r["rel_rms"] for r in recs),
                   "frozen_mismatch_final": last["frozen_mismatch"],
                   "ms_per_iteration": float(np.median([r["ms"] for r in recs])),
                   "fp64_ms_per_iteration": float(np.median([r["ms_fp64"] for r in recs])),
                   "iterations": len(recs)}
    return s


def main(argv=None) -> int:
    p = argparse.ArgumentParser(description=__doc__)
    p.add_argument("--workload", default="c1")
    p.add_argument("--iterations", type=int, default=None)
    p.add_argument("--forms", default="fp32,fp32-kahan,fp32-reference")
    p.add_argument("--out", default=None, help="write the per-iteration records as JSON")
    a = p.parse_args(argv)
    from . import synth
    w = synth.WORKLOADS[a.workload]
    its = a.iterations or w.iterations
    with tempfile.TemporaryDirectory(prefix="updc_prec_") as d:
        t0 = time.time()
        ds = synth.generate(w.name, d)
        gen = time.time() - t0
        try:
            import torch
            torch.cuda.empty_cache()         # the generator's device buffers
        except ImportError:
            pass
        res = run_forms(str(ds.manifest), w.W, w.H, w.iw, w.ih, w.nexp, its, a.forms.split(","))
    s = summary(res)
    print(json.dumps({"workload": a.workload, "iterations": its, "generate_s": round(gen, 1), "forms": s}))
    if a.out:
        Path(a.out).write_text(json.dumps({"summary": s, "records": res}, indent=1))
    return 0


if __name__ == "__main__":
    sys.exit(main())
