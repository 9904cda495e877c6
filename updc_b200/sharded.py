"""Exposure-sharded solve of one field, one process per GPU.

The iteration of updc/c_core/updc_core.c:1410-1456 sums the adjoint of every
exposure before its single inverse transform (core:1280-1287); that sum is
the only place exposures meet.  So each rank sets up the whole field
(LinkMaps, PSF spectra, the drizzle x0 and the denominator D over all
exposures, identical on every rank) and then iterates only its own
contiguous share of the exposures: forward model, detector loop, transposed
gather and adjoint of its exposures give a partial correction plane, the
partial planes are summed over ranks with one all-reduce, and every rank
applies the same multiplicative update, so the estimate stays replicated
without ever being exchanged.  FreezeMu state stays with the rank that owns
the exposure.

``ShardedSolver`` drives any shard object with the two calls below; the GPU
shard is ``EngineShard`` (the engine's stage hooks through the C ABI), and
the collective is ``torch.distributed.all_reduce`` (NCCL between GPUs).
"""
from __future__ import annotations

from typing import List, Optional, Tuple


def shard_range(nexp: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous, balanced exposure range (first, count) of a rank."""
    if not 1 <= world <= nexp:
        raise ValueError(f"{world} ranks cannot share {nexp} exposures")
    base, extra = divmod(nexp, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


class EngineShard:
    """One rank's exposure shard of a field on its GPU."""

    def __init__(self, engine, first: int, count: int):
        import torch
        self.engine = engine
        self.first, self.count = first, count
        engine.set_active_exposures(first, count)
        self.double = engine.form == "fp64"
        dtype = torch.float64 if self.double else torch.float32
        self.buffer = torch.empty((engine.H, engine.W), dtype=dtype, device="cuda")

    def partial_correction(self):
        """Forward model, detector loop, gather and adjoint of this shard's
        exposures; returns the partial correction plane (a CUDA tensor)."""
        import torch
        e = self.engine
        e.stage_forward()
        new, total, _ = e.stage_detector()
        e.stage_correction()
        e.copy_plane_device("correction", self.buffer.data_ptr(), to_engine=False, as_double=self.double,
                            stream=torch.cuda.current_stream().cuda_stream)
        self.frozen = int(total[self.first:self.first + self.count].sum())
        return self.buffer

    def broadcast_denominator(self, dist, group=None) -> None:
        """Every rank takes rank 0's denominator plane, so that ranks whose
        transforms round differently still apply the identical update."""
        import torch
        e = self.engine
        stream = torch.cuda.current_stream().cuda_stream
        d = torch.empty_like(self.buffer)
        e.copy_plane_device("denominator", d.data_ptr(), to_engine=False, as_double=self.double, stream=stream)
        dist.broadcast(d, src=0, group=group)
        e.copy_plane_device("denominator", d.data_ptr(), to_engine=True, as_double=self.double, stream=stream)
        e.refresh_sensitivity()

    def apply_update(self, correction) -> Tuple[float, int]:
        """Write the summed correction back and run the update; returns the
        signed sum and the negative count of the new estimate."""
        import torch
        self.engine.copy_plane_device("correction", correction.data_ptr(), to_engine=True, as_double=self.double,
                                      stream=torch.cuda.current_stream().cuda_stream)
        return self.engine.stage_update()


class ShardedSolver:
    """Iterations of an exposure-sharded field: partial correction, one
    all-reduce (sum) over the ranks, the same update on every rank."""

    def __init__(self, shard, dist=None, group=None):
        self.shard = shard
        self.dist = dist
        self.group = group
        if dist is not None:
            shard.broadcast_denominator(dist, group)

    def iterate(self, n: int = 1) -> List[dict]:
        out = []
        for _ in range(n):
            c = self.shard.partial_correction()
            if self.dist is not None:
                self.dist.all_reduce(c, op=self.dist.ReduceOp.SUM, group=self.group)
            s, neg = self.shard.apply_update(c)
            out.append({"signed_sum": s, "negative": neg, "frozen": getattr(self.shard, "frozen", 0)})
        return out


def open_engine_shard(manifest: str, W: int, H: int, iw: int, ih: int, nexp: int, rank: int, world: int,
                      form: str = "fp32", device: int = 0, **engine_kw) -> EngineShard:
    """Set up the whole field on this rank's GPU and keep its exposure shard."""
    from .engine import Engine
    e = Engine(form=form, device=device, use_graph=False, **engine_kw)
    e.load(manifest, W, H, iw, ih, nexp).setup()
    first, count = shard_range(nexp, rank, world)
    return EngineShard(e, first, count)
