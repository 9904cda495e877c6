"""Exposure-sharded solve of one field, one process per GPU.

The iteration of updc/c_core/updc_core.c:1410-1456 sums the adjoint of every
exposure before its single inverse transform (core:1280-1287); that sum is
the only place exposures meet.  So each rank sets up only its own
contiguous share of the exposures (LinkMaps, PSF spectra), the setup's
cross-exposure sums (the drizzle x0's coverage, data and background, and the
denominator D) are all-reduced once, and every rank then iterates its
share: forward model, detector loop, transposed
gather and adjoint of its exposures give a partial correction plane, the
partial planes are summed over ranks with one all-reduce, and every rank
applies the same multiplicative update, so the estimate stays replicated
without ever being exchanged.  FreezeMu state stays with the rank that owns
the exposure.

``ShardedSolver`` drives any shard object that has partial_correction()
(returns the tensor to sum), enqueue_update(summed), finish() -> (signed
sum, negative count) and broadcast_denominator(dist); the GPU shard is
``EngineShard``: the engine's own correction plane, viewed as a CUDA tensor
without a copy, is summed in place by ``torch.distributed.all_reduce`` (NCCL
between GPUs) on the engine's stream between the engine's two non-blocking
halves of an iteration (updc_enqueue_partial / updc_enqueue_update), so an
iteration takes no host round trip and can be captured as one CUDA graph.
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


class _DevicePlane:
    """A W x H plane the engine owns, described for torch.as_tensor (zero copy)."""

    def __init__(self, ptr: int, shape, double: bool):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f8" if double else "<f4",
                                         "data": (ptr, False), "version": 3, "strides": None, "stream": None}


class EngineShard:
    """One rank's exposure shard of a field on its GPU.  The partial
    correction is the engine's own correction plane, viewed as a CUDA tensor
    without a copy; everything is ordered on the engine's stream (`stream`),
    on which the caller runs the collective between the two halves."""

    def __init__(self, engine, first: int, count: int):
        import torch
        self.engine = engine
        self.first, self.count = first, count
        engine.set_active_exposures(first, count)
        self.double = engine.form == "fp64"
        dev = torch.cuda.current_device()
        self.stream = torch.cuda.ExternalStream(engine.stream_handle(), device=dev)
        shape = (engine.H, engine.W)
        self.correction = torch.as_tensor(_DevicePlane(engine.plane_device_pointer("correction"), shape, self.double),
                                          device=dev)
        self.denominator = torch.as_tensor(_DevicePlane(engine.plane_device_pointer("denominator"), shape,
                                                        self.double), device=dev)
        self.frozen = 0

    def partial_correction(self):
        """Forward model, detector loop, gather and adjoint of this shard's
        exposures, enqueued on `stream`; returns the correction plane (valid on
        `stream` once the work has run)."""
        self.engine.enqueue_partial()
        return self.correction

    def broadcast_denominator(self, dist, group=None) -> None:
        """Every rank takes rank 0's denominator plane, so that ranks whose
        transforms round differently still apply the identical update."""
        import torch
        with torch.cuda.stream(self.stream):
            dist.broadcast(self.denominator, src=0, group=group)
        self.stream.synchronize()
        self.engine.refresh_sensitivity()

    def enqueue_update(self, correction=None) -> None:
        """The update from the summed correction, enqueued on `stream` (a
        tensor other than the engine's own plane is copied into it first)."""
        import torch
        if correction is not None and correction.data_ptr() != self.correction.data_ptr():
            with torch.cuda.stream(self.stream):
                self.correction.copy_(correction)
        self.engine.enqueue_update()

    def finish(self) -> Tuple[float, int]:
        """Waits for the iteration; returns the signed sum and the negative
        count of the new estimate (FreezeMu total of the shard in `frozen`)."""
        s, neg, _, total, _ = self.engine.finish_iteration()
        self.frozen = int(total[self.first:self.first + self.count].sum())
        return s, neg

    def apply_update(self, correction) -> Tuple[float, int]:
        self.enqueue_update(correction)
        return self.finish()


class ShardedSolver:
    """Iterations of an exposure-sharded field: partial correction, one
    all-reduce (sum) over the ranks, the same update on every rank.  With a
    GPU shard the three steps run on the engine's stream with no host round
    trip, and `capture()` records them as one CUDA graph that `iterate`
    then replays."""

    def __init__(self, shard, dist=None, group=None):
        self.shard = shard
        self.dist = dist
        self.group = group
        self.graph = None
        if dist is not None:
            shard.broadcast_denominator(dist, group)

    def _stream_ctx(self):
        import contextlib
        stream = getattr(self.shard, "stream", None)
        if stream is None:
            return contextlib.nullcontext()
        import torch
        return torch.cuda.stream(stream)

    def _enqueue(self) -> None:
        c = self.shard.partial_correction()
        if self.dist is not None:
            self.dist.all_reduce(c, op=self.dist.ReduceOp.SUM, group=self.group)
        self.shard.enqueue_update(c)

    def capture(self) -> None:
        """Record one iteration (partial correction, all-reduce, update) as a
        CUDA graph on the engine's stream; every rank must capture."""
        import torch
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=self.shard.stream):
            self._enqueue()
        self.graph = g

    def release(self) -> None:
        """Drop the captured graph (before the process group is destroyed)."""
        self.graph = None

    def iterate(self, n: int = 1, records: bool = True) -> List[dict]:
        """n iterations; with records=False they are enqueued back to back and
        only the last one's record is read (no host wait in between)."""
        out = []
        for i in range(n):
            if self.graph is not None:
                self.graph.replay()
            else:
                with self._stream_ctx():
                    self._enqueue()
            if records or i == n - 1:
                s, neg = self.shard.finish()
                out.append({"signed_sum": s, "negative": neg, "frozen": getattr(self.shard, "frozen", 0)})
        return out


def open_engine_shard(manifest: str, W: int, H: int, iw: int, ih: int, nexp: int, rank: int, world: int,
                      form: str = "fp32", device: int = 0, dist=None, group=None, **engine_kw) -> EngineShard:
    """This rank's exposure shard on its GPU.  With `dist` and more than one
    rank the shard is set up alone — LinkMaps and PSF spectra of its own
    exposures only — and the partial planes the setup leaves (coverage, the
    drizzle's data and background sums, the denominator) are all-reduced
    before the engine finishes the drizzle estimate and the maximum
    sensitivity; results then equal the whole field's up to the order of the
    cross-rank sums.  Without, every rank sets up the whole field."""
    import torch
    from .engine import Engine
    e = Engine(form=form, device=device, use_graph=False, **engine_kw)
    e.load(manifest, W, H, iw, ih, nexp)
    first, count = shard_range(nexp, rank, world)
    if dist is not None and world > 1:
        e.set_active_exposures(first, count)
        e.setup()
        dev = torch.cuda.current_device()
        stream = torch.cuda.ExternalStream(e.stream_handle(), device=dev)
        with torch.cuda.stream(stream):
            for name in ("coverage", "estimate", "correction", "denominator"):
                plane = torch.as_tensor(_DevicePlane(e.plane_device_pointer(name), (H, W), form == "fp64"), device=dev)
                dist.all_reduce(plane, op=dist.ReduceOp.SUM, group=group)
        stream.synchronize()
        e.finish_shard_setup()
    else:
        e.setup()
    return EngineShard(e, first, count)
