"""Exposure-sharded solve (updc_b200/sharded.py).

CPU: the exposure split, and two gloo ranks driving a small linear model of
the same iteration (partial corrections, one all-reduce, the same update on
both ranks) against one process holding every exposure.
GPU: two exposure shards of one field on the same GPU, their partial
corrections summed by the host, against the engine's own iteration.
"""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch

from conftest import rel_rms
from updc_b200.sharded import ShardedSolver, shard_range


def test_shard_range_covers_every_exposure_once():
    for nexp in range(1, 13):
        for world in range(1, nexp + 1):
            got = [shard_range(nexp, r, world) for r in range(world)]
            assert got[0][0] == 0 and sum(c for _, c in got) == nexp
            assert all(a[0] + a[1] == b[0] for a, b in zip(got, got[1:]))
            assert max(c for _, c in got) - min(c for _, c in got) <= 1
    with pytest.raises(ValueError):
        shard_range(3, 0, 4)


class ToyShard:
    """The iteration of the solver on a dense stand-in for H_k (FP64 on CPU):
    C = sum_k H_k^T (W_k y_k / (H_k x + b_k)), D = sum_k H_k^T W_k, x *= C/D."""

    def __init__(self, seed, nexp, first, count, partial=False):
        g = torch.Generator().manual_seed(seed)
        m, n = 40, 30
        self.H = torch.rand((nexp, m, n), generator=g, dtype=torch.float64)
        self.W = torch.rand((nexp, m), generator=g, dtype=torch.float64) + 0.5
        self.b = torch.rand(nexp, generator=g, dtype=torch.float64)
        xt = torch.rand(n, generator=g, dtype=torch.float64) * 10
        self.y = torch.einsum("kmn,n->km", self.H, xt) + self.b[:, None]
        self.x = torch.ones(n, dtype=torch.float64)
        # partial: this shard's terms of D only (the shard set up alone; the
        # ranks all-reduce them before iterating)
        ks = slice(first, first + count) if partial else slice(0, nexp)
        self.D = torch.einsum("kmn,km->n", self.H[ks], self.W[ks])
        self.first, self.count = first, count

    def partial_correction(self):
        c = torch.zeros_like(self.x)
        for k in range(self.first, self.first + self.count):
            mu = self.H[k] @ self.x + self.b[k]
            c += self.H[k].T @ (self.W[k] * self.y[k] / mu)
        return c

    def broadcast_denominator(self, dist, group=None):
        dist.broadcast(self.D, src=0, group=group)

    def enqueue_update(self, c):
        self.x = self.x * (c / self.D)

    def finish(self):
        return float(self.x.sum()), int((self.x < 0).sum())


def _gloo_rank(rank, world, port, nexp, iters, out, partial=False):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        first, count = shard_range(nexp, rank, world)
        shard = ToyShard(3, nexp, first, count, partial=partial)
        if partial:
            dist.all_reduce(shard.D, op=dist.ReduceOp.SUM)   # the setup's one exchange
        recs = ShardedSolver(shard, dist).iterate(iters)
        xs = [torch.zeros_like(shard.x) for _ in range(world)]
        dist.all_gather(xs, shard.x)
        if rank == 0:
            torch.save({"x": [t.clone() for t in xs], "sums": [r["signed_sum"] for r in recs]}, out)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("partial", [False, True])
def test_two_gloo_ranks_match_one_process(tmp_path, partial):
    """Two gloo ranks against one process; with `partial` each rank builds
    only its own exposures' denominator terms and the ranks all-reduce D once
    before iterating (the shard setup)."""
    nexp, iters = 7, 6
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = tmp_path / "rank0.pt"
    torch.multiprocessing.spawn(_gloo_rank, args=(2, port, nexp, iters, str(out), partial), nprocs=2, join=True)
    got = torch.load(out)
    ref = ToyShard(3, nexp, 0, nexp)
    sums = [r["signed_sum"] for r in ShardedSolver(ref).iterate(iters)]
    assert torch.equal(got["x"][0], got["x"][1])            # the estimate stays replicated
    np.testing.assert_allclose(got["x"][0].numpy(), ref.x.numpy(), rtol=1e-12)
    np.testing.assert_allclose(got["sums"], sums, rtol=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("form,tol", [("fp64", 1e-12), ("fp32", 1e-5)])
def test_two_exposure_shards_match_the_whole_field(engine_lib, datasets, form, tol):
    from updc_b200.engine import Engine
    from updc_b200.sharded import EngineShard
    ds = datasets("c0")
    w = ds.workload

    def engine():
        e = Engine(form=form, use_graph=False)
        return e.load(str(ds.manifest), w.W, w.H, w.iw, w.ih, w.nexp).setup()

    whole = engine()
    shards = [EngineShard(engine(), *shard_range(w.nexp, r, 2)) for r in range(2)]
    cur = torch.cuda.current_stream()
    for _ in range(5):
        whole.iterate(1)
        parts = [s.partial_correction() for s in shards]   # enqueued on each engine's stream
        for s in shards:
            cur.wait_stream(s.stream)
        c = parts[0] + parts[1]                             # the all-reduce of two ranks, on one GPU
        for s in shards:
            s.stream.wait_stream(cur)
            s.apply_update(c)
    ref = whole.plane("estimate", as_double=True)
    for s in shards:
        x = s.engine.plane("estimate", as_double=True)
        assert float(np.sqrt(np.mean((x - ref) ** 2) / np.mean(ref ** 2))) <= tol
    np.testing.assert_array_equal(shards[0].engine.plane("estimate"), shards[1].engine.plane("estimate"))


def _nccl_single_rank(ds, form, capture):
    """One NCCL rank holding every exposure: ShardedSolver's iteration (the
    engine's own correction plane all-reduced in place on the engine's
    stream between the two non-blocking halves), eager or replayed from one
    captured CUDA graph."""
    import datetime
    import torch.distributed as dist
    from updc_b200.sharded import ShardedSolver, open_engine_shard
    w = ds.workload
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        shard = open_engine_shard(str(ds.manifest), w.W, w.H, w.iw, w.ih, w.nexp, 0, 1, form=form)
        solver = ShardedSolver(shard, dist)
        if capture:
            solver.capture()
        recs = solver.iterate(4)
        solver.release()
        x = shard.engine.plane("estimate")
        shard.engine.close()
        return x, recs
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
@pytest.mark.parametrize("capture", [False, True])
def test_nccl_shard_iteration_matches_engine(engine_lib, datasets, capture):
    """With one rank the NCCL sum is the identity, so the sharded iteration
    (zero-copy correction plane, collective on the engine's stream, and
    optionally the whole iteration captured in a CUDA graph with the NCCL
    call) must equal the engine's own iterations bit for bit."""
    from updc_b200.engine import Engine
    ds = datasets("c0")
    w = ds.workload
    x, recs = _nccl_single_rank(ds, "fp32", capture)
    e = Engine(form="fp32", use_graph=False)
    e.load(str(ds.manifest), w.W, w.H, w.iw, w.ih, w.nexp).setup()
    st = e.iterate(4)
    np.testing.assert_array_equal(x, e.plane("estimate"))
    assert [r["signed_sum"] for r in recs] == [s.signed_sum for s in st]
    assert [r["negative"] for r in recs] == [s.negative for s in st]
    e.close()


@pytest.mark.gpu
@pytest.mark.parametrize("form,tol", [("fp64", 1e-12), ("fp32", 1e-5)])
def test_shard_setup_alone_matches_the_whole_field(engine_lib, datasets, form, tol):
    """Two exposure shards each set up alone (their own LinkMaps and PSF
    spectra only) on one GPU: their partial coverage, drizzle sums and
    denominator summed on the device, then finish_shard_setup; the drizzle
    estimate, coverage and denominator equal the whole field's to rounding,
    and so does x after iterating with the summed partial corrections."""
    from updc_b200.engine import Engine
    from updc_b200.sharded import EngineShard, _DevicePlane
    ds = datasets("c0")
    w = ds.workload
    whole = Engine(form=form, use_graph=False)
    whole.load(str(ds.manifest), w.W, w.H, w.iw, w.ih, w.nexp).setup()
    engines = []
    for r in range(2):
        e = Engine(form=form, use_graph=False)
        e.load(str(ds.manifest), w.W, w.H, w.iw, w.ih, w.nexp)
        e.set_active_exposures(*shard_range(w.nexp, r, 2))
        e.setup()
        with pytest.raises(Exception):
            e.iterate(1)                                   # refused until the sums are in
        engines.append(e)
    torch.cuda.synchronize()
    dt = torch.float64 if form == "fp64" else torch.float32
    for name in ("coverage", "estimate", "correction", "denominator"):
        planes = [torch.as_tensor(_DevicePlane(e.plane_device_pointer(name), (w.H, w.W), form == "fp64"),
                                  device="cuda") for e in engines]
        total = planes[0] + planes[1]
        for p in planes:
            p.copy_(total)
        assert total.dtype == dt
    torch.cuda.synchronize()
    for e in engines:
        e.finish_shard_setup()
    for name in ("estimate", "coverage", "denominator"):
        ref = whole.plane(name, as_double=True)
        for e in engines:
            assert rel_rms(e.plane(name, as_double=True), ref) <= tol, name
    assert engines[0].max_sensitivity == pytest.approx(whole.max_sensitivity, rel=10 * tol)
    shards = [EngineShard(e, *shard_range(w.nexp, r, 2)) for r, e in enumerate(engines)]
    cur = torch.cuda.current_stream()
    for _ in range(3):
        whole.iterate(1)
        parts = [s.partial_correction() for s in shards]
        for s in shards:
            cur.wait_stream(s.stream)
        c = parts[0] + parts[1]
        for s in shards:
            s.stream.wait_stream(cur)
            s.apply_update(c)
    ref = whole.plane("estimate", as_double=True)
    for s in shards:
        assert rel_rms(s.engine.plane("estimate", as_double=True), ref) <= 10 * tol
        s.engine.close()
    whole.close()
