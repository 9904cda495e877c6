"""GPU parity of every stage of the B200 engine against the oracle, through the C ABI.

Integer and ordered-FP32 stages are compared bit for bit (LinkMap bytes and
decode, weight normalisation, drizzle, the detector loop and its adjoint
gather, the update); FFT-based stages against the FP64 oracle with the
tolerances written in each test; whole solves against the compiled
reference core.
"""
from __future__ import annotations

import csv
import filecmp
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import fft_shape_for, rel_rms

pytestmark = pytest.mark.gpu


def _engine(ds, form="fp32", **kw):
    from updc_b200.engine import Engine
    w = ds.workload
    e = Engine(form=form, **kw)
    e.load(str(ds.manifest), w.W, w.H, w.iw, w.ih, w.nexp)
    e.setup()
    return e


def _oracle_solver(oracle, ds, precision=32, fft_shape=None):
    w = ds.workload
    fw, fh = fft_shape or fft_shape_for(ds)
    return oracle.Solver(str(ds.manifest), w.W, w.H, w.iw, w.ih, w.nexp, fw, fh, precision=precision)


# ---------------------------------------------------------------------------- geometry / LinkMap
def test_self_test_on_device(engine_lib):
    from updc_b200.engine import self_test
    assert "OK" in self_test()


def test_bounded_device_wait_times_out_and_context_stays_usable(engine_lib, datasets):
    """Failure detection without a fault: a bounded mbarrier wait that nothing
    completes (no copy issued) runs out, the block returns together and the
    host raises "device wait timed out"; the context stays usable, so an
    engine solve afterwards runs normally."""
    from updc_b200 import _lib
    from updc_b200.engine import UpdcError
    L = _lib.load()
    for polls in (1, 1000):
        with pytest.raises(UpdcError, match="device wait timed out"):
            _lib.check(L.updc_device_wait_check(polls))
    e = _engine(datasets("small"))
    st = e.iterate(2)
    assert len(st) == 2 and np.isfinite(e.plane("estimate")).all()
    e.close()


@pytest.mark.parametrize("name", ["small", "abs32", "c0", "medium"])
def test_linkmap_build_byte_identical(engine_lib, oracle, datasets, name, tmp_path):
    from updc_b200.engine import build_linkmap
    ds = datasets(name)
    w = ds.workload
    for k, row in enumerate(ds.rows):
        mine = tmp_path / f"gpu_{k}.links"
        ref = tmp_path / f"orc_{k}.links"
        nl, enc = build_linkmap(row.vertices, mine, w.iw, w.ih, w.W, w.H)
        onl, oenc = oracle.linkmap_build(row.vertices, w.iw, w.ih, w.W, w.H, str(ref))
        assert (nl, enc) == (onl, oenc)
        assert filecmp.cmp(mine, ref, shallow=False), f"exposure {k}: LinkMap bytes differ"
    if name == "abs32":
        assert enc == 1


@pytest.mark.parametrize("name", ["small", "abs32", "c0"])
def test_linkmap_decode_bit_exact(engine_lib, oracle, datasets, name):
    ds = datasets(name)
    w = ds.workload
    e = _engine(ds, form="fp32-reference")
    for k, row in enumerate(ds.rows):
        off, tgt, frac, enc = oracle.linkmap_decode(row.links, w.iw, w.ih, w.W, w.H)
        assert e.link_encoding(k) == enc
        assert e.link_count(k) == len(tgt)
        np.testing.assert_array_equal(e.decode_links(k), tgt)


# ---------------------------------------------------------------------------- setup stages
@pytest.mark.parametrize("form", ["fp32-reference", "fp32"])
def test_setup_planes_bit_exact(engine_lib, oracle, datasets, form):
    """Weight scale, masked/normalised SCI/WHT, coverage and the drizzle x0."""
    ds = datasets("c0")
    e = _engine(ds, form=form)
    s = _oracle_solver(oracle, ds)
    assert np.float32(e.weight_scale) == np.float32(s.weight_scale)
    for k in range(ds.workload.nexp):
        np.testing.assert_array_equal(e.plane("science", k), s.sci[k])
        np.testing.assert_array_equal(e.plane("weight", k), s.wht[k])
    np.testing.assert_array_equal(e.plane("coverage"), s.coverage)
    np.testing.assert_array_equal(e.plane("estimate"), s.estimate)


@pytest.mark.parametrize("form,tol", [("fp32", 2e-6), ("fp32-reference", 2e-5), ("fp64", 1e-12)])
def test_denominator_vs_fp64_oracle(engine_lib, oracle, datasets, form, tol):
    """D = sum_k H_k^T W_k against the FP64 oracle (relative RMS <= tol)."""
    ds = datasets("c0")
    e = _engine(ds, form=form)
    s64 = _oracle_solver(oracle, ds, precision=64)
    d = e.plane("denominator", as_double=True)
    assert rel_rms(d, s64.denominator) <= tol
    assert abs(e.max_sensitivity - s64.max_sensitivity) <= 10 * tol * s64.max_sensitivity


@pytest.mark.parametrize("form,tol", [("fp32", 2e-6), ("fp64", 1e-12)])
def test_forward_model_vs_fp64_oracle(engine_lib, oracle, datasets, form, tol):
    """blur_k = crop(C2R(R2C(pad(x)) K_k))/nf for every exposure (relative RMS <= tol)."""
    ds = datasets("c0")
    e = _engine(ds, form=form)
    s64 = _oracle_solver(oracle, ds, precision=64)
    e.set_plane("estimate", s64.estimate)
    e.stage_forward()
    for k in range(ds.workload.nexp):
        ref = s64.forward_blur(k)
        assert rel_rms(e.plane("blur", k, as_double=True), ref) <= tol


@pytest.mark.parametrize("form,tol", [("fp32", 2e-6), ("fp64", 1e-12)])
def test_minimum_fft_shape_rules(engine_lib, oracle, datasets, form, tol):
    """The default shape is the smallest 7-smooth one >= W + pw/2 (even width),
    the fft_linear one the reference's smallest >= W + pw - 1; the forward
    model on the smaller shape equals the FP64 oracle's on the reference's
    shape, and so does the denominator (the kept window is exact)."""
    from conftest import crop_min_shape
    ds = datasets("medium")
    w = ds.workload
    s64 = _oracle_solver(oracle, ds, precision=64)
    lin = _engine(ds, form=form, fft_linear=True)
    assert lin.fft_shape == fft_shape_for(ds)
    crop = _engine(ds, form=form)
    cw, ch = crop_min_shape(ds)
    fw, fh = crop.fft_shape
    assert fw % 2 == 0 and fw >= cw and fh >= ch
    assert fw < lin.fft_shape[0] and fh < lin.fft_shape[1]
    assert all(oracle.next_fast_size(v) == v for v in (fw, fh))
    assert rel_rms(crop.plane("denominator", as_double=True), s64.denominator) <= tol
    for e in (crop, lin):
        e.set_plane("estimate", s64.estimate)
        e.stage_forward()
        for k in range(w.nexp):
            assert rel_rms(e.plane("blur", k, as_double=True), s64.forward_blur(k)) <= tol
    crop.close()
    lin.close()


@pytest.mark.parametrize("form,tol", [("fp32", 2e-6), ("fp64", 1e-12)])
def test_large_column_transforms(engine_lib, oracle, datasets, form, tol):
    """FFT heights above the small column capacity (the 11264-point kernels;
    FP64 keeps X-hat and the adjoint accumulator in global memory): forward
    model and two iterations against the FP64 oracle on the same shape."""
    ds = datasets("c0")
    shape = (288, 9720)
    e = _engine(ds, form=form, fft_shape=shape)
    assert e.fft_shape == shape
    s64 = _oracle_solver(oracle, ds, precision=64, fft_shape=shape)
    e.set_plane("estimate", s64.estimate)
    e.stage_forward()
    for k in range(ds.workload.nexp):
        assert rel_rms(e.plane("blur", k, as_double=True), s64.forward_blur(k)) <= tol
    e2 = _engine(ds, form=form, fft_shape=shape)
    e2.iterate(2)
    s64.iterate(2)
    assert rel_rms(e2.plane("estimate", as_double=True), s64.estimate) <= 10 * tol


@pytest.mark.parametrize("shape", [(12000, 288), (288, 12000)])
@pytest.mark.parametrize("form,tol", [("fp32", 2e-6), ("fp64", 1e-12)])
def test_long_row_transforms(engine_lib, oracle, datasets, form, tol, shape):
    """FFT shapes beyond one block's transform: rows of FW/2 = 6000 > 5632
    complex points (four-step rows, 6000 = 10 x 600) and columns of
    FH = 12000 > 11264 points (four-step columns, 12000 = 10 x 1200, with the
    OTF product and the cross-exposure sum as separate passes): forward
    model, denominator and two iterations against the FP64 oracle on the same
    shape."""
    ds = datasets("c0")
    e = _engine(ds, form=form, fft_shape=shape)
    assert e.fft_shape == shape
    s64 = _oracle_solver(oracle, ds, precision=64, fft_shape=shape)
    assert rel_rms(e.plane("denominator", as_double=True), s64.denominator) <= tol
    e.set_plane("estimate", s64.estimate)
    e.stage_forward()
    for k in range(ds.workload.nexp):
        assert rel_rms(e.plane("blur", k, as_double=True), s64.forward_blur(k)) <= tol
    e2 = _engine(ds, form=form, fft_shape=shape)
    e2.iterate(2)
    s64.iterate(2)
    assert rel_rms(e2.plane("estimate", as_double=True), s64.estimate) <= 10 * tol
    e.close()
    e2.close()


def test_wide_abs32_field_matches_reference_core(engine_lib, reference_binary, datasets, tmp_path):
    """The reference's ABS32 validation geometry (a 66000-pixel-wide target,
    docs/V17_VALIDATION.md): ABS32 LinkMaps built on the GPU, rows of
    33075 complex points through the four-step kernels; the whole solve within
    1e-5 relative RMS of the reference core, with the same FreezeMu counts."""
    ds = datasets("abs32_wide")
    w = ds.workload
    xref, rows = _reference_run(reference_binary, ds, w.iterations, tmp_path)
    e = _engine(ds, form="fp32")
    assert e.fft_shape[0] // 2 > 5632
    assert all(e.link_encoding(k) == 1 for k in range(w.nexp))
    st = e.iterate(w.iterations)
    assert rel_rms(e.plane("estimate"), xref) <= 1e-5
    assert [(int(s.new_frozen[k]), int(s.total_frozen[k])) for s in st for k in range(w.nexp)] == \
        [(int(r["n_new_frozen"]), int(r["n_total_frozen"])) for r in rows]
    e.close()


@pytest.mark.parametrize("shape", [(3600, 300), (3840, 288), (9072, 288)])
@pytest.mark.parametrize("form,tol", [("fp32", 2e-6), ("fp64", 1e-12)])
def test_two_row_tiles(engine_lib, oracle, datasets, form, tol, shape):
    """FFT widths whose rows go two to a tile (the row kernels' two-row
    instantiation, with TMA tiles).  3600 x 300 gets unpadded row and column
    plans (the no-padding instantiations), 3840 x 288 padded ones; the FP32
    rows of 9072 x 288 (4536 complex points, more than half a block) take
    the 1024-thread wide-row tiles.  Forward model and two iterations against
    the FP64 oracle on the same shape."""
    ds = datasets("c0")
    e = _engine(ds, form=form, fft_shape=shape)
    assert e.fft_shape == shape
    s64 = _oracle_solver(oracle, ds, precision=64, fft_shape=shape)
    e.set_plane("estimate", s64.estimate)
    e.stage_forward()
    for k in range(ds.workload.nexp):
        assert rel_rms(e.plane("blur", k, as_double=True), s64.forward_blur(k)) <= tol
    e2 = _engine(ds, form=form, fft_shape=shape)
    e2.iterate(2)
    s64.iterate(2)
    assert rel_rms(e2.plane("estimate", as_double=True), s64.estimate) <= 10 * tol


@pytest.mark.parametrize("form", ["fp32", "fp32-reference"])
def test_compile_time_transforms_and_fused_gather(engine_lib, oracle, datasets, form):
    """A 5040 x 5040 FFT, the shape whose row (2520 = 14 x 12 x 15) and column
    (5040 = 21 x 16 x 15) transforms are compiled for their radix sequence,
    and whose iteration gathers S^T(wr) inside the scatter row R2C (no scatter
    plane).  The forward model against the FP64 oracle; iterations through
    the fused kernel bit-identical to the stage hooks' separate gather
    (k_scatter_t) and row R2C; and x after two iterations within 1e-5 of the
    same form on the default (smallest) shape, since both keep the exact
    linear convolution."""
    ds = datasets("c0")
    w = ds.workload
    shape = (5040, 5040)
    a = _engine(ds, form=form, fft_shape=shape, use_graph=False)
    assert a.fft_shape == shape
    assert a.fft_radices(0) == [14, 12, 15] and a.fft_radices(1) == [21, 16, 15]
    s64 = _oracle_solver(oracle, ds, precision=64, fft_shape=shape)
    x0 = a.plane("estimate")
    a.set_plane("estimate", s64.estimate)
    a.stage_forward()
    for k in (0, w.nexp - 1):
        assert rel_rms(a.plane("blur", k, as_double=True), s64.forward_blur(k)) <= 2e-6
    a.set_plane("estimate", x0)
    b = _engine(ds, form=form, fft_shape=shape, use_graph=False)
    for it in range(2):
        a.iterate(1)
        b.stage_forward()
        b.stage_detector()
        b.stage_correction()
        b.stage_update()
        np.testing.assert_array_equal(a.plane("estimate"), b.plane("estimate"), err_msg=f"iteration {it + 1}")
    small = _engine(ds, form=form)
    assert small.fft_shape != shape
    small.iterate(2)
    assert rel_rms(a.plane("estimate"), small.plane("estimate")) <= 1e-5
    for e in (a, b, small):
        e.close()


# ---------------------------------------------------------------------------- detector / update
@pytest.mark.parametrize("name,background", [("c0", None), ("c0", -100.0), ("abs32", None)])
def test_detector_and_adjoint_gather_bit_exact(engine_lib, oracle, datasets, name, background):
    """Same blur in, same scatter out: the fused detector loop, FreezeMu and the
    target-major gather reproduce updc_core.c:1152-1177 bit for bit, for a
    DELTA16 and an ABS32 LinkMap."""
    ds = datasets(name, background)
    e = _engine(ds, form="fp32-reference")
    s = _oracle_solver(oracle, ds)
    blurs = [s.forward_blur(k) for k in range(ds.workload.nexp)]
    for k, b in enumerate(blurs):
        e.set_plane("blur", b, k)
    new, tot, mn = e.stage_detector()
    for k, b in enumerate(blurs):
        sc, nn, nt, m = s.detector(k, b)
        np.testing.assert_array_equal(e.plane("scatter", k), sc)
        assert (int(new[k]), int(tot[k])) == (nn, nt)
        assert np.float32(mn[k]) == np.float32(m)
        np.testing.assert_array_equal(e.plane("frozen", k), s.frozen[k])
    if background is not None:
        assert int(tot.sum()) > 0


def test_update_bit_exact(engine_lib, oracle, datasets):
    ds = datasets("c0")
    e = _engine(ds, form="fp32-reference")
    s = _oracle_solver(oracle, ds)
    x0 = s.estimate.copy()
    s.iterate(1)
    # feed the oracle's correction and denominator, start from the same x
    e.set_plane("estimate", x0)
    e.set_plane("correction", s.correction)
    e.set_plane("denominator", s.denominator)
    total, neg = e.stage_update()
    np.testing.assert_array_equal(e.plane("estimate"), s.estimate)
    assert neg == int((s.estimate < 0).sum())


# ---------------------------------------------------------------------------- whole solves
def _reference_run(ref_bin, ds, iterations, tmp_path, prefix="ref"):
    args = ds.engine_args(iterations=iterations, prefix=prefix).argv()
    r = subprocess.run([str(ref_bin), *args], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    w = ds.workload
    x = np.fromfile(f"{ds.directory}/{prefix}_{iterations:02d}.bin", np.float32).reshape(w.H, w.W)
    with open(f"{ds.directory}/{prefix}_mufreeze.csv") as f:
        rows = list(csv.DictReader(f))
    return x, rows


@pytest.mark.parametrize("name", ["c0", "medium"])
def test_fp32_solve_matches_reference(engine_lib, reference_binary, datasets, name, tmp_path):
    """FP32 form after the workload's iterations within 1e-5 relative RMS of
    the reference core, with the reference's FreezeMu counts, and the
    min_raw_mu column of its freeze CSV (updc_core.c:1429, "%.9g" of the
    FP32 minimum) within 1e-5 relative for both FP32 forms.  The column cannot
    match byte for byte: raw_mu is a sum over blurred pixels, and this FFT
    rounds differently from the reference's, so the minima differ in their
    last bits (the detector itself is bit-exact given the same blur)."""
    ds = datasets(name)
    w = ds.workload
    xref, rows = _reference_run(reference_binary, ds, w.iterations, tmp_path)
    for form in ("fp32", "fp32-reference"):
        e = _engine(ds, form=form)
        st = e.iterate(w.iterations)
        x = e.plane("estimate")
        if form == "fp32":
            assert rel_rms(x, xref) <= 1e-5
        mine = [(int(s.new_frozen[k]), int(s.total_frozen[k]), float(np.float32(s.min_raw_mu[k])))
                for s in st for k in range(w.nexp)]
        assert [(a, b) for a, b, _ in mine] == [(int(r["n_new_frozen"]), int(r["n_total_frozen"])) for r in rows]
        ref_mu = np.array([float(r["min_raw_mu"]) for r in rows])
        np.testing.assert_allclose(np.array([m for _, _, m in mine]), ref_mu, rtol=1e-5)
        e.close()


def test_fp64_solve_matches_fp64_oracle(engine_lib, oracle, datasets):
    ds = datasets("c0")
    w = ds.workload
    s64 = _oracle_solver(oracle, ds, precision=64)
    s64.iterate(w.iterations)
    e = _engine(ds, form="fp64")
    e.iterate(w.iterations)
    assert rel_rms(e.plane("estimate", as_double=True), s64.estimate) <= 1e-12


def test_forced_freeze_rows_match_reference(engine_lib, reference_binary, datasets, tmp_path):
    """Background -100 (the reference smoke test's forced FreezeMu): per-iteration
    freeze counts equal the reference core's to within 0.1% of the frozen
    total, and the totals accumulate.  Exact equality is not expected here:
    with the -100 background many raw_mu sit within FFT rounding of the
    freeze threshold (raw_mu <= 0), and this FFT rounds differently from the
    reference's, so a few pixels can freeze one iteration earlier or later.
    Given the same blur planes the freeze decisions are bit-exact
    (test_detector_and_adjoint_gather_bit_exact), and on the reference's own
    forced-freeze fixture the counts match exactly (test_golden)."""
    ds = datasets("c0", -100.0)
    w = ds.workload
    iters = 4
    xref, rows = _reference_run(reference_binary, ds, iters, tmp_path)
    e = _engine(ds, form="fp32-reference")
    st = e.iterate(iters)
    mine = [(int(s.new_frozen[k]), int(s.total_frozen[k])) for s in st for k in range(w.nexp)]
    theirs = [(int(r["n_new_frozen"]), int(r["n_total_frozen"])) for r in rows]
    mismatch = sum(abs(a[1] - b[1]) for a, b in zip(mine, theirs))
    total = sum(b[1] for b in theirs)
    assert total > 0
    assert mismatch <= max(2, total // 1000), (mine, theirs)
    for k in range(w.nexp):
        assert st[0].total_frozen[k] == st[0].new_frozen[k]
        assert st[1].total_frozen[k] == st[0].total_frozen[k] + st[1].new_frozen[k]


def test_graph_and_eager_paths_identical(engine_lib, datasets):
    """The CUDA-graph replay and eager launches give bit-identical results, and
    two runs are bit-identical (no float atomics anywhere)."""
    ds = datasets("c0")
    outs = []
    for graph in (True, False, True):
        e = _engine(ds, form="fp32", use_graph=graph)
        e.iterate(5, check_each=False)
        outs.append(e.plane("estimate"))
    np.testing.assert_array_equal(outs[0], outs[1])
    np.testing.assert_array_equal(outs[0], outs[2])


def test_whole_loop_graph_matches_per_iteration_launches(engine_lib, datasets):
    """iterate(n) without per-iteration checks replays one graph of all n
    iterations; its estimate and per-iteration records equal those of n
    checked single-iteration launches."""
    ds = datasets("c0", background=-100.0)        # FreezeMu counters change per iteration
    a = _engine(ds, form="fp32")
    b = _engine(ds, form="fp32")
    ra = a.iterate(6, check_each=False)
    rb = [b.iterate(1, check_each=True)[0] for _ in range(6)]
    np.testing.assert_array_equal(a.plane("estimate"), b.plane("estimate"))
    for x, y in zip(ra, rb):
        assert x.signed_sum == y.signed_sum and x.negative == y.negative
        np.testing.assert_array_equal(x.new_frozen, y.new_frozen)
        np.testing.assert_array_equal(x.total_frozen, y.total_frozen)
        assert x.seconds > 0
    assert int(rb[-1].total_frozen.sum()) > 0
    ra2 = a.iterate(6, check_each=False)          # the cached loop graph again
    rb2 = [b.iterate(1, check_each=True)[0] for _ in range(6)]
    np.testing.assert_array_equal(a.plane("estimate"), b.plane("estimate"))
    assert [r.signed_sum for r in ra2] == [r.signed_sum for r in rb2]


def test_dropin_executable(engine_lib, reference_binary, datasets, tmp_path):
    """updc_b200/bin/updc_jwst_c with the 18-argument contract writes the
    reference's outputs; the WHT product (coverage x weight scale) is
    bit-identical and x is within 1e-5 relative RMS."""
    from updc_b200 import _lib
    ds = datasets("c0")
    w = ds.workload
    iters = 5
    xref, rows_ref = _reference_run(reference_binary, ds, iters, tmp_path, prefix="refd")
    args = ds.engine_args(iterations=iters, prefix="b200", save_every=2).argv()
    r = subprocess.run([str(_lib.EXE_PATH), *args], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    d = Path(ds.directory)
    assert (d / "b200_02.bin").is_file() and (d / "b200_04.bin").is_file() and (d / "b200_05.bin").is_file()
    x = np.fromfile(d / "b200_05.bin", np.float32).reshape(w.H, w.W)
    assert rel_rms(x, xref) <= 1e-5
    wht = np.fromfile(d / "b200_wht.bin", np.float32)
    wref = np.fromfile(d / "refd_wht.bin", np.float32)
    np.testing.assert_array_equal(wht, wref)
    with open(d / "b200_mufreeze.csv") as f:
        rows = list(csv.DictReader(f))
    assert len(rows) == iters * w.nexp
    assert list(rows[0].keys()) == list(rows_ref[0].keys())
    timing = (d / "b200_timing.csv").read_text().splitlines()
    assert timing[0] == "stage,wall_seconds" and any(t.startswith(f"iteration_{iters:02d}_total") for t in timing)
    st = subprocess.run([str(_lib.EXE_PATH), "--self-test"], capture_output=True, text=True)
    assert st.returncode == 0


def test_error_negative_yeff(engine_lib, datasets, tmp_path):
    """A pedestal too small for the data fails setup with the reference's message."""
    from updc_b200 import handoff
    from updc_b200.engine import Engine, UpdcError
    ds = datasets("small")
    rows = [handoff.ExposureRow(**{**r.__dict__}) for r in ds.rows]
    for r in rows:
        r.pedestal = 0.0
    m = tmp_path / "manifest_bad.txt"
    handoff.write_manifest(m, rows)
    w = ds.workload
    e = Engine(form="fp32")
    e.load(str(m), w.W, w.H, w.iw, w.ih, w.nexp)
    with pytest.raises(UpdcError, match="negative/non-finite y_eff reached solver"):
        e.setup()


@pytest.mark.parametrize("form", ["fp32", "fp64"])
def test_checkpoint_resume_continues_exactly(engine_lib, datasets, form, tmp_path):
    """3 iterations, save, a fresh engine loads the state and runs 3 more:
    identical to 6 straight iterations (estimate and FreezeMu masks), under
    forced FreezeMu so the masks matter."""
    from updc_b200 import _lib
    ds = datasets("c0", background=-100.0)
    straight = _engine(ds, form=form)
    straight.iterate(6)
    first = _engine(ds, form=form)
    first.iterate(3)
    first.save_state(tmp_path / "state.bin")
    second = _engine(ds, form=form)
    assert second.load_state(tmp_path / "state.bin") == 3
    second.iterate(3)
    np.testing.assert_array_equal(second.plane("estimate", as_double=True), straight.plane("estimate", as_double=True))
    for k in range(ds.workload.nexp):
        np.testing.assert_array_equal(second.plane("frozen", k), straight.plane("frozen", k))
    other = _engine(datasets("small"), form=form)
    with pytest.raises(_lib.UpdcError, match="does not match"):
        other.load_state(tmp_path / "state.bin")
