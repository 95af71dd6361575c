"""Plain (FP32 CUDA-core) engine on the GPU versus the CPU oracle, through the C ABI."""
import ctypes as C

import numpy as np
import pytest

from gnomon_b200 import _lib, synth
from gnomon_b200.pipeline import PipelineContext, PipelineError, ScoreCheckpoint, run
from gnomon_b200.prepare import PreparationResult
from helpers import GOLDEN, case_prep, cohort_prep, expected_final, known_answer_cases, synth_case
from oracle import oracle

pytestmark = pytest.mark.gpu
PLAIN = _lib.ENGINE_PLAIN
CASES = known_answer_cases()["engine_cases"]


def host_run(prep, rows, **kw):
    return run(PipelineContext(prep), np.ascontiguousarray(rows).reshape(-1), engine=PLAIN, **kw)


def assert_parity(got, want_ref, want_ext=None):
    s, c = got
    rs, rc = want_ref
    np.testing.assert_array_equal(c, rc)                       # counts: bit exact
    ok = oracle.within_reference_tolerance(s, rs)              # gpu_tests.rs:135-147
    assert ok.all(), f"{(~ok).sum()} cells outside 1e-6; worst {oracle.rel_err(s, rs).max():.3e}"
    if want_ext is not None:   # FP32 stage sums vs the extended-precision oracle
        assert oracle.rel_err(s, want_ext[0]).max() < 1e-6


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_known_answers(cuda, case):
    prep, rows = case_prep(case)
    s, c = host_run(prep, rows)
    ws, wc = expected_final(case, prep)
    np.testing.assert_allclose(s, ws, rtol=0, atol=1e-9)
    np.testing.assert_array_equal(c, wc)


def test_reference_gpu_tests_cohort(cuda):
    """score/tests/gpu_tests.rs:78-170: GPU vs CPU on the deterministic cohort,
    compared the way the reference compares them: .sscore AVG within 1e-6 abs
    or rel, MISSING_PCT within 1e-6, counts exact."""
    from gnomon_b200.sscore import averages
    prep, rows = cohort_prep(16)
    s, c = host_run(prep, rows)
    rs, rc = oracle.score_reference(rows, prep, threads=4)
    np.testing.assert_array_equal(c, rc)
    avg, pct = averages(s, c, prep.score_variant_counts)
    ravg, rpct = averages(rs, rc, prep.score_variant_counts)
    assert oracle.within_reference_tolerance(avg, ravg).all()
    assert np.abs(pct - rpct).max() <= 1e-6
    # raw sums: weights of magnitude ~1 put FP32 stage rounding near 1e-6 of |sum|
    assert oracle.rel_err(s, oracle.score_extended(rows, prep)[0]).max() < 5e-6


def test_plain_config_full_size(cuda):
    """2,000 samples x 50,000 variants, one score, 1% missing, 10% flipped."""
    _, prep, rows, _ = synth_case(2_000, 50_000)
    got = host_run(prep, rows)
    assert_parity(got, oracle.score_reference(rows, prep, threads=8),
                  oracle.score_extended(rows, prep))
    assert got[1].sum() > 0


@pytest.mark.parametrize("people,variants", [(1, 1), (3, 47), (4, 48), (5, 49), (4095, 97),
                                             (4097, 145), (8197, 50), (1030, 1000)])
def test_edge_shapes(cuda, people, variants):
    _, prep, rows, _ = synth_case(people, variants, seed_offset=people + variants)
    assert_parity(host_run(prep, rows), oracle.score_reference(rows, prep, threads=2),
                  oracle.score_extended(rows, prep))


def test_multi_score_uneven_membership(cuda):
    _, prep, rows, _ = synth_case(3000, 2000, scores=5, config="batched_100k_x_500k_k512")
    assert len(set(np.diff(prep.sparse_row_offsets.astype(np.int64)))) > 1
    assert_parity(host_run(prep, rows), oracle.score_reference(rows, prep, threads=4),
                  oracle.score_extended(rows, prep))


def test_keep_subset_and_row_map(cuda):
    rng = np.random.default_rng(7)
    _, prep, rows, _ = synth_case(5000, 900, scores=2, config="diff_20k_x_200k_k16")
    # shuffle the .bed row order; required_bim_indices maps reconciled -> bed row
    perm = rng.permutation(900)
    bed = np.empty_like(rows)
    bed[perm] = rows
    keep = rng.choice(5000, 1234, replace=False).astype(np.uint32)
    p2 = PreparationResult(prep.sparse_weights, prep.sparse_missing_corrections,
                           prep.sparse_score_columns, prep.sparse_row_offsets, prep.score_names,
                           5000, required_bim_indices=perm.astype(np.uint64),
                           output_idx_to_fam_idx=keep)
    got = host_run(p2, bed)
    assert_parity(got, oracle.score_reference(rows, p2, threads=4),
                  oracle.score_extended(rows, p2))


def test_streaming_blocks_and_resume(cuda):
    _, prep, rows, _ = synth_case(2500, 1000)
    full = host_run(prep, rows)
    streamed = host_run(prep, rows, block_variants=100)
    np.testing.assert_array_equal(streamed[1], full[1])
    # block boundaries move the FP32 stage grouping: agreement at FP32 level
    assert oracle.rel_err(streamed[0], full[0]).max() < 1e-6
    seen = []
    host_run(prep, rows, block_variants=300, on_block=lambda n, s, c: seen.append(n))
    assert seen == [300, 600, 900, 1000]
    # resume: first 400 variants from a checkpoint computed on the CPU oracle
    head = PreparationResult(prep.sparse_weights[:400], prep.sparse_missing_corrections[:400],
                             prep.sparse_score_columns[:400], prep.sparse_row_offsets[:401],
                             prep.score_names, 2500, baseline=prep.baseline)
    hs, hc = oracle.score_extended(rows[:400], head)
    ctx = PipelineContext(prep, ScoreCheckpoint(400, hs, hc))
    got = run(ctx, rows.reshape(-1), engine=PLAIN)
    np.testing.assert_array_equal(got[1], full[1])
    assert oracle.rel_err(got[0], full[0]).max() < 1e-6


def test_rows_without_cells(cuda):
    _, prep, rows, _ = synth_case(700, 200, scores=3, config="diff_20k_x_200k_k16")
    offs = prep.sparse_row_offsets.astype(np.int64)
    keep_rows = np.ones(200, bool)
    keep_rows[::7] = False   # every 7th variant loses all its cells (e.g. a complex-only row)
    sel = np.repeat(keep_rows, np.diff(offs))
    counts = np.where(keep_rows, np.diff(offs), 0)
    new_offs = np.zeros(201, np.uint64)
    np.cumsum(counts, out=new_offs[1:])
    p2 = PreparationResult(prep.sparse_weights[sel], prep.sparse_missing_corrections[sel],
                           prep.sparse_score_columns[sel], new_offs, prep.score_names, 700)
    assert_parity(host_run(p2, rows), oracle.score_reference(rows, p2, threads=2),
                  oracle.score_extended(rows, p2))


def test_truncated_bed_is_an_io_error(cuda):
    _, prep, rows, _ = synth_case(400, 100)
    with pytest.raises(PipelineError) as e:
        run(PipelineContext(prep), rows.reshape(-1)[:-5], engine=PLAIN)
    assert e.value.kind == "Io"


def test_device_api_matches_host_api(cuda):
    import torch
    from gnomon_b200.device import DevicePlan, row_pitch
    _, prep, rows, _ = synth_case(3333, 777, scores=2, config="diff_20k_x_200k_k16")
    pitch = row_pitch(prep.bytes_per_variant)
    dev = np.zeros((777, pitch), np.uint8)
    dev[:, :rows.shape[1]] = rows
    d_rows = torch.from_numpy(dev).cuda()
    plan = DevicePlan(prep, engine=PLAIN)
    s, c = plan.score(d_rows, pitch)
    plan.sync()
    host = host_run(prep, rows)
    np.testing.assert_array_equal(c.cpu().numpy().astype(np.uint32), host[1])
    np.testing.assert_array_equal(s.cpu().numpy(), host[0])
    assert plan.launches == 2 * 2   # one accumulate + one finalize launch per score


def test_decode_parity_ld_fixture_and_synthetic(cuda):
    import torch
    from gnomon_b200.device import decode
    z = np.load(GOLDEN / "ld_fixture.npz")
    rows, P = z["rows"], int(z["num_people"])
    for r, p in [(rows, P)] + [(synth_case(pp, 33)[2], pp) for pp in (1, 6, 4099)]:
        pitch = (r.shape[1] + 15) // 16 * 16
        dev = np.zeros((r.shape[0], pitch), np.uint8)
        dev[:, :r.shape[1]] = r
        got = decode(torch.from_numpy(dev).cuda(), pitch, r.shape[0], p).cpu().numpy()
        np.testing.assert_array_equal(got, oracle.decode(r, p))


@pytest.mark.parametrize("people", [1, 13, 4096, 50_000])
def test_gpu_generator_matches_numpy(cuda, people):
    import torch
    from gnomon_b200.device import row_pitch, synth_fill
    w = synth.WORKLOADS["bandwidth_50k_x_1m"]
    n, v0 = 37, 123_456
    thr = synth.variant_thresholds(w.seed, v0, n, w.p_lo, w.p_hi, w.missing_rate)
    pitch = row_pitch((people + 3) // 4)
    d = torch.full((n, pitch), 0xAB, dtype=torch.uint8, device="cuda")
    synth_fill(d, pitch, v0, n, people, thr, w.seed)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d.cpu().numpy(), synth.synth_rows(w.seed, v0, n, people, thr, pitch))
    # a person shard's columns: cohort people person_begin .. person_begin+people-1
    synth_fill(d, pitch, v0, n, people, thr, w.seed, person_begin=40_000)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d.cpu().numpy(), synth.synth_rows(w.seed, v0, n, people, thr, pitch,
                                                                    person_begin=40_000))


@pytest.mark.parametrize("engine", [PLAIN, _lib.ENGINE_TENSOR])
@pytest.mark.parametrize("subset", [False, True])
def test_person_shards_reassemble_cohort(cuda, engine, subset):
    """The multi-GPU layout run shard by shard on one device: every shard's
    rows are a byte-column slice, scored by its own plan; reassembled in output
    order they match the unsharded run (counts exact, sums at the reference
    tolerance; FP32 grouping may differ with the shard's launch shape)."""
    import torch
    from gnomon_b200 import sharding
    from gnomon_b200.device import DevicePlan, row_pitch
    _, prep, rows, _ = synth_case(9001, 700, scores=3, config="diff_20k_x_200k_k16")
    if subset:
        keep = np.random.default_rng(3).permutation(9001)[:6000].astype(np.uint32)
        prep = PreparationResult(prep.sparse_weights, prep.sparse_missing_corrections,
                                 prep.sparse_score_columns, prep.sparse_row_offsets,
                                 list(prep.score_names), 9001, output_idx_to_fam_idx=keep)

    def score(p, r):
        pitch = row_pitch(p.bytes_per_variant)
        dev = np.zeros((r.shape[0], pitch), np.uint8)
        dev[:, :r.shape[1]] = r
        plan = DevicePlan(p, engine=engine)
        s, c = plan.score(torch.from_numpy(dev).cuda(), pitch)
        plan.sync()
        out = s.cpu().numpy(), c.cpu().numpy()
        plan.close()
        return out

    s0, c0 = score(prep, rows)
    K = prep.num_scores
    world = 3
    s = np.zeros((prep.num_people_to_score, K))
    c = np.zeros((prep.num_people_to_score, K), np.uint32)
    for r in range(world):
        sh = sharding.make_shard(prep, r, world)
        ss, cc = score(sh.prep, sharding.slice_rows(rows, sh.start, sh.stop))
        s[sh.output_rows] = ss.reshape(-1, K)
        c[sh.output_rows] = cc.reshape(-1, K)
    np.testing.assert_array_equal(c.reshape(-1), c0.reshape(-1).astype(np.uint32))
    assert oracle.within_reference_tolerance(s.reshape(-1), s0.reshape(-1)).all()


@pytest.mark.parametrize("engine", [PLAIN, _lib.ENGINE_TENSOR])
def test_cuda_graph_replay_and_autotune(cuda, engine):
    """A captured scoring pass replays to the same result; autotuning picks a
    candidate shape and leaves results unchanged (up to FP32 regrouping)."""
    import torch
    from gnomon_b200.device import DevicePlan, row_pitch
    _, prep, rows, _ = synth_case(6000, 1500, scores=3, config="diff_20k_x_200k_k16")
    pitch = row_pitch(prep.bytes_per_variant)
    dev = np.zeros((1500, pitch), np.uint8)
    dev[:, :rows.shape[1]] = rows
    d_rows = torch.from_numpy(dev).cuda()
    plan = DevicePlan(prep, engine=engine)
    s0, c0 = plan.score(d_rows, pitch)
    plan.sync()
    s0, c0 = s0.cpu().numpy(), c0.cpu().numpy()
    graph, gs, gc = plan.capture(d_rows, pitch)
    for _ in range(3):
        gs.fill_(float("nan"))
        graph.replay()
        torch.cuda.synchronize()
        np.testing.assert_array_equal(gs.cpu().numpy(), s0)
        np.testing.assert_array_equal(gc.cpu().numpy(), c0)
    del graph
    shape = plan.autotune(d_rows, pitch)
    assert shape >= 0
    s1, c1 = plan.score(d_rows, pitch)
    plan.sync()
    np.testing.assert_array_equal(c1.cpu().numpy(), c0)
    assert oracle.rel_err(s1.cpu().numpy(), s0).max() < 1e-6
    plan.close()


@pytest.mark.parametrize("engine", [PLAIN, _lib.ENGINE_TENSOR])
def test_checkpoint_file_interrupt_and_resume(cuda, tmp_path, engine):
    """A run with a checkpoint path writes gnomon-format checkpoints after its
    variant blocks; a run aborted after the second block leaves the first
    block's checkpoint on disk (saves are at most every 30 s), and resuming
    from that file gives the uninterrupted result.  A completed run leaves a
    final checkpoint equal to its output."""
    from gnomon_b200 import checkpoint as ck
    _, prep, rows, _ = synth_case(2500, 1000, scores=3, config="diff_20k_x_200k_k16")
    flat = rows.reshape(-1)
    full = run(PipelineContext(prep), flat, engine=engine, block_variants=320)
    fp = ck.fingerprint_preparation(prep)
    path = tmp_path / "cohort.sscore.gnomon-checkpoint.bin"

    ctx = PipelineContext.with_checkpoint(prep, None, path, fp)
    with pytest.raises(PipelineError):
        run(ctx, flat, engine=engine, block_variants=320, on_block=lambda n, s, c: n < 640)
    saved = ck.load_checkpoint(path, fp, prep.num_people_to_score * prep.num_scores, 1000)
    assert saved.completed_variants == 320

    resumed = run(PipelineContext.with_checkpoint(prep, saved, path, fp), flat, engine=engine,
                  block_variants=320)
    np.testing.assert_array_equal(resumed[1], full[1])
    assert oracle.within_reference_tolerance(resumed[0], full[0]).all()
    final = ck.load_checkpoint(path, fp, prep.num_people_to_score * prep.num_scores, 1000)
    assert final.completed_variants == 1000
    np.testing.assert_array_equal(final.sum_scores, resumed[0])
    np.testing.assert_array_equal(final.missing_counts, resumed[1])


@pytest.mark.parametrize("engine", [PLAIN, _lib.ENGINE_TENSOR])
def test_complex_rules_after_the_engine(cuda, engine):
    """Multi-row loci are resolved on the CPU after the GPU pass, onto the
    engine's final sums (cuda_backend.rs:1465-1535): the result equals the
    engine's output followed by the per-person restatement of the resolver."""
    from gnomon_b200.complex import GroupedComplexRule, ScoreInfo
    from test_complex import _per_person_loop
    _, prep, rows, _ = synth_case(1500, 600, scores=3, config="diff_20k_x_200k_k16")
    rng = np.random.default_rng(5)
    rules = []
    for r in range(12):
        ctx_rows = rng.choice(600, 3, replace=False)
        ctxs = [(int(ctx_rows[0]), "A", "G"), (int(ctx_rows[1]), "G", "A"),
                (int(ctx_rows[2]), "A", "AT")]
        apps = [ScoreInfo("A", "G", float(np.float32(rng.normal())), k) for k in range(3)]
        rules.append(GroupedComplexRule(("2", 500 + r), ctxs, apps))
    base = run(PipelineContext(prep), rows.reshape(-1), engine=engine)
    p2 = PreparationResult(prep.sparse_weights, prep.sparse_missing_corrections,
                           prep.sparse_score_columns, prep.sparse_row_offsets, prep.score_names,
                           1500, complex_rules=rules)
    got = run(PipelineContext(p2), rows.reshape(-1), engine=engine)
    S, C = base[0].reshape(1500, 3).copy(), base[1].reshape(1500, 3).copy()
    codes = synth.unpack_codes(rows, 1500)
    _per_person_loop(rules, lambda v, f: int(codes[v, f]), np.arange(1500), 3, S, C)
    np.testing.assert_array_equal(got[0].reshape(1500, 3), S)
    np.testing.assert_array_equal(got[1].reshape(1500, 3), C)


@pytest.mark.parametrize("engine", [PLAIN, _lib.ENGINE_TENSOR])
def test_pinned_rows_staged_copy_and_repitch(cuda, engine):
    """Pinned .bed rows (the direct path) are copied back to back in 128 MB
    chunks and re-pitched on the device; the result equals the gathered path
    bit for bit, with one block, several blocks and a resume."""
    import torch
    from gnomon_b200.pipeline import BedSource
    _, prep, rows, _ = synth_case(10_001, 60_000, scores=2, config="diff_20k_x_200k_k16")
    assert rows.nbytes > (128 << 20)                 # more than one staging chunk
    ref = run(PipelineContext(prep), rows.reshape(-1), engine=engine)        # gathered
    host = torch.empty(rows.size, dtype=torch.uint8, pin_memory=True)
    host.copy_(torch.from_numpy(rows.reshape(-1)))
    src = BedSource(host.numpy())
    for kw in ({}, {"block_variants": 20_480}):
        got = run(PipelineContext(prep), src, engine=engine, **kw)
        np.testing.assert_array_equal(got[1], ref[1])
        if kw:
            assert oracle.within_reference_tolerance(got[0], ref[0]).all()
        else:
            np.testing.assert_array_equal(got[0], ref[0])
    # resume from the gathered path's state after 30,720 variants
    seen = {}
    run(PipelineContext(prep), rows.reshape(-1), engine=engine, block_variants=30_720,
        on_block=lambda n, s, c: seen.setdefault(n, (s.copy(), c.copy())))
    cp = ScoreCheckpoint(30_720, *seen[30_720])
    got = run(PipelineContext(prep, cp), src, engine=engine)
    np.testing.assert_array_equal(got[1], ref[1])
    assert oracle.within_reference_tolerance(got[0], ref[0]).all()
    e = _lib.gnm_error()
    assert _lib.load().gnm_release_cached_memory(0, C.byref(e)) == _lib.GNM_OK, e.message


def test_best_device_choice(cuda):
    """device = GNM_DEVICE_BEST probes every visible device and runs on the
    sm_100 device with the most free memory (score/cuda_backend.rs:894-991);
    the result equals the run on an explicit ordinal.  An ordinal that does
    not exist declines (the reference's Ok(None))."""
    import torch
    _, prep, rows, _ = synth_case(3000, 700, scores=2)
    flat = np.ascontiguousarray(rows).reshape(-1)
    best = run(PipelineContext(prep), flat, engine=PLAIN, device=_lib.DEVICE_BEST)
    zero = run(PipelineContext(prep), flat, engine=PLAIN, device=0)
    np.testing.assert_array_equal(best[1], zero[1])
    np.testing.assert_array_equal(best[0], zero[0])
    from gnomon_b200.pipeline import try_run_cuda
    assert try_run_cuda(PipelineContext(prep), flat, engine=PLAIN,
                        device=torch.cuda.device_count()) is None


def _c_rows_case(people, variants, scores, config="plain_2k_x_50k"):
    """Workload weights with rows from the threaded C generator (large cases)."""
    import os
    from gnomon_b200.prepare import from_workload
    w = synth.scaled(synth.WORKLOADS[config], people, variants, scores)
    thr = synth.variant_thresholds(w.seed, 0, variants, w.p_lo, w.p_hi, w.missing_rate)
    rows = oracle.synth_rows(w.seed, 0, variants, people, thr, w.bytes_per_variant,
                             threads=os.cpu_count() or 1)
    return from_workload(w), rows


@pytest.mark.parametrize("kernel", _lib.PLAIN_KERNELS)
@pytest.mark.parametrize("people,variants", [(20_001, 2_001), (2_000, 4_000), (9_000, 70),
                                             (130, 301)])
def test_every_plain_kernel_and_split(cuda, kernel, people, variants):
    """Each plain accumulate kernel (512 / 1024-byte tiles; 1024 / 2048-byte
    tiles with a producer warp), pinned with gnm_plan_set_shape at several
    split counts (one split, uneven splits, more splits than a full tile has
    CTA slots), against the restated reference engine: counts bit-exact, sums
    within the reference's 1e-6 metric.  Ragged last tiles and last stages
    included."""
    import torch
    from gnomon_b200.device import DevicePlan, row_pitch
    prep, rows = _c_rows_case(people, variants, 2)
    pitch = row_pitch(prep.bytes_per_variant)
    dev = np.zeros((variants, pitch), np.uint8)
    dev[:, :rows.shape[1]] = rows
    d_rows = torch.from_numpy(dev).cuda()
    rs, rc = oracle.score_reference(rows, prep, threads=8)
    plan = DevicePlan(prep, engine=PLAIN)
    try:
        for splits in (1, 7, 64):
            plan.set_shape((kernel << 16) | splits)
            assert plan.shape >> 16 == kernel
            s, c = plan.score(d_rows, pitch)
            plan.sync()
            np.testing.assert_array_equal(c.cpu().numpy().astype(np.uint32), rc)
            assert oracle.within_reference_tolerance(s.cpu().numpy(), rs).all(), splits
    finally:
        plan.close()


def test_set_shape_rejects_unknown_kernels(cuda):
    from gnomon_b200.device import DevicePlan
    from gnomon_b200.prepare import from_workload
    # 6,667 stages: more than the 4,736 splits the autotuner's largest
    # candidate (8x the CTA slots of the 512-byte kernel) allocates for
    prep = from_workload(synth.scaled(synth.WORKLOADS["plain_2k_x_50k"], 500, 200_000, 1))
    plan = DevicePlan(prep, engine=PLAIN)
    try:
        with pytest.raises(_lib.GnomonGpuError):
            plan.set_shape((768 << 16) | 4)
        with pytest.raises(_lib.GnomonGpuError):   # more partial slots than allocated
            plan.set_shape((1024 << 16) | 0xFFFF)
        assert plan.shape >> 16 in _lib.PLAIN_KERNELS
    finally:
        plan.close()


@pytest.mark.parametrize("people,variants", [(2_000, 50_000), (50_000, 60_000)])
def test_autotuned_shapes_keep_results(cuda, people, variants):
    """The autotuner times every plain kernel at three split counts on the
    resident rows and keeps the fastest; the tuned plan's result equals the
    default plan's (counts exact, sums within 1e-9 relative: only the FP64
    grouping of split partials changes).  The chosen shape is printed
    (TUNED_SHAPE line, pytest -s) for the small- and large-cohort shapes."""
    import json
    import torch
    from gnomon_b200.device import DevicePlan, row_pitch
    prep, rows = _c_rows_case(people, variants, 1)
    pitch = row_pitch(prep.bytes_per_variant)
    dev = np.zeros((variants, pitch), np.uint8)
    dev[:, :rows.shape[1]] = rows
    d_rows = torch.from_numpy(dev).cuda()
    del dev
    plan = DevicePlan(prep, engine=PLAIN)
    try:
        s0, c0 = plan.score(d_rows, pitch)
        plan.sync()
        s0, c0 = s0.cpu().numpy(), c0.cpu().numpy()
        default = plan.shape
        shape = plan.autotune(d_rows, pitch)
        s1, c1 = plan.score(d_rows, pitch)
        plan.sync()
        np.testing.assert_array_equal(c1.cpu().numpy(), c0)
        assert oracle.rel_err(s1.cpu().numpy(), s0).max() < 1e-9
        print("TUNED_SHAPE " + json.dumps({"people": people, "variants": variants,
                                           "default": [default >> 16, default & 0xFFFF],
                                           "tuned": [shape >> 16, shape & 0xFFFF]}))
    finally:
        plan.close()
