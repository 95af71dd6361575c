"""Person sharding (the multi-GPU path) on CPU: shard arithmetic, and a
world_size-2 gloo job whose ranks score their shards with the oracle and
gather the cohort, compared with one unsharded oracle run."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

from gnomon_b200 import sharding, synth
from gnomon_b200.prepare import PreparationResult
from oracle import oracle

from helpers import synth_case


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("total,world", [(0, 2), (3, 2), (5, 2), (4096, 3), (50_001, 8),
                                         (17, 8), (12, 1)])
def test_person_ranges_partition(total, world):
    r = sharding.person_ranges(total, world)
    assert len(r) == world
    pos = 0
    for start, stop in r:
        assert start == pos and start <= stop
        assert start % 4 == 0 or start == total
        pos = stop
    assert pos == total
    sizes = [(b - a + 3) // 4 for a, b in r]   # bytes per shard
    assert max(sizes) - min(sizes) <= 1


def test_slice_rows_matches_generator_offset():
    """A shard's column slice of the cohort rows is the generator run with the
    shard's first person (the device generator's person_begin)."""
    w = synth.scaled(synth.WORKLOADS["plain_2k_x_50k"], 403, 37)
    thr = synth.variant_thresholds(w.seed, 0, 37, w.p_lo, w.p_hi, w.missing_rate)
    full = synth.synth_rows(w.seed, 0, 37, 403, thr)
    for start, stop in sharding.person_ranges(403, 3):
        part = synth.synth_rows(w.seed, 0, 37, stop - start, thr, person_begin=start)
        np.testing.assert_array_equal(sharding.slice_rows(full, start, stop), part)


def _keep_subset(prep: PreparationResult, seed: int) -> PreparationResult:
    rng = np.random.default_rng(seed)
    P = prep.total_people_in_fam
    keep = rng.permutation(P)[: P * 2 // 3].astype(np.uint32)
    return PreparationResult(prep.sparse_weights, prep.sparse_missing_corrections,
                             prep.sparse_score_columns, prep.sparse_row_offsets,
                             list(prep.score_names), P, output_idx_to_fam_idx=keep)


def _shards_concat(prep, rows, world):
    K = prep.num_scores
    s_full = np.zeros((prep.num_people_to_score, K))
    c_full = np.zeros((prep.num_people_to_score, K), np.uint32)
    for r in range(world):
        sh = sharding.make_shard(prep, r, world)
        if sh.num_people == 0:
            continue
        s, c = oracle.score_extended(sharding.slice_rows(rows, sh.start, sh.stop), sh.prep)
        s_full[sh.output_rows] = s.reshape(-1, K)
        c_full[sh.output_rows] = c.reshape(-1, K)
    return s_full, c_full


@pytest.mark.parametrize("subset", [False, True])
def test_shards_reassemble_to_cohort(subset):
    _, prep, rows, _ = synth_case(333, 500, scores=3)
    if subset:
        prep = _keep_subset(prep, 5)
    s0, c0 = oracle.score_extended(rows, prep)
    for world in (2, 3, 5):
        s, c = _shards_concat(prep, rows, world)
        np.testing.assert_array_equal(c.reshape(-1), c0)
        np.testing.assert_allclose(s.reshape(-1), s0, rtol=1e-13, atol=1e-13)


def test_bad_shard_range_rejected():
    _, prep, _, _ = synth_case(40, 10)
    with pytest.raises(ValueError):
        sharding.shard_prep(prep, 2, 10)
    with pytest.raises(ValueError):
        sharding.shard_prep(prep, 0, 41)


def _gloo_worker(rank, world, port, outdir, subset):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        _, prep, rows, _ = synth_case(259, 300, scores=2)
        if subset:
            prep = _keep_subset(prep, 11)
        res = sharding.score_sharded(prep, rows, rank, world,
                                     lambda p, r: oracle.score_extended(r, p))
        if rank == 0:
            s0, c0 = oracle.score_extended(rows, prep)
            s, c = res
            ok = (np.array_equal(c.reshape(-1), c0)
                  and np.allclose(s.reshape(-1), s0, rtol=1e-13, atol=1e-13))
            Path(outdir, "result").write_text("ok" if ok else "mismatch")
        else:
            assert res is None
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("subset", [False, True])
def test_gloo_world2_sharded_job(tmp_path, subset):
    import torch.multiprocessing as mp
    mp.spawn(_gloo_worker, args=(2, _free_port(), str(tmp_path), subset), nprocs=2, join=True)
    assert (tmp_path / "result").read_text() == "ok"
