"""Index arithmetic of the SM-pair 8-bit kernel (gnm_t8_pairs in
gnomon_b200/csrc/gnm_tensor.cu), restated and checked on the CPU:

* the static work-item list covers passes 0-3 once per (people tile, score
  pair) and the member pass once per score tile, whatever the order;
* the score rows a CTA loads (srow) stay on 128-row tiles, and every row of
  the plan's K_pad falls to exactly one CTA per pass;
* a CTA's operand row n = 32 q + col for person 4 col + q of its half, placed
  at TMEM column 128 rank + n, is the slot the finalize reads for that person
  (gnm_tc_finalize: slot = 128 h + 32 (r % 4) + r / 4 with r the person's
  index in its half h).
"""
import itertools

import pytest

TILE_M = 128   # score rows per CTA


def pair_item(w, ptiles, spairs, spairs_m, raster):
    """(pass, people tile, score pair or pair of score pairs) of work item w."""
    per = ptiles * spairs
    if w < 4 * per:
        pas, t, sp = w // per, w % per, spairs
    else:
        pas, t, sp = 4, w - 4 * per, spairs_m
    ptile = t // sp if raster else t % ptiles
    spair = t % sp if raster else t // ptiles
    return pas, ptile, spair


def srow(pas, spair, j, rank):
    if pas == 4:
        return (2 * (2 * spair + j) + rank) * TILE_M
    return (2 * spair + rank) * TILE_M


@pytest.mark.parametrize("ptiles,stiles", [(1, 1), (3, 2), (391, 4), (5, 5), (2, 7), (17, 3)])
@pytest.mark.parametrize("raster", [0, 1])
def test_items_cover_every_tile_once(ptiles, stiles, raster):
    spairs = (stiles + 1) // 2
    spairs_m = (spairs + 1) // 2
    items = 4 * ptiles * spairs + ptiles * spairs_m
    k_pad = stiles * TILE_M
    sums = {}      # (pass, ptile, score row) -> CTAs that write it
    counts = {}    # (ptile, score row) -> CTAs that count it
    for w in range(items):
        pas, ptile, spair = pair_item(w, ptiles, spairs, spairs_m, raster)
        assert 0 <= ptile < ptiles
        assert 0 <= spair < (spairs_m if pas == 4 else spairs)
        for rank in (0, 1):
            for j in ((0, 1) if pas == 4 else (0,)):
                r0 = srow(pas, spair, j, rank)
                assert r0 % TILE_M == 0
                if r0 >= k_pad:   # a CTA past the last score tile writes nothing
                    continue
                key = (ptile, r0)
                if pas == 4:
                    counts[key] = counts.get(key, 0) + 1
                else:
                    sums[(pas,) + key] = sums.get((pas,) + key, 0) + 1
    for pas, p, r in itertools.product(range(4), range(ptiles), range(0, k_pad, TILE_M)):
        assert sums.get((pas, p, r)) == 1
    for p, r in itertools.product(range(ptiles), range(0, k_pad, TILE_M)):
        assert counts.get((p, r)) == 1


def test_tmem_column_is_the_finalize_slot():
    seen = set()
    for rank in (0, 1):
        for col in range(32):
            for q in range(4):
                person = 128 * rank + 4 * col + q          # index in the 256-person tile
                column = 128 * rank + 32 * q + col         # TMEM column of its sums
                h, r = divmod(person, 128)
                slot = 128 * h + 32 * (r % 4) + r // 4      # gnm_tc_finalize
                assert column == slot
                seen.add(column)
    assert seen == set(range(256))
