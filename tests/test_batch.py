"""cuvhs_batch_*: many independent captures of mixed sample rates decoded
concurrently.  Every capture's output must equal its single-capture decode
(fresh context, cuvhs_decode_capture), whatever the lane count or item order."""
import numpy as np
import pytest

import cuvhs_b200 as cv


def test_batch_specs_cover_the_mixed_configuration():
    sp = cv.batch_specs(64)
    assert len(sp) == 64
    assert {s["sample_rate_hz"] for s in sp} == {28e6, 35.8e6, 40e6}
    assert all(2 <= s["n_fields"] <= 240 for s in sp)
    assert all(30 <= s["snr_db"] <= 45 and 0 <= s["dropout_line_rate"] <= 0.005 for s in sp)
    assert len({s["seed"] for s in sp}) == 64
    assert cv.batch_specs(64) == sp  # seeded


@pytest.mark.gpu
def test_batch_matches_single_capture_decodes():
    caps = cv.make_batch_workload(count=6, min_fields=2, max_fields=12, seed=77)
    assert len({mhz for _, mhz in caps}) == 3
    single = []
    for x, mhz in caps:
        with cv.Decoder(mhz) as d:
            single.append(d.decode_capture(x))
    with cv.Batch(lanes=3) as b:
        assert b.lanes == 3
        got = b.decode(caps)
        got_rev = b.decode(caps[::-1], pinned=True)[::-1]  # reused contexts, other order, pinned
    with cv.Batch(lanes=1) as b:
        got_one = b.decode(caps)
    for i, s in enumerate(single):
        assert s.n_fields > 0
        for g in (got[i], got_rev[i], got_one[i]):
            assert g.n_fields == s.n_fields, i
            assert np.array_equal(g.luma, s.luma) and np.array_equal(g.chroma, s.chroma), i
            assert g.json == s.json, i


@pytest.mark.gpu
def test_batch_reports_per_item_errors():
    x, mhz = cv.make_batch_workload(count=1, min_fields=3, max_fields=3, seed=5)[0]
    with cv.Batch(lanes=2) as b:
        items, keep = b.prepare([(x, mhz), (x, mhz), (x[:1000], mhz)])
        keep[1]["out"].max_fields = 1  # room for one of its fields only
        st = cv.lib.cuvhs_batch_decode(b._h, items, 3)
        assert items[0].status == 0 and keep[0]["out"].fields_out > 1
        assert items[1].status == 5 and st == 5  # CUVHS_ERR_CAPACITY, the failing item's status
        assert b"too small" in cv.lib.cuvhs_batch_last_error(b._h)
        # a capture shorter than one field decodes to nothing and is not an error
        assert items[2].status == 0 and keep[2]["out"].fields_out == 0


@pytest.mark.gpu
@pytest.mark.parametrize("round_fields", [16, 0])
def test_batched_rounds_match_single_decodes_with_multichunk_captures(round_fields):
    """Rounds of several captures (one launch per stage over all of them),
    captures longer than one chunk (carried state between rounds), mixed
    rates, and a round size either fixed small (many rounds, captures split
    across rounds) or chosen by the autotuner: every capture equals its
    single-capture decode with the same chunk size."""
    caps = cv.make_batch_workload(count=10, min_fields=3, max_fields=20, seed=91)
    single = []
    for x, mhz in caps:
        with cv.Decoder(mhz, batch_fields=8) as d:
            single.append(d.decode_capture(x))
    with cv.Batch(lanes=2, max_fields=8, round_fields=round_fields) as b:
        got = b.decode(caps)
        for mhz in {m for _, m in caps}:
            rf = b.round_fields(mhz)
            assert rf >= 8 and (round_fields == 0 or rf == round_fields), (mhz, rf)
    for i, s in enumerate(single):
        assert s.n_fields > 0
        g = got[i]
        assert g.n_fields == s.n_fields, i
        assert np.array_equal(g.file_loc, s.file_loc), i
        assert np.array_equal(g.luma, s.luma) and np.array_equal(g.chroma, s.chroma), i
        assert g.json == s.json, i
