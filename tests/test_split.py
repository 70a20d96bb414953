"""One capture decoded as segments one after another on one GPU and joined
(cuvhs_b200.shard) equals the single-pass decode byte for byte: field
metadata, .tbc.json, luma and chroma.  Each segment starts its own chunk chain
with fresh state at a predicted chunk boundary; the join replays chunks until
the chains and the carried state meet."""
import numpy as np
import pytest

import cuvhs_b200 as cv
from cuvhs_b200 import shard
from conftest import rate_mhz, system, workload


@pytest.mark.gpu
@pytest.mark.parametrize("name,parts,batch", [("plain40_28", 2, 8), ("plain40_28", 3, 6), ("dropouts28pal", 2, 2)])
def test_split_decode_equals_single_pass(name, parts, batch):
    x = workload(name)
    kw = dict(system=system(name))
    with cv.Decoder(rate_mhz(name), batch_fields=batch, **kw) as d:
        single = d.decode_capture(x)
    joined, replays, seg_chunks = shard.decode_split(x, rate_mhz(name), parts=parts, batch_fields=batch, **kw)
    assert len(seg_chunks) == parts and min(seg_chunks) >= 1, seg_chunks
    assert joined.n_fields == single.n_fields > 0
    assert np.array_equal(joined.file_loc, single.file_loc)
    assert joined.json == single.json
    assert np.array_equal(joined.luma, single.luma)
    assert np.array_equal(joined.chroma, single.chroma)
    # the predicted chunk boundaries hold on a constant-speed tape and later
    # segments take the capture's chroma threshold: each join replays at most
    # the segment's first two chunks
    assert all(r <= 2 for r in replays), (replays, seg_chunks)


@pytest.mark.gpu
def test_state_round_trip_continues_the_decode():
    """cuvhs_get_state after a chunk, cuvhs_set_state into a fresh context,
    then the next chunk: the same as the next chunk in the first context."""
    x = workload("plain40_28")
    with cv.Decoder(28.0, batch_fields=8) as a, cv.Decoder(28.0, batch_fields=8) as b:
        r0, nxt = a.decode_chunk(x, 0, 8)
        st = a.get_state()
        r1, n1 = a.decode_chunk(x[nxt:], nxt, 8)
        b.set_state(st)
        r2, n2 = b.decode_chunk(x[nxt:], nxt, 8)
    assert n1 == n2 and r1.json == r2.json
    assert np.array_equal(r1.luma, r2.luma) and np.array_equal(r1.chroma, r2.chroma)
