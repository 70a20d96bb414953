"""Stage-level entry points (cuvhs_stage_*, cuvhs_b200.stages) and the
asynchronous chunk call with cuvhs_flush.

Run in the reference's order over one chunk, the stages must reproduce the
chunk decode bit for bit (they share its kernels and host code).  Fed the FP64
oracle's own intermediates, each stage must meet the parity bar on its own:
pulses, field windows and coarse line locations bit-exact, refined line
locations within 0.01 sample, luma and chroma within 1 LSB on >= 99.9% of
samples, phase IDs exact."""
import numpy as np
import pytest

import cuvhs_b200 as cv
from conftest import inside_fields, json_fields, oracle_decode, rate_mhz, single_pass, system, workload
from cuvhs_b200 import stages

POS_TOL = 0.01
LSB_FRACTION = 1e-3


def _chunk_shape(dec, n):
    """(requested fields, tiles, samples read) of the first chunk
    cuvhs_decode_capture takes."""
    nf = min(dec.batch_fields, n // dec.samples_per_field)
    n_read = min(nf * dec.tile_stride, n)
    return nf, min(n_read // dec.samples_per_field, nf), n_read


def _u16(t):
    return t.cpu().numpy().view(np.uint16)


def _run_stages(s, x):
    import torch
    nf, T, n_read = _chunk_shape(s, x.size)
    raw = torch.from_numpy(x).cuda()
    video, sync, env = stages.fm_demod(s, raw, T, n_read)
    offs, nxt = stages.discover_vsyncs(s, sync, T, nf)
    assert len(offs) <= T  # every field's slot was demodulated
    starts, lengths, counts = stages.sync_pulses(s, sync, T, offs)
    ll, first = stages.line_locations(s, 0, offs, starts, lengths, counts)
    dll = torch.from_numpy(ll).cuda()
    stages.hsync_refine(s, sync, dll)
    luma = stages.tbc_resample(s, video, dll)
    chroma, ids = stages.chroma_decode(s, raw, dll, n_read)
    # the dropout stage (cuvhs_dropouts_noalloc) takes NTSC fields
    do = stages.dropout_detect(s, env, dll, luma, chroma) if s.lines_per_frame == 525 else None
    return dict(T=T, video=video, sync=sync, env=env, offs=offs, nxt=nxt, starts=starts, lengths=lengths,
                counts=counts, ll_coarse=ll, first=first, ll=dll.cpu().numpy(), luma=_u16(luma),
                chroma=_u16(chroma), ids=ids, do=None if do is None else [t.cpu().numpy() for t in do])


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["small28", "dropouts28", "small28pal", "dropouts28_singlepass"])
def test_stages_in_order_reproduce_the_chunk_decode(name):
    x = workload(name)
    mhz = rate_mhz(name)
    opts = dict(system=system(name), single_pass_lines=single_pass(name))
    with cv.Decoder(mhz, debug=True, **opts) as d:
        r = d.decode_capture(x)
        dbg = {k: d.debug_array(k) for k in ("field_offsets", "k2_pulse_count", "k2_pulse_starts",
                                             "k2_pulse_lengths", "linelocs_coarse", "linelocs", "is_first",
                                             "video", "sync", "envelope")}
    with cv.Decoder(mhz, **opts) as s:
        g = _run_stages(s, x)
        spp = s.tile_stride
    P = len(g["offs"])
    assert P == r.n_fields
    assert np.array_equal(g["offs"], dbg["field_offsets"])
    nt = dbg["video"].size  # the debug copies cover the first tiles
    for k, dk in (("video", "video"), ("sync", "sync"), ("env", "envelope")):
        assert np.array_equal(g[k][:nt].cpu().numpy(), dbg[dk]), k
    assert np.array_equal(g["counts"], dbg["k2_pulse_count"])
    assert np.array_equal(g["starts"].ravel(), dbg["k2_pulse_starts"][:P * 800])
    assert np.array_equal(g["lengths"].ravel(), dbg["k2_pulse_lengths"][:P * 800])
    assert np.array_equal(g["ll_coarse"].ravel(), dbg["linelocs_coarse"])
    assert np.array_equal(g["first"], dbg["is_first"])
    assert np.array_equal(g["ll"].ravel(), dbg["linelocs"])
    assert np.array_equal(g["ids"], r.field_phase_id)
    if g["do"] is None:  # PAL: no dropout stage; fields the decoder left unconcealed match
        clean = [f for f in range(P) if r.dropouts[f][0].size == 0]
        assert len(clean) >= P - 1
        assert np.array_equal(g["luma"][clean], r.luma[clean])
        assert np.array_equal(g["chroma"][clean], r.chroma[clean])
        assert 0 < g["nxt"] <= P * spp
        return
    assert np.array_equal(g["luma"], r.luma)
    assert np.array_equal(g["chroma"], r.chroma)
    cnt, lines, sx, ex = g["do"]
    for f in range(P):
        dl, ds, de = r.dropouts[f]
        c = int(cnt[f])
        assert c == dl.size, f
        o = f * 512
        assert np.array_equal(lines[o:o + c], dl) and np.array_equal(sx[o:o + c], ds) and np.array_equal(ex[o:o + c], de)
    assert 0 < g["nxt"] <= P * spp


@pytest.mark.gpu
def test_each_stage_on_the_oracle_inputs():
    import torch
    name = "small28"
    x = workload(name)
    o = oracle_decode(name)
    P = len(o.array(0, "field_offsets"))
    inside = inside_fields([f["fileLoc"] for f in json_fields(o.json)], x.size, 28.0)
    with cv.Decoder(28.0) as s:
        nf, T, n_read = _chunk_shape(s, x.size)
        raw = torch.from_numpy(x).cuda()
        video, sync, env = stages.fm_demod(s, raw, T, n_read)
        # field windows and pulses from the GPU sync
        offs, _ = stages.discover_vsyncs(s, sync, T, nf)
        assert np.array_equal(offs, o.array(0, "field_offsets"))
        starts, lengths, counts = stages.sync_pulses(s, sync, T, o.array(0, "field_offsets"))
        oc = o.array(0, "k2_pulse_count")
        os_ = o.array(0, "k2_pulse_starts").reshape(P, 800)
        ol = o.array(0, "k2_pulse_lengths").reshape(P, 800)
        for f in inside:
            assert counts[f] == oc[f]
            assert np.array_equal(starts[f, :oc[f]], os_[f, :oc[f]])
            assert np.array_equal(lengths[f, :oc[f]], ol[f, :oc[f]])
        # host line locations from the oracle's own pulses: the same FP64 code path
        ll, first = stages.line_locations(s, 0, o.array(0, "field_offsets"), os_, ol, oc)
        assert np.array_equal(ll, o.array(0, "linelocs_coarse").reshape(P, 525))
        assert np.array_equal(first, o.array(0, "is_first"))
        # hsync refinement of the oracle's coarse line locations
        dll = torch.from_numpy(o.array(0, "linelocs_coarse").reshape(P, 525).copy()).cuda()
        stages.hsync_refine(s, sync, dll)
        ref = o.array(0, "linelocs").reshape(P, 525)
        for f in inside:
            assert np.abs(dll.cpu().numpy()[f, :264] - ref[f, :264]).max() <= POS_TOL, f
        # luma and chroma on the oracle's refined line locations
        oll = torch.from_numpy(ref.copy()).cuda()
        luma = _u16(stages.tbc_resample(s, video, oll))
        chroma, ids = stages.chroma_decode(s, raw, oll, n_read)
        chroma = _u16(chroma)
    ofields = json_fields(o.json)
    for i in inside:
        for a, b, what in ((luma[i], o.luma[i], "luma"), (chroma[i], o.chroma[i], "chroma")):
            dd = np.abs(a.astype(np.int32) - b.astype(np.int32))
            assert (dd > 1).mean() <= LSB_FRACTION, (what, i, int(dd.max()))
        assert ids[i] == ofields[i].get("fieldPhaseID", 0), i


@pytest.mark.gpu
def test_stage_arguments_are_checked():
    import torch
    with cv.Decoder(28.0, batch_fields=4) as s:
        sync = torch.zeros(4 * s.tile_stride, dtype=torch.float32, device="cuda")
        with pytest.raises(cv.CuvhsError):
            stages.discover_vsyncs(s, sync, 5)  # more tiles than the allocation
        with pytest.raises(cv.CuvhsError):
            stages.sync_pulses(s, sync, 4, np.array([4 * s.tile_stride], np.int64))  # offset outside the chunk
        # more windows than demodulated slots: the line stages read only the slots given
        with pytest.raises(ValueError):
            stages.dropout_detect(s, sync[:2 * s.tile_stride], torch.zeros(3 * 525, dtype=torch.float64,
                                                                             device="cuda"),
                                  torch.zeros((3, 263, 910), dtype=torch.int16, device="cuda"),
                                  torch.zeros((3, 263, 910), dtype=torch.int16, device="cuda"))
        # a flat sync has no pulses: uniform field windows, empty pulse lists
        offs, _ = stages.discover_vsyncs(s, sync + 1e6, 4)
        assert np.array_equal(offs, np.arange(4) * s.samples_per_field)
        _, _, counts = stages.sync_pulses(s, sync + 1e6, 4, offs)
        assert not counts.any()


@pytest.mark.gpu
@pytest.mark.parametrize("batch", [7, 0])
def test_async_chunks_and_flush_match_the_capture_decode(batch):
    x = workload("plain40_28")
    with cv.Decoder(28.0, batch_fields=batch) as d:
        a = d.decode_capture(x)
    with cv.Decoder(28.0, batch_fields=batch) as d:
        b = d.decode_chunks_async(x)
        assert lib_flush_ok(d)
    assert a.json == b.json
    assert np.array_equal(a.luma, b.luma) and np.array_equal(a.chroma, b.chroma)


def lib_flush_ok(d):
    return cv.lib.cuvhs_flush(d._h) == 0
