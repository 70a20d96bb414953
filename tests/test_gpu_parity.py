"""GPU decoder (through the C ABI) against the FP64 oracle and the reference.

Bar: on every field whose analysis window lies inside the capture, field
metadata (.tbc.json entries: file location, field order, phase ID, dropouts),
sync pulses before and after validation and coarse line locations are
bit-exact; refined line locations agree within 0.01 sample; luma and chroma
agree within 1 LSB on at least 99.9% of samples."""
import json

import numpy as np
import pytest

import cuvhs_b200 as cv
from conftest import (GOLDEN, golden, inside_fields, json_fields, oracle_decode, rate_mhz, single_pass, system,
                      workload)

LSB_FRACTION = 1e-3
POS_TOL = 0.01


def decode(name, batch_fields=0):
    x = workload(name)
    mhz = rate_mhz(name)
    with cv.Decoder(mhz, batch_fields=batch_fields, debug=True, system=system(name),
                    single_pass_lines=single_pass(name)) as d:
        r = d.decode_capture(x)
        dbg = {k: d.debug_array(k) for k in ("field_offsets", "k2_pulse_count", "k2_pulse_starts",
                                             "k2_pulse_lengths", "k2b_pulse_count", "k2b_pulse_starts",
                                             "k2b_pulse_lengths", "k2b_pulse_types", "linelocs_coarse",
                                             "linelocs", "is_first")}
    return x, mhz, r, dbg


def assert_tbc_close(a, b, what):
    d = np.abs(a.astype(np.int32) - b.astype(np.int32))
    frac = float((d > 1).mean())
    assert frac <= LSB_FRACTION, (what, frac, int(d.max()))
    return frac, int(d.max())


def compare_to_oracle(name, r, dbg, x, mhz, o, chunk_last_only=False):
    assert r.n_fields == o.n_fields
    ofields = json_fields(o.json)
    mfields = json_fields(r.json)
    assert [f["fileLoc"] for f in mfields] == [f["fileLoc"] for f in ofields]
    inside = inside_fields([f["fileLoc"] for f in mfields], x.size, mhz, system(name))
    assert len(inside) >= r.n_fields - 1
    for i in inside:
        assert mfields[i] == ofields[i], i
    for i in inside:
        assert_tbc_close(r.luma[i], o.luma[i], ("luma", i))
        assert_tbc_close(r.chroma[i], o.chroma[i], ("chroma", i))
    return inside


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["small28", "dropouts28", "plain40_28", "small358", "small28pal",
                                  "dropouts28pal", "pal20_40", "small28_singlepass", "dropouts28_singlepass",
                                  "small28pal_singlepass", "tipthr28", "hard600_40"])
def test_decoder_matches_oracle(name):
    x, mhz, r, dbg = decode(name)
    o = oracle_decode(name)
    inside = compare_to_oracle(name, r, dbg, x, mhz, o)
    P = len(o.array(0, "field_offsets"))
    assert o.n_chunks == 1
    assert np.array_equal(dbg["field_offsets"], o.array(0, "field_offsets"))
    for pre in ("k2", "k2b"):
        cm, co = dbg[f"{pre}_pulse_count"], o.array(0, f"{pre}_pulse_count")
        for part in ["starts", "lengths"] + (["types"] if pre == "k2b" else []):
            a = dbg[f"{pre}_pulse_{part}"].reshape(P, 800)
            b = o.array(0, f"{pre}_pulse_{part}").reshape(P, 800)
            for f in inside:
                assert cm[f] == co[f], (pre, f)
                assert np.array_equal(a[f, :cm[f]], b[f, :co[f]]), (pre, part, f)
    lpf, rows = o.lines_per_frame, o.field_shape[0] + 1  # the lines the resamplers read
    llc = dbg["linelocs_coarse"].reshape(P, lpf)
    ll = dbg["linelocs"].reshape(P, lpf)
    for f in inside:
        assert np.array_equal(llc[f, :rows], o.array(0, "linelocs_coarse").reshape(P, lpf)[f, :rows])
        assert np.abs(ll[f, :rows] - o.array(0, "linelocs").reshape(P, lpf)[f, :rows]).max() <= POS_TOL


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["small28", "dropouts28", "plain40_28", "small28pal", "dropouts28pal",
                                  "small28_singlepass", "dropouts28_singlepass", "small28pal_singlepass"])
def test_decoder_matches_reference_fixture(name):
    g = golden(name)
    x, mhz, r, dbg = decode(name)
    gfields = json_fields(g["json_text"])
    mfields = json_fields(r.json)
    assert len(mfields) == len(gfields)
    inside = inside_fields([f["fileLoc"] for f in gfields], x.size, mhz, system(name))
    for i in inside:
        assert mfields[i] == gfields[i], i
    assert np.array_equal(dbg["field_offsets"], g["field_offsets"])
    P = len(g["field_offsets"])
    lpf = g["linelocs"].shape[1]
    rows = r.luma.shape[1] + 1
    off = np.concatenate([[0], np.cumsum(g["k2_count"])])
    starts = dbg["k2_pulse_starts"].reshape(P, 800)
    for f in inside:
        assert np.array_equal(starts[f, :g["k2_count"][f]], g["k2_starts"][off[f]:off[f + 1]]), f
        assert np.abs(dbg["linelocs"].reshape(P, lpf)[f, :rows] - g["linelocs"][f, :rows]).max() <= POS_TOL
    d = np.abs(r.luma[0, ::16].astype(np.int32) - g["luma_rows_f0"].astype(np.int32))
    assert (d > 1).mean() <= LSB_FRACTION


@pytest.mark.gpu
def test_hard600_40_matches_reference_json():
    """600 fields at 40 MHz, 32 dB, +/-2 jitter, 0.1% dropouts, head switch:
    every field inside the capture has the reference's exact metadata."""
    with open(f"{GOLDEN}/hard600_40.tbc.json") as f:
        gtext = f.read()
    x = workload("hard600_40")
    with cv.Decoder(40.0) as d:
        r = d.decode_capture(x)
    gfields = json_fields(gtext)
    mfields = json_fields(r.json)
    assert len(mfields) == len(gfields) == 599
    inside = inside_fields([f["fileLoc"] for f in gfields], x.size, 40.0)
    assert len(inside) >= 598
    bad = [i for i in inside if mfields[i] != gfields[i]]
    assert not bad, (bad[:5], [mfields[i] for i in bad[:2]], [gfields[i] for i in bad[:2]])
    assert sum(len(f["dropOuts"]["fieldLine"]) for f in mfields) >= 1


@pytest.mark.gpu
def test_multi_chunk_matches_oracle_with_same_chunking():
    """Chunks of 8 fields: chunk restarts, carried line-location, chroma-track
    and parity state must follow the reference's chunk loop."""
    name = "plain40_28"
    x, mhz, r, dbg = decode(name, batch_fields=8)
    from oracle.oracle import Oracle
    o = Oracle(mhz, batch_fields=8)
    o.decode(x)
    assert o.n_chunks > 3
    compare_to_oracle(name, r, dbg, x, mhz, o)


@pytest.mark.gpu
def test_drifting_40mhz_stream_matches_oracle_over_chunks():
    """A long-stream sample: 300 NTSC fields at 40 MHz u8 with +/-0.2% tape-speed
    drift, dropouts on 0.2% of lines, head switching and +/-1 sample jitter,
    decoded in 64-field chunks (the stream-mode chunk) from page-locked
    memory; the oracle with the same chunking must agree on every field's
    metadata, luma and chroma."""
    from oracle.oracle import Oracle
    x = workload("drift300_40")
    with cv.Decoder(40.0, batch_fields=64, debug=True) as d:
        r = d.decode_capture(x, pinned=True)
    o = Oracle(40.0, batch_fields=64)
    o.decode(x)
    assert o.n_chunks >= 4
    inside = compare_to_oracle("drift300_40", r, None, x, 40.0, o)
    assert len(inside) >= 290
    gaps = np.diff(r.file_loc.astype(np.int64))
    assert (gaps.max() - gaps.min()) / gaps.mean() > 0.002  # the drift shows in the field spacing


@pytest.mark.gpu
def test_decode_is_deterministic_and_chunk_api_matches_capture_api():
    x = workload("dropouts28")
    with cv.Decoder(28.0) as d:
        a = d.decode_capture(x)
        d.reset()
        b = d.decode_capture(x)
        d.reset()
        c, nxt = d.decode_chunk(x, 0, min(d.batch_fields, x.size // d.samples_per_field))
    assert np.array_equal(a.luma, b.luma) and np.array_equal(a.chroma, b.chroma) and a.json == b.json
    assert np.array_equal(a.luma[:c.n_fields], c.luma)
    assert nxt > 0


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["dropouts28", "dropouts28pal"])
def test_chained_launches_match_event_separated_launches(name):
    """The decode kernels are launched as a chain (each may be scheduled
    while its predecessor drains and waits for it on the device); with every
    stage bracketed by timing events they run strictly one after another.
    Both must give the same bytes."""
    x = workload(name)
    with cv.Decoder(rate_mhz(name), system=system(name)) as d:
        chained = d.decode_capture(x)
        d.reset()
        d.set_timing(True)
        separated = d.decode_capture(x)
        d.set_timing(False)
    assert np.array_equal(chained.luma, separated.luma)
    assert np.array_equal(chained.chroma, separated.chroma)
    assert chained.json == separated.json


@pytest.mark.gpu
@pytest.mark.parametrize("name,batch", [("dropouts28", 0), ("plain40_28", 8)])
def test_pinned_buffers_give_identical_output(name, batch):
    """Page-locked input and output buffers take the overlapped path (input in
    pieces with K1a per piece, luma copied out while chroma decodes); the
    result must equal the pageable path byte for byte."""
    x = workload(name)
    mhz = cv.WORKLOADS[name]["sample_rate_hz"] / 1e6
    with cv.Decoder(mhz, batch_fields=batch) as d:
        a = d.decode_capture(x)
        d.reset()
        b = d.decode_capture(x, pinned=True)
    assert a.n_fields == b.n_fields > 0
    assert np.array_equal(a.luma, b.luma) and np.array_equal(a.chroma, b.chroma)
    assert a.json == b.json


def _as_format(x, fmt, dc=0):
    """The u8 capture x as s16 / u16 samples of the same converted values
    ((x - 128) * 256), plus a constant DC offset."""
    v = (x.astype(np.int32) - 128) * 256 + dc
    if fmt == "s16":
        return np.clip(v, -32768, 32767).astype(np.int16)
    return np.clip(v + 32768, 0, 65535).astype(np.uint16)


@pytest.mark.gpu
@pytest.mark.parametrize("fmt", ["s16", "u16"])
def test_16_bit_inputs_decode_as_the_u8_capture(fmt):
    """s16 and u16 samples carrying the u8 capture's converted values decode
    to the same bytes (conversion of src/io/raw_reader.cpp:71-91), in one
    chunk and in chunks of 4 fields."""
    x = workload("small28")
    y = _as_format(x, fmt)
    for batch in (0, 4):
        with cv.Decoder(28.0, batch_fields=batch) as d:
            a = d.decode_capture(x)
        with cv.Decoder(28.0, batch_fields=batch, input_format=fmt) as d:
            b = d.decode_capture(y)
        assert b.n_fields == a.n_fields > 0
        assert np.array_equal(a.luma, b.luma) and np.array_equal(a.chroma, b.chroma) and a.json == b.json


@pytest.mark.gpu
def test_dc_correction_matches_oracle():
    """--dc-correct on an s16 capture with a DC offset of 2500 (the chunk mean
    of the samples read is subtracted before the zero fill,
    src/io/raw_reader.cpp:93-99): against the oracle with the same option."""
    x = workload("small28")
    y = _as_format(x, "s16", dc=2500)
    with cv.Decoder(28.0, input_format="s16", dc_correct=True) as d:
        r = d.decode_capture(y)
    from oracle.oracle import Oracle
    o = Oracle(28.0, input_format="s16", dc_correct=True)
    o.decode(y)
    compare_to_oracle("small28", r, None, x, 28.0, o)


@pytest.mark.gpu
def test_field_locations_past_32_bits():
    """A chunk whose first sample is capture sample 5*2^32 + 12345 (a long
    stream): field locations are that offset plus the chunk-relative ones,
    everything else is unchanged."""
    x = workload("small28")
    off = 5 * 2**32 + 12345
    with cv.Decoder(28.0) as d:
        nf = min(d.batch_fields, x.size // d.samples_per_field)
        a, na = d.decode_chunk(x, 0, nf)
        d.reset()
        b, nb = d.decode_chunk(x, off, nf)
    assert a.n_fields == b.n_fields > 0
    assert np.array_equal(b.file_loc - np.uint64(off), a.file_loc)
    assert nb == na + off
    assert np.array_equal(a.luma, b.luma) and np.array_equal(a.chroma, b.chroma)
    assert np.array_equal(a.is_first_field, b.is_first_field)
    assert [json.loads(b.json)["fields"][i]["fileLoc"] for i in range(b.n_fields)] == [int(v) for v in b.file_loc]


@pytest.mark.gpu
def test_cli_end_to_end(tmp_path):
    import subprocess
    name = "plain40_28"
    x = workload(name)
    inp = tmp_path / "cap.u8"
    x.tofile(inp)
    base = tmp_path / "out"
    p = subprocess.run([cv.CLI_PATH, "-f", "28", "--overwrite", str(inp), str(base)], capture_output=True,
                       text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    assert "Done." in p.stderr
    g = golden(name)
    assert (tmp_path / "out.tbc.json").read_text() == g["json_text"]
    luma = np.fromfile(tmp_path / "out.tbc", np.uint16).reshape(-1, 263, 910)
    chroma = np.fromfile(tmp_path / "out_chroma.tbc", np.uint16).reshape(-1, 263, 910)
    with cv.Decoder(28.0) as d:
        r = d.decode_capture(x)
    assert np.array_equal(luma, r.luma) and np.array_equal(chroma, r.chroma)
    # a second run without --overwrite refuses
    p2 = subprocess.run([cv.CLI_PATH, "-f", "28", str(inp), str(base)], capture_output=True, text=True, timeout=60)
    assert p2.returncode == 1 and "Output exists" in p2.stderr
    # the same capture as .s16 (format from the extension) and as raw u16 named
    # with --format, read in 2-byte samples from the file, give the same files
    for ext, fmt, extra in (("s16", "s16", []), ("bin", "u16", ["--format", "u16"])):
        f16 = tmp_path / f"cap16.{ext}"
        _as_format(x, fmt).tofile(f16)
        b16 = tmp_path / f"out_{fmt}"
        p3 = subprocess.run([cv.CLI_PATH, "-f", "28", "--overwrite"] + extra + [str(f16), str(b16)],
                            capture_output=True, text=True, timeout=300)
        assert p3.returncode == 0, p3.stderr
        assert (tmp_path / f"out_{fmt}.tbc.json").read_text() == g["json_text"]
        assert (tmp_path / f"out_{fmt}.tbc").read_bytes() == (tmp_path / "out.tbc").read_bytes()
        assert (tmp_path / f"out_{fmt}_chroma.tbc").read_bytes() == (tmp_path / "out_chroma.tbc").read_bytes()


@pytest.mark.gpu
@pytest.mark.parametrize("how", ["stdin", "fifo"])
def test_cli_stream_mode_matches_file_mode(tmp_path, how):
    """Stream mode (src/io/raw_reader.cpp:35-54,175-198): a capture piped in
    through stdin ("-") or a FIFO is read forward in 64-field chunks (the
    reference's stream cap); the files must equal file mode with --batch 64."""
    import os
    import subprocess
    import threading
    name = "plain40_28"
    x = workload(name)
    inp = tmp_path / "cap.u8"
    x.tofile(inp)
    ref = subprocess.run([cv.CLI_PATH, "-f", "28", "--overwrite", "--batch", "64", str(inp), str(tmp_path / "file")],
                         capture_output=True, text=True, timeout=300)
    assert ref.returncode == 0, ref.stderr
    base = tmp_path / "piped"
    if how == "stdin":
        with open(inp, "rb") as f:
            p = subprocess.run([cv.CLI_PATH, "-f", "28", "--overwrite", "-", str(base)], stdin=f,
                               capture_output=True, text=True, timeout=300)
    else:
        fifo = tmp_path / "cap.fifo"
        os.mkfifo(fifo)

        def feed():  # small writes, so the reader sees short reads
            with open(fifo, "wb") as w:
                data = x.tobytes()
                for i in range(0, len(data), 1 << 20):
                    w.write(data[i:i + (1 << 20)])
        t = threading.Thread(target=feed)
        t.start()
        p = subprocess.run([cv.CLI_PATH, "-f", "28", "--overwrite", "--format", "u8", str(fifo), str(base)],
                           capture_output=True, text=True, timeout=300)
        t.join(60)
    assert p.returncode == 0, p.stderr
    assert "Done." in p.stderr
    for suffix in (".tbc", "_chroma.tbc", ".tbc.json"):
        a = (tmp_path / f"file{suffix}").read_bytes()
        b = (tmp_path / f"piped{suffix}").read_bytes()
        assert a == b, suffix
    assert len((tmp_path / "piped.tbc").read_bytes()) > 0


@pytest.mark.gpu
def test_cli_pal(tmp_path):
    """--system PAL through the CLI: the reference's .tbc.json for the same
    capture, and the 1135 x 313 fields the library decodes."""
    import subprocess
    name = "dropouts28pal"
    x = workload(name)
    inp = tmp_path / "cap.u8"
    x.tofile(inp)
    base = tmp_path / "pal"
    p = subprocess.run([cv.CLI_PATH, "--system", "PAL", "-f", "28", "--overwrite", str(inp), str(base)],
                       capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    g = golden(name)
    mine = json_fields((tmp_path / "pal.tbc.json").read_text())
    ref = json_fields(g["json_text"])
    inside = inside_fields([f["fileLoc"] for f in ref], x.size, 28.0, "PAL")
    assert len(mine) == len(ref) and all(mine[i] == ref[i] for i in inside)
    head = (tmp_path / "pal.tbc.json").read_text().split('"fields"')[0]
    assert head == g["json_text"].split('"fields"')[0]  # PAL video parameters
    luma = np.fromfile(tmp_path / "pal.tbc", np.uint16).reshape(-1, 313, 1135)
    with cv.Decoder(28.0, system="PAL") as d:
        r = d.decode_capture(x)
    assert r.luma.shape[1:] == (313, 1135)
    assert np.array_equal(luma, r.luma)


@pytest.mark.gpu
def test_short_and_empty_captures():
    with cv.Decoder(28.0) as d:
        r = d.decode_capture(np.full(1000, 128, np.uint8))
        assert r.n_fields == 0
        x = workload("small28")[: d.samples_per_field - 1]
        assert d.decode_capture(x).n_fields == 0
        # exactly one field of samples: one chunk, zero-filled to the tile stride
        x1 = workload("small28")[: d.samples_per_field + 5000]
        r1 = d.decode_capture(x1)
        assert r1.n_fields <= 1


@pytest.mark.gpu
def test_device_memory_limit_backs_off_the_batch():
    """With less device memory than the free-memory sizing assumes (other
    users of the GPU), the context halves its batch until its buffers fit
    (the reference's VRAM back-off, src/pipeline/pipeline.cu:1384-1475) and
    decodes as before; an explicit batch that does not fit, or a limit below
    one field's buffers, fails with CUVHS_ERR_OUT_OF_MEMORY."""
    x = workload("small28")
    with cv.Decoder(28.0) as d:
        full, b_full = d.decode_capture(x), d.batch_fields
    with cv.Decoder(28.0, device_memory_limit_mb=3000) as d:
        lim, b_lim = d.decode_capture(x), d.batch_fields
    assert 1 <= b_lim < b_full and b_lim * 2 > 64, (b_lim, b_full)
    assert lim.json == full.json
    assert np.array_equal(lim.luma, full.luma) and np.array_equal(lim.chroma, full.chroma)
    for kw in (dict(batch_fields=2000, device_memory_limit_mb=3000), dict(device_memory_limit_mb=10)):
        with pytest.raises(cv.CuvhsError) as e:
            cv.Decoder(28.0, **kw)
        assert e.value.status == 3, str(e.value)  # CUVHS_ERR_OUT_OF_MEMORY
