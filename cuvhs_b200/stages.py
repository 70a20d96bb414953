"""The decode one stage at a time (cuvhs_stage_* in include/cuvhs.h).

Each function is the counterpart of one stage function of the reference's
Pipeline::process_chunk (src/pipeline/pipeline.cu:1557-2548), with the
reference's name and argument meaning, on torch CUDA tensors instead of raw
device pointers.  They run the library's kernels and host code on the
decoder's stream and scratch and share its carried state, so running them in
order over a chunk gives exactly what Decoder's chunk decode gives.

A chunk is `tiles` field slots of dec.tile_stride samples; positions are
sample indices from the chunk's first sample.  Video and sync are FP32 Hz
relative to the 0 IRE frequency (ire0_hz(dec)); line locations FP64,
dec.lines_per_frame per field; luma and chroma u16 (held in int16 tensors)
[fields, *dec.field_shape].
"""
import ctypes

import numpy as np

from ._lib import lib

MAX_PULSES = 800


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _np(a):
    return ctypes.c_void_p(a.ctypes.data)


def _ready(t):
    """The decoder's stream does not wait for torch's: finish torch's work on
    the inputs first."""
    import torch
    torch.cuda.current_stream(t.device).synchronize()


def ire0_hz(dec):
    return lib.cuvhs_ire0_hz(dec._h)


def fm_demod(dec, raw, tiles, n_read=None):
    """fm_demod (src/pipeline/fm_demod.h:46-53): (video, sync, envelope) of a
    raw chunk held in a CUDA tensor of the decoder's input format (uint8 or
    16-bit); samples past n_read (default: all of raw) count as 0."""
    import torch
    n = tiles * dec.tile_stride
    video = torch.empty(n, dtype=torch.float32, device=raw.device)
    sync = torch.empty_like(video)
    env = torch.empty_like(video)
    n_read = raw.numel() if n_read is None else n_read
    _ready(raw)
    dec._check(lib.cuvhs_stage_fm_demod(dec._h, _p(raw), n_read, tiles, _p(video), _p(sync), _p(env)))
    return video, sync, env


def discover_vsyncs(dec, sync, tiles, max_fields=None):
    """discover_vsyncs and its clustering (src/pipeline/vsync_discover.h:6-11,
    src/pipeline/pipeline.cu:1567-1651): (field_offsets int64, next chunk start).
    max_fields is the chunk's requested field count (default batch_fields); a
    window may start past the last demodulated tile, so up to tiles + 1
    windows come back."""
    cap = dec.batch_fields if max_fields is None else max_fields
    offs = np.zeros(max(cap, 1), np.int64)
    n = ctypes.c_int(0)
    nxt = ctypes.c_int64(0)
    _ready(sync)
    dec._check(lib.cuvhs_stage_discover_vsyncs(dec._h, _p(sync), tiles, cap, _np(offs), ctypes.byref(n),
                                               ctypes.byref(nxt)))
    return offs[:n.value].copy(), nxt.value


def sync_pulses(dec, sync, tiles, field_offsets):
    """sync_pulses (src/pipeline/sync_pulses.h:20-27): (starts, lengths)
    [fields, 800] int32 and counts [fields]."""
    offs = np.ascontiguousarray(field_offsets, np.int64)
    n = offs.size
    starts = np.zeros((max(n, 1), MAX_PULSES), np.int32)
    lengths = np.zeros_like(starts)
    counts = np.zeros(max(n, 1), np.int32)
    _ready(sync)
    dec._check(lib.cuvhs_stage_sync_pulses(dec._h, _p(sync), tiles, _np(offs), n, _np(starts), _np(lengths),
                                           _np(counts)))
    return starts[:n], lengths[:n], counts[:n]


def line_locations(dec, raw_offset, field_offsets, starts, lengths, counts):
    """The host line locations after sync_pulses (src/pipeline/pipeline.cu:1717-1778):
    (linelocs [fields, lines_per_frame] float64, is_first_field [fields] int32)."""
    offs = np.ascontiguousarray(field_offsets, np.int64)
    n = offs.size
    starts = np.ascontiguousarray(starts, np.int32).reshape(n, MAX_PULSES) if n else np.zeros((1, MAX_PULSES), np.int32)
    lengths = np.ascontiguousarray(lengths, np.int32).reshape(n, MAX_PULSES) if n else np.zeros_like(starts)
    counts = np.ascontiguousarray(counts, np.int32) if n else np.zeros(1, np.int32)
    ll = np.zeros((max(n, 1), dec.lines_per_frame), np.float64)
    first = np.zeros(max(n, 1), np.int32)
    dec._check(lib.cuvhs_stage_line_locations(dec._h, raw_offset, _np(offs), n, _np(starts), _np(lengths),
                                              _np(counts), _np(ll), _np(first)))
    return ll[:n], first[:n]


def hsync_refine(dec, sync, linelocs):
    """hsync_refine (src/pipeline/hsync_refine.h:18-22): refines the float64
    CUDA tensor linelocs [fields, lines_per_frame] in place."""
    tiles = sync.numel() // dec.tile_stride
    _ready(sync)
    dec._check(lib.cuvhs_stage_hsync_refine(dec._h, _p(sync), tiles, _p(linelocs),
                                            linelocs.numel() // dec.lines_per_frame))
    return linelocs


def tbc_resample(dec, video, linelocs):
    """tbc_resample (src/pipeline/tbc_resample.h:16-27): luma [fields, rows, columns]."""
    import torch
    n = linelocs.numel() // dec.lines_per_frame
    luma = torch.empty((n,) + dec.field_shape, dtype=torch.int16, device=video.device)
    tiles = video.numel() // dec.tile_stride
    _ready(video)
    dec._check(lib.cuvhs_stage_tbc_resample(dec._h, _p(video), tiles, _p(linelocs), n, _p(luma)))
    return luma


def chroma_decode(dec, raw, linelocs, n_read=None):
    """chroma_decode (src/pipeline/chroma_decode.h:38-46): (chroma [fields,
    rows, columns], field phase IDs) from the raw chunk."""
    import torch
    n = linelocs.numel() // dec.lines_per_frame
    chroma = torch.empty((n,) + dec.field_shape, dtype=torch.int16, device=raw.device)
    ids = np.zeros(max(n, 1), np.int32)
    n_read = raw.numel() if n_read is None else n_read
    _ready(raw)
    dec._check(lib.cuvhs_stage_chroma_decode(dec._h, _p(raw), n_read, _p(linelocs), n, _p(chroma), _np(ids)))
    return chroma, ids[:n]


def dropout_detect(dec, envelope, linelocs, luma, chroma):
    """dropout_detect (src/pipeline/dropout_detect.h:22-32) through
    cuvhs_dropouts_noalloc on torch's current stream: conceals luma and chroma
    in place; returns (counts, lines, startx, endx) as int32 CUDA tensors.
    NTSC fields only, as cuvhs_dropouts_noalloc."""
    import torch
    if dec.lines_per_frame != 525:
        raise ValueError("cuvhs_dropouts_noalloc takes NTSC fields")
    n = linelocs.numel() // dec.lines_per_frame
    if envelope.numel() < n * dec.tile_stride:
        raise ValueError(f"the envelope covers {envelope.numel() // dec.tile_stride} field slots, "
                         f"the line locations {n} fields")
    dev = envelope.device
    count = torch.zeros(n, dtype=torch.int32, device=dev)
    lines = torch.zeros(n * 512, dtype=torch.int32, device=dev)
    sx = torch.zeros_like(lines)
    ex = torch.zeros_like(lines)
    st = torch.cuda.current_stream(dev)  # ordered after the fills above
    if lib.cuvhs_dropouts_noalloc(_p(envelope), _p(linelocs), n, dec.tile_stride, _p(luma), _p(chroma),
                                  _p(count), _p(lines), _p(sx), _p(ex), ctypes.c_void_p(st.cuda_stream)) != 0:
        raise ValueError("cuvhs_dropouts_noalloc rejected its arguments")
    st.synchronize()
    return count, lines, sx, ex
