"""ctypes binding of libcuvhs (include/cuvhs.h).

The decoder itself is native: CUDA kernels for sm_100a behind a C ABI, with
C++ host orchestration.  This module only loads that library and moves numpy
buffers across the boundary.  There is no Python fallback: importing fails if
the built library is missing.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libcuvhs.so")
CLI_PATH = os.path.join(_HERE, "bin", "cuvhs")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"libcuvhs.so not found at {LIB_PATH}; build it with `make -C cuvhs_b200/csrc` "
        "(or __graft_entry__.build())")

lib = ctypes.CDLL(LIB_PATH)

FIELD_W, FIELD_H = 910, 263
FIELD_PIXELS = FIELD_W * FIELD_H
MAX_DROPOUTS_PER_FIELD = 512

STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "out of device memory", 4: "I/O error",
          5: "capacity exceeded", 6: "unsupported", 7: "output exists"}


class CuvhsError(RuntimeError):
    def __init__(self, status, message=""):
        super().__init__(f"cuvhs: {STATUS.get(status, status)}: {message}")
        self.status = status


class Config(ctypes.Structure):
    _fields_ = [("system", ctypes.c_int), ("sample_rate_mhz", ctypes.c_double), ("device", ctypes.c_int),
                ("batch_fields", ctypes.c_int), ("stream_mode", ctypes.c_int), ("input_format", ctypes.c_int),
                ("dc_correct", ctypes.c_int), ("single_pass_lines", ctypes.c_int), ("guard_band_hz", ctypes.c_double),
                ("device_memory_limit_mb", ctypes.c_double)]


class FieldInfo(ctypes.Structure):
    _fields_ = [("file_loc", ctypes.c_uint64), ("is_first_field", ctypes.c_int32),
                ("field_phase_id", ctypes.c_int32), ("dropout_count", ctypes.c_int32),
                ("dropout_offset", ctypes.c_int32)]


class Output(ctypes.Structure):
    _fields_ = [("luma", ctypes.c_void_p), ("chroma", ctypes.c_void_p), ("fields", ctypes.c_void_p),
                ("dropout_line", ctypes.c_void_p), ("dropout_startx", ctypes.c_void_p),
                ("dropout_endx", ctypes.c_void_p), ("max_fields", ctypes.c_size_t),
                ("max_dropouts", ctypes.c_size_t), ("fields_out", ctypes.c_size_t),
                ("dropouts_out", ctypes.c_size_t), ("next_raw_offset", ctypes.c_uint64)]


class State(ctypes.Structure):
    """cuvhs_state: what a decode carries from chunk to chunk."""
    _fields_ = [("last_parity", ctypes.c_int32), ("prev_first_field", ctypes.c_int32),
                ("prev_progressive_field", ctypes.c_int32), ("chroma_valid", ctypes.c_int32),
                ("prev_first_hsync_readloc", ctypes.c_int64), ("prev_first_hsync_loc", ctypes.c_double),
                ("prev_first_hsync_diff", ctypes.c_double), ("chroma_threshold", ctypes.c_double),
                ("chroma_track", ctypes.c_int32), ("chroma_cycle_start", ctypes.c_int32)]

    def as_tuple(self):
        return tuple(getattr(self, k) for k, _ in self._fields_)


class BatchConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("lanes", ctypes.c_int), ("max_fields", ctypes.c_int),
                ("round_fields", ctypes.c_int)]


class BatchItem(ctypes.Structure):
    _fields_ = [("samples", ctypes.c_void_p), ("n", ctypes.c_size_t), ("sample_rate_mhz", ctypes.c_double),
                ("out", ctypes.POINTER(Output)), ("status", ctypes.c_int)]


class AdjointParams(ctypes.Structure):
    _fields_ = [("deemph", ctypes.c_double * 4), ("carrier_hz", ctypes.c_double), ("deviation", ctypes.c_double),
                ("line_offset", ctypes.c_void_p), ("chroma_phase", ctypes.c_void_p)]


class SynthParams(ctypes.Structure):
    _fields_ = [("sample_rate_hz", ctypes.c_double), ("n_fields", ctypes.c_int), ("tail_lines", ctypes.c_int),
                ("seed", ctypes.c_uint64), ("snr_db", ctypes.c_double), ("jitter_bound", ctypes.c_double),
                ("jitter_step", ctypes.c_double), ("dropout_line_rate", ctypes.c_double),
                ("dropout_min", ctypes.c_int), ("dropout_max", ctypes.c_int), ("headswitch_min", ctypes.c_int),
                ("headswitch_max", ctypes.c_int), ("speed_drift", ctypes.c_double),
                ("start_line", ctypes.c_double), ("chroma_level", ctypes.c_double),
                ("carrier_offset_hz", ctypes.c_double), ("deviation_scale", ctypes.c_double),
                ("first_track", ctypes.c_int), ("threads", ctypes.c_int),
                ("preemph_perturb", ctypes.c_double * 3), ("line_offset_bound", ctypes.c_double),
                ("chroma_phase_bound", ctypes.c_double), ("system", ctypes.c_int)]


_vp = ctypes.c_void_p
lib.cuvhs_default_config.argtypes = [ctypes.POINTER(Config)]
lib.cuvhs_create.argtypes = [ctypes.POINTER(Config), ctypes.POINTER(_vp)]
lib.cuvhs_create.restype = ctypes.c_int
lib.cuvhs_destroy.argtypes = [_vp]
lib.cuvhs_last_error.argtypes = [_vp]
lib.cuvhs_last_error.restype = ctypes.c_char_p
lib.cuvhs_status_string.argtypes = [ctypes.c_int]
lib.cuvhs_status_string.restype = ctypes.c_char_p
lib.cuvhs_batch_fields.argtypes = [_vp]
lib.cuvhs_samples_per_field.argtypes = [_vp]
lib.cuvhs_samples_per_field.restype = ctypes.c_size_t
lib.cuvhs_tile_stride.argtypes = [_vp]
lib.cuvhs_tile_stride.restype = ctypes.c_size_t
lib.cuvhs_reset.argtypes = [_vp]
lib.cuvhs_set_debug.argtypes = [_vp, ctypes.c_int]
lib.cuvhs_decode_chunk.argtypes = [_vp, _vp, ctypes.c_size_t, ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(Output)]
lib.cuvhs_decode_chunk.restype = ctypes.c_int
lib.cuvhs_decode_chunk_device.argtypes = [_vp, _vp, ctypes.c_size_t, ctypes.c_uint64, ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_uint64)]
lib.cuvhs_decode_chunk_device.restype = ctypes.c_int
lib.cuvhs_device_outputs.argtypes = [_vp, ctypes.POINTER(_vp), ctypes.POINTER(_vp)]
lib.cuvhs_device_outputs.restype = ctypes.c_int
lib.cuvhs_decode_capture.argtypes = [_vp, _vp, ctypes.c_size_t, ctypes.POINTER(Output)]
lib.cuvhs_decode_capture.restype = ctypes.c_int
lib.cuvhs_json.argtypes = [_vp, ctypes.POINTER(Output), ctypes.c_char_p, ctypes.c_longlong]
lib.cuvhs_json.restype = ctypes.c_longlong
lib.cuvhs_decode_file.argtypes = [ctypes.POINTER(Config), ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int]
lib.cuvhs_decode_file.restype = ctypes.c_int
lib.cuvhs_debug_array.argtypes = [_vp, ctypes.c_char_p, _vp, ctypes.c_longlong]
lib.cuvhs_debug_array.restype = ctypes.c_longlong
lib.cuvhs_stream.argtypes = [_vp]
lib.cuvhs_stream.restype = _vp
lib.cuvhs_set_timing.argtypes = [_vp, ctypes.c_int]
lib.cuvhs_stage_count.restype = ctypes.c_int
lib.cuvhs_stage_name.argtypes = [ctypes.c_int]
lib.cuvhs_stage_name.restype = ctypes.c_char_p
lib.cuvhs_stage_times.argtypes = [_vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong), ctypes.c_int]
lib.cuvhs_stage_times.restype = ctypes.c_int
lib.cuvhs_reset_stage_times.argtypes = [_vp]
lib.cuvhs_launch_count.argtypes = [_vp]
lib.cuvhs_launch_count.restype = ctypes.c_longlong
lib.cuvhs_dropouts_noalloc.argtypes = [_vp, _vp, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp]
lib.cuvhs_dropouts_noalloc.restype = ctypes.c_int
lib.cuvhs_batch_create.argtypes = [ctypes.POINTER(BatchConfig), ctypes.POINTER(_vp)]
lib.cuvhs_batch_create.restype = ctypes.c_int
lib.cuvhs_batch_destroy.argtypes = [_vp]
lib.cuvhs_batch_lanes.argtypes = [_vp]
lib.cuvhs_batch_lanes.restype = ctypes.c_int
lib.cuvhs_batch_round_fields.argtypes = [_vp, ctypes.c_double]
lib.cuvhs_batch_round_fields.restype = ctypes.c_int
lib.cuvhs_batch_set_timing.argtypes = [_vp, ctypes.c_int]
lib.cuvhs_batch_stage_times.argtypes = [_vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong),
                                        ctypes.c_int]
lib.cuvhs_batch_stage_times.restype = ctypes.c_int
lib.cuvhs_batch_decode.argtypes = [_vp, ctypes.POINTER(BatchItem), ctypes.c_int]
lib.cuvhs_batch_decode.restype = ctypes.c_int
lib.cuvhs_batch_last_error.argtypes = [_vp]
lib.cuvhs_batch_last_error.restype = ctypes.c_char_p
lib.cuvhs_batch_json.argtypes = [ctypes.POINTER(BatchItem), ctypes.c_char_p, ctypes.c_longlong]
lib.cuvhs_batch_json.restype = ctypes.c_longlong
lib.cuvhs_adjoint_create.argtypes = [ctypes.POINTER(Config), _vp, ctypes.c_size_t, ctypes.c_int, ctypes.POINTER(_vp)]
lib.cuvhs_adjoint_create.restype = ctypes.c_int
lib.cuvhs_adjoint_destroy.argtypes = [_vp]
lib.cuvhs_adjoint_fields.argtypes = [_vp]
lib.cuvhs_adjoint_fields.restype = ctypes.c_int
lib.cuvhs_adjoint_default_params.argtypes = [_vp, ctypes.POINTER(AdjointParams)]
lib.cuvhs_adjoint_default_params.restype = ctypes.c_int
lib.cuvhs_adjoint_set_target.argtypes = [_vp, _vp, _vp]
lib.cuvhs_adjoint_set_target.restype = ctypes.c_int
lib.cuvhs_adjoint_fwd.argtypes = [_vp, ctypes.POINTER(AdjointParams), ctypes.POINTER(ctypes.c_double), _vp, _vp]
lib.cuvhs_adjoint_fwd.restype = ctypes.c_int
lib.cuvhs_adjoint_bwd.argtypes = [_vp, ctypes.POINTER(AdjointParams), ctypes.POINTER(ctypes.c_double),
                                  ctypes.POINTER(AdjointParams)]
lib.cuvhs_adjoint_bwd.restype = ctypes.c_int
lib.cuvhs_adjoint_array.argtypes = [_vp, ctypes.c_char_p, _vp, ctypes.c_longlong]
lib.cuvhs_adjoint_array.restype = ctypes.c_longlong
lib.cuvhs_synth_default_params.argtypes = [ctypes.POINTER(SynthParams)]
lib.cuvhs_synth_length.argtypes = [ctypes.POINTER(SynthParams)]
lib.cuvhs_synth_length.restype = ctypes.c_longlong
lib.cuvhs_synth_ntsc.argtypes = [ctypes.POINTER(SynthParams), _vp, ctypes.c_longlong]
lib.cuvhs_synth_ntsc.restype = ctypes.c_int
lib.cuvhs_synth_open.argtypes = [ctypes.POINTER(SynthParams), ctypes.c_longlong]
lib.cuvhs_synth_open.restype = _vp
lib.cuvhs_synth_next.argtypes = [_vp, _vp, ctypes.c_longlong]
lib.cuvhs_synth_next.restype = ctypes.c_longlong
lib.cuvhs_synth_close.argtypes = [_vp]
lib.cuvhs_synth_lines.argtypes = [ctypes.POINTER(SynthParams), ctypes.c_longlong, _vp, _vp, _vp, ctypes.c_longlong]
lib.cuvhs_synth_lines.restype = ctypes.c_longlong
lib.cuvhs_synth_preemphasis.argtypes = [ctypes.POINTER(SynthParams), _vp, _vp]
lib.cuvhs_field_width.argtypes = [_vp]
lib.cuvhs_field_width.restype = ctypes.c_int
lib.cuvhs_field_height.argtypes = [_vp]
lib.cuvhs_field_height.restype = ctypes.c_int
lib.cuvhs_lines_per_frame.argtypes = [_vp]
lib.cuvhs_lines_per_frame.restype = ctypes.c_int
lib.cuvhs_set_timing_mask.argtypes = [_vp, ctypes.c_uint]
lib.cuvhs_stage_timeline.argtypes = [_vp, _vp, _vp, _vp, ctypes.c_int]
lib.cuvhs_stage_timeline.restype = ctypes.c_int
lib.cuvhs_decode_chunk_async.argtypes = [_vp, _vp, ctypes.c_size_t, ctypes.c_uint64, ctypes.c_int,
                                         ctypes.POINTER(Output)]
lib.cuvhs_decode_chunk_async.restype = ctypes.c_int
lib.cuvhs_flush.argtypes = [_vp]
lib.cuvhs_flush.restype = ctypes.c_int
lib.cuvhs_ire0_hz.argtypes = [_vp]
lib.cuvhs_ire0_hz.restype = ctypes.c_double
lib.cuvhs_get_state.argtypes = [_vp, _vp]
lib.cuvhs_set_state.argtypes = [_vp, _vp]
lib.cuvhs_pulse_threshold_hz.argtypes = [_vp]
lib.cuvhs_pulse_threshold_hz.restype = ctypes.c_double
lib.cuvhs_stage_fm_demod.argtypes = [_vp, _vp, ctypes.c_size_t, ctypes.c_int, _vp, _vp, _vp]
lib.cuvhs_stage_fm_demod.restype = ctypes.c_int
lib.cuvhs_stage_discover_vsyncs.argtypes = [_vp, _vp, ctypes.c_int, ctypes.c_int, _vp, ctypes.POINTER(ctypes.c_int),
                                            ctypes.POINTER(ctypes.c_int64)]
lib.cuvhs_stage_discover_vsyncs.restype = ctypes.c_int
lib.cuvhs_stage_sync_pulses.argtypes = [_vp, _vp, ctypes.c_int, _vp, ctypes.c_int, _vp, _vp, _vp]
lib.cuvhs_stage_sync_pulses.restype = ctypes.c_int
lib.cuvhs_stage_line_locations.argtypes = [_vp, ctypes.c_uint64, _vp, ctypes.c_int, _vp, _vp, _vp, _vp, _vp]
lib.cuvhs_stage_line_locations.restype = ctypes.c_int
lib.cuvhs_stage_hsync_refine.argtypes = [_vp, _vp, ctypes.c_int, _vp, ctypes.c_int]
lib.cuvhs_stage_hsync_refine.restype = ctypes.c_int
lib.cuvhs_stage_tbc_resample.argtypes = [_vp, _vp, ctypes.c_int, _vp, ctypes.c_int, _vp]
lib.cuvhs_stage_tbc_resample.restype = ctypes.c_int
lib.cuvhs_stage_chroma_decode.argtypes = [_vp, _vp, ctypes.c_size_t, _vp, ctypes.c_int, _vp, _vp]
lib.cuvhs_stage_chroma_decode.restype = ctypes.c_int

# every symbol include/cuvhs.h and include/cuvhs_synth.h declare
EXPORTED = [
    "cuvhs_default_config", "cuvhs_create", "cuvhs_destroy", "cuvhs_last_error", "cuvhs_status_string",
    "cuvhs_batch_fields", "cuvhs_samples_per_field", "cuvhs_tile_stride", "cuvhs_reset", "cuvhs_decode_chunk",
    "cuvhs_decode_chunk_device", "cuvhs_device_outputs", "cuvhs_decode_capture", "cuvhs_json",
    "cuvhs_decode_file", "cuvhs_set_debug", "cuvhs_debug_array", "cuvhs_stream", "cuvhs_set_timing",
    "cuvhs_stage_count", "cuvhs_stage_name", "cuvhs_stage_times", "cuvhs_reset_stage_times", "cuvhs_launch_count",
    "cuvhs_dropouts_noalloc", "cuvhs_batch_create", "cuvhs_batch_destroy", "cuvhs_batch_lanes",
    "cuvhs_batch_decode", "cuvhs_batch_last_error", "cuvhs_batch_json", "cuvhs_batch_round_fields",
    "cuvhs_batch_set_timing", "cuvhs_batch_stage_times",
    "cuvhs_adjoint_create",
    "cuvhs_adjoint_destroy", "cuvhs_adjoint_fields", "cuvhs_adjoint_default_params", "cuvhs_adjoint_set_target",
    "cuvhs_adjoint_fwd", "cuvhs_adjoint_bwd", "cuvhs_adjoint_array", "cuvhs_synth_default_params",
    "cuvhs_synth_length", "cuvhs_synth_ntsc", "cuvhs_synth_lines", "cuvhs_synth_preemphasis",
    "cuvhs_synth_open", "cuvhs_synth_next", "cuvhs_synth_close",
    "cuvhs_decode_chunk_async", "cuvhs_flush", "cuvhs_ire0_hz", "cuvhs_pulse_threshold_hz", "cuvhs_get_state",
    "cuvhs_set_state", "cuvhs_stage_fm_demod",
    "cuvhs_stage_discover_vsyncs", "cuvhs_stage_sync_pulses", "cuvhs_stage_line_locations",
    "cuvhs_stage_hsync_refine", "cuvhs_stage_tbc_resample", "cuvhs_stage_chroma_decode",
    "cuvhs_field_width", "cuvhs_field_height", "cuvhs_lines_per_frame", "cuvhs_stage_timeline",
    "cuvhs_set_timing_mask",
]


def synth_params(**kw) -> SynthParams:
    p = SynthParams()
    lib.cuvhs_synth_default_params(ctypes.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        if k == "preemph_perturb":
            v = (ctypes.c_double * 3)(*v)
        setattr(p, k, v)
    return p


def synth_lines(**kw):
    """Program-line table of a synthetic capture: (start sample, picture
    delay in samples, colour-under phase offset in radians) per line."""
    p = synth_params(**kw)
    n = lib.cuvhs_synth_length(ctypes.byref(p))
    m = lib.cuvhs_synth_lines(ctypes.byref(p), n, None, None, None, 0)
    st, off, ph = (np.empty(m, np.float64) for _ in range(3))
    lib.cuvhs_synth_lines(ctypes.byref(p), n, st.ctypes.data, off.ctypes.data, ph.ctypes.data, m)
    return st, off, ph


def synth_preemphasis(**kw):
    """(b, a) of the capture's pre-emphasis biquad, a[0] = 1."""
    p = synth_params(**kw)
    b = np.empty(3, np.float64)
    a = np.empty(3, np.float64)
    lib.cuvhs_synth_preemphasis(ctypes.byref(p), b.ctypes.data, a.ctypes.data)
    return b, a


class SynthStream:
    """A synthetic capture generated front to back in pieces (cuvhs_synth_open /
    next / close): the pieces concatenate to synth_capture(**kw), with a few
    tens of MB of working memory however long the capture is."""

    def __init__(self, **kw):
        self._p = synth_params(**kw)
        self.length = int(lib.cuvhs_synth_length(ctypes.byref(self._p)))
        self._h = lib.cuvhs_synth_open(ctypes.byref(self._p), self.length)
        if not self._h:
            raise CuvhsError(1, "cuvhs_synth_open failed")
        self.position = 0

    def read_into(self, out) -> int:
        """Fill the writable u8 buffer `out` (numpy array or pointer-sized
        object with .ctypes) with the next samples; returns how many."""
        got = lib.cuvhs_synth_next(self._h, out.ctypes.data, out.size)
        if got < 0:
            raise CuvhsError(1, "cuvhs_synth_next failed")
        self.position += int(got)
        return int(got)

    def close(self):
        if getattr(self, "_h", None):
            lib.cuvhs_synth_close(self._h)
            self._h = None

    def __del__(self):
        self.close()


def synth_capture(**kw) -> np.ndarray:
    """Seeded synthetic NTSC VHS RF capture (u8)."""
    p = synth_params(**kw)
    n = lib.cuvhs_synth_length(ctypes.byref(p))
    buf = np.empty(n, np.uint8)
    rc = lib.cuvhs_synth_ntsc(ctypes.byref(p), buf.ctypes.data, ctypes.c_longlong(n))
    if rc != 0:
        raise CuvhsError(1, f"synthesizer returned {rc}")
    return buf


@dataclass
class DecodeResult:
    luma: np.ndarray          # [fields, rows, columns] u16: 263 x 910 NTSC, 313 x 1135 PAL
    chroma: np.ndarray        # [fields, rows, columns] u16
    file_loc: np.ndarray      # [fields] u64
    is_first_field: np.ndarray
    field_phase_id: np.ndarray
    dropouts: list = field(default_factory=list)  # per field: (line, startx, endx) int32 arrays
    json: str = ""

    @property
    def n_fields(self):
        return self.luma.shape[0]


def max_fields_for(n_samples, samples_per_field):
    """Output room for a capture: its nominal field count plus 1% (tape running
    fast packs more fields into the same samples) and a few fields."""
    return int(n_samples / samples_per_field * 1.01) + 4


def alloc_output(max_fields, pinned=False, shape=(FIELD_H, FIELD_W)):
    """Host output buffers for max_fields fields of `shape` (rows, columns;
    NTSC by default), page-locked when pinned."""
    if pinned:
        import torch
        planes = [torch.empty((max_fields,) + tuple(shape), dtype=torch.int16, pin_memory=True) for _ in range(2)]
        luma, chroma = (p.numpy().view(np.uint16) for p in planes)
    else:
        planes = []
        luma = np.empty((max_fields,) + tuple(shape), np.uint16)
        chroma = np.empty((max_fields,) + tuple(shape), np.uint16)
    bufs = {
        "planes": planes,
        "luma": luma,
        "chroma": chroma,
        "fields": (FieldInfo * max_fields)(),
        "dl": np.empty(max_fields * MAX_DROPOUTS_PER_FIELD, np.int32),
        "ds": np.empty(max_fields * MAX_DROPOUTS_PER_FIELD, np.int32),
        "de": np.empty(max_fields * MAX_DROPOUTS_PER_FIELD, np.int32),
    }
    out = Output()
    out.luma = bufs["luma"].ctypes.data
    out.chroma = bufs["chroma"].ctypes.data
    out.fields = ctypes.addressof(bufs["fields"])
    out.dropout_line = bufs["dl"].ctypes.data
    out.dropout_startx = bufs["ds"].ctypes.data
    out.dropout_endx = bufs["de"].ctypes.data
    out.max_fields = max_fields
    out.max_dropouts = max_fields * MAX_DROPOUTS_PER_FIELD
    return out, bufs


def collect_result(out, bufs, json_text):
    """DecodeResult from a filled cuvhs_output (json_text() gives the .tbc.json)."""
    n = out.fields_out
    fi = bufs["fields"]
    dropouts = []
    for i in range(n):
        o, c = fi[i].dropout_offset, fi[i].dropout_count
        dropouts.append((bufs["dl"][o:o + c].copy(), bufs["ds"][o:o + c].copy(), bufs["de"][o:o + c].copy()))
    own = (lambda a: a.copy()) if bufs["planes"] else (lambda a: a)  # pinned staging is not kept
    return DecodeResult(
        luma=own(bufs["luma"][:n]), chroma=own(bufs["chroma"][:n]),
        file_loc=np.array([fi[i].file_loc for i in range(n)], np.uint64),
        is_first_field=np.array([fi[i].is_first_field for i in range(n)], np.int32),
        field_phase_id=np.array([fi[i].field_phase_id for i in range(n)], np.int32),
        dropouts=dropouts, json=json_text())


class Decoder:
    """One libcuvhs context (device memory and stream, carried decode state)."""

    FORMATS = {"u8": (0, np.uint8), "s16": (1, np.int16), "u16": (2, np.uint16)}
    SYSTEMS = {"NTSC": 0, "PAL": 1}

    def __init__(self, sample_rate_mhz=28.0, device=0, batch_fields=0, stream_mode=False, debug=False,
                 input_format="u8", dc_correct=False, system="NTSC", single_pass_lines=False, guard_band_hz=0.0,
                 device_memory_limit_mb=0.0):
        cfg = Config()
        lib.cuvhs_default_config(ctypes.byref(cfg))
        cfg.guard_band_hz = float(guard_band_hz)
        cfg.device_memory_limit_mb = float(device_memory_limit_mb)
        cfg.system = self.SYSTEMS[system.upper()]
        cfg.single_pass_lines = 1 if single_pass_lines else 0
        cfg.sample_rate_mhz = float(sample_rate_mhz)
        cfg.device = int(device)
        cfg.batch_fields = int(batch_fields)
        cfg.stream_mode = 1 if stream_mode else 0
        cfg.input_format, self._dtype = self.FORMATS[input_format]
        cfg.dc_correct = 1 if dc_correct else 0
        h = _vp()
        st = lib.cuvhs_create(ctypes.byref(cfg), ctypes.byref(h))
        if st != 0:
            raise CuvhsError(st, "cuvhs_create failed")
        self._h = h
        # held by the instance so that close() still works while the module's
        # globals are torn down at interpreter exit
        self._lib = lib
        if debug:
            lib.cuvhs_set_debug(self._h, 1)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.cuvhs_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def batch_fields(self):
        return lib.cuvhs_batch_fields(self._h)

    @property
    def samples_per_field(self):
        return lib.cuvhs_samples_per_field(self._h)

    @property
    def tile_stride(self):
        return lib.cuvhs_tile_stride(self._h)

    @property
    def field_shape(self):
        """(rows, columns) of an output field: (263, 910) NTSC, (313, 1135) PAL."""
        return lib.cuvhs_field_height(self._h), lib.cuvhs_field_width(self._h)

    @property
    def lines_per_frame(self):
        return lib.cuvhs_lines_per_frame(self._h)

    def reset(self):
        lib.cuvhs_reset(self._h)

    def get_state(self) -> "State":
        st = State()
        self._check(lib.cuvhs_get_state(self._h, ctypes.byref(st)))
        return st

    def set_state(self, st: "State"):
        self._check(lib.cuvhs_set_state(self._h, ctypes.byref(st)))

    def _check(self, st):
        if st != 0:
            raise CuvhsError(st, lib.cuvhs_last_error(self._h).decode())

    def _alloc_output(self, max_fields, pinned=False):
        return alloc_output(max_fields, pinned, self.field_shape)

    def _result(self, out, bufs):
        def json_text():
            jl = lib.cuvhs_json(self._h, ctypes.byref(out), None, 0)
            jb = ctypes.create_string_buffer(int(jl) + 1)
            lib.cuvhs_json(self._h, ctypes.byref(out), jb, jl + 1)
            return jb.value.decode()
        return collect_result(out, bufs, json_text)

    def decode_capture(self, samples: np.ndarray, pinned: bool = False) -> DecodeResult:
        """Decode a whole capture.  pinned=True stages the input and the output
        planes in page-locked memory, which lets the library overlap the
        host<->device copies with the decode."""
        samples = np.ascontiguousarray(samples, dtype=self._dtype)
        max_fields = max_fields_for(samples.size, self.samples_per_field)
        out, bufs = self._alloc_output(max_fields, pinned)
        if pinned:
            import torch
            pin = torch.from_numpy(samples).pin_memory()
            bufs["input"] = pin
            src = pin.data_ptr()
        else:
            src = samples.ctypes.data
        self._check(lib.cuvhs_decode_capture(self._h, src, samples.size, ctypes.byref(out)))
        return self._result(out, bufs)

    def decode_chunk(self, samples: np.ndarray, raw_offset: int, num_fields: int):
        """One reference-style chunk; `samples` starts at capture sample raw_offset."""
        samples = np.ascontiguousarray(samples, dtype=self._dtype)
        out, bufs = self._alloc_output(num_fields)
        self._check(lib.cuvhs_decode_chunk(self._h, samples.ctypes.data, samples.size, raw_offset, num_fields,
                                           ctypes.byref(out)))
        return self._result(out, bufs), int(out.next_raw_offset)

    def decode_chunks_async(self, samples: np.ndarray, num_fields: int = 0) -> DecodeResult:
        """A capture chunk by chunk through cuvhs_decode_chunk_async into
        page-locked planes (each chunk's plane copies overlap the next chunk's
        decode), completed by cuvhs_flush."""
        samples = np.ascontiguousarray(samples, dtype=self._dtype)
        nf = num_fields or self.batch_fields
        spf = self.samples_per_field
        out, bufs = self._alloc_output(max_fields_for(samples.size, spf), pinned=True)
        raw = 0
        while raw < samples.size and (samples.size - raw) // spf > 0:
            before = out.fields_out
            n = min(nf, (samples.size - raw) // spf)
            st = lib.cuvhs_decode_chunk_async(self._h, samples[raw:].ctypes.data, samples.size - raw, raw, n,
                                              ctypes.byref(out))
            if st != 0:
                lib.cuvhs_flush(self._h)
                self._check(st)
            if out.fields_out == before:
                break
            raw = int(out.next_raw_offset)
        self._check(lib.cuvhs_flush(self._h))
        return self._result(out, bufs)

    def decode_chunk_device(self, d_ptr: int, n_avail: int, raw_offset: int, num_fields: int):
        fo = ctypes.c_int(0)
        nxt = ctypes.c_uint64(0)
        self._check(lib.cuvhs_decode_chunk_device(self._h, _vp(d_ptr), n_avail, raw_offset, num_fields,
                                                  ctypes.byref(fo), ctypes.byref(nxt)))
        return fo.value, nxt.value

    _DTYPES = {"field_offsets": np.int64, "linelocs_coarse": np.float64, "linelocs": np.float64,
               "guard_positions": np.int64, "guard_values": np.float64,
               "lineloc_clocks": np.int64, "guard_clocks": np.int64,
               "demod": np.float32, "video": np.float32, "sync": np.float32, "envelope": np.float32,
               "chroma_prefilt": np.float32}

    @property
    def stream(self) -> int:
        return lib.cuvhs_stream(self._h) or 0

    def set_timing(self, on=True, stages=None):
        """Per-stage CUDA-event timing; `stages` (names) restricts the events
        to those stages (default all)."""
        if stages is None:
            mask = 0xFFFFFFFF
        else:
            names = [lib.cuvhs_stage_name(i).decode() for i in range(lib.cuvhs_stage_count())]
            mask = sum(1 << names.index(n) for n in stages)
        lib.cuvhs_set_timing_mask(self._h, mask)
        lib.cuvhs_set_timing(self._h, 1 if on else 0)

    def reset_stage_times(self):
        lib.cuvhs_reset_stage_times(self._h)

    def stage_times(self) -> dict:
        n = lib.cuvhs_stage_count()
        ms = (ctypes.c_double * n)()
        la = (ctypes.c_longlong * n)()
        lib.cuvhs_stage_times(self._h, ms, la, n)
        return {lib.cuvhs_stage_name(i).decode(): (ms[i], la[i]) for i in range(n)}

    def stage_timeline(self):
        """[(stage name, start ms, end ms)] of the last chunk's device stages
        (timing on), from its first timed event."""
        n = lib.cuvhs_stage_timeline(self._h, None, None, None, 0)
        st = np.zeros(n, np.int32)
        a = np.zeros(n)
        b = np.zeros(n)
        if n:
            lib.cuvhs_stage_timeline(self._h, st.ctypes.data, a.ctypes.data, b.ctypes.data, n)
        return [(lib.cuvhs_stage_name(int(k)).decode(), float(x), float(y)) for k, x, y in zip(st, a, b)]

    @property
    def launch_count(self) -> int:
        return lib.cuvhs_launch_count(self._h)

    def debug_array(self, name: str) -> np.ndarray:
        n = lib.cuvhs_debug_array(self._h, name.encode(), None, 0)
        if n < 0:
            raise KeyError(name)
        a = np.empty(n, self._DTYPES.get(name, np.int32))
        if n:
            lib.cuvhs_debug_array(self._h, name.encode(), a.ctypes.data, n)
        return a


class Batch:
    """cuvhs_batch: many independent captures (mixed rates) decoded together in
    batched rounds (round_fields: field slots per round, 0 = autotune)."""

    def __init__(self, lanes=0, max_fields=0, device=0, round_fields=0):
        cfg = BatchConfig(int(device), int(lanes), int(max_fields), int(round_fields))
        h = _vp()
        st = lib.cuvhs_batch_create(ctypes.byref(cfg), ctypes.byref(h))
        if st != 0:
            raise CuvhsError(st, "cuvhs_batch_create failed")
        self._h = h

    @property
    def lanes(self):
        return lib.cuvhs_batch_lanes(self._h)

    def round_fields(self, sample_rate_mhz):
        """Field slots per round in use for this sample rate (0 before first use)."""
        return lib.cuvhs_batch_round_fields(self._h, float(sample_rate_mhz))

    def set_timing(self, on=True):
        lib.cuvhs_batch_set_timing(self._h, 1 if on else 0)

    def stage_times(self):
        """{stage: (ms, launches)} summed over the batch's contexts."""
        n = lib.cuvhs_stage_count()
        ms = (ctypes.c_double * n)()
        ln = (ctypes.c_longlong * n)()
        lib.cuvhs_batch_stage_times(self._h, ms, ln, n)
        return {lib.cuvhs_stage_name(i).decode(): (ms[i], ln[i]) for i in range(n)}

    def close(self):
        if getattr(self, "_h", None):
            lib.cuvhs_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def prepare(self, captures, pinned=False):
        """Items and buffers for [(samples u8, sample_rate_mhz), ...]; pinned
        stages inputs and output planes in page-locked memory."""
        items = (BatchItem * len(captures))()
        keep = []
        for i, (x, mhz) in enumerate(captures):
            x = np.ascontiguousarray(x, dtype=np.uint8)
            spf = int(round(mhz * 1e6 / (525 * 30 / 1.001))) * 263
            out, bufs = alloc_output(max_fields_for(x.size, spf), pinned)
            if pinned:
                import torch
                t = torch.from_numpy(x).pin_memory()
                bufs["input"] = t
                items[i].samples = t.data_ptr()
            else:
                bufs["input"] = x
                items[i].samples = x.ctypes.data
            items[i].n = x.size
            items[i].sample_rate_mhz = float(mhz)
            bufs["out"] = out
            items[i].out = ctypes.pointer(out)
            keep.append(bufs)
        return items, keep

    def run(self, items):
        st = lib.cuvhs_batch_decode(self._h, items, len(items))
        if st != 0:
            raise CuvhsError(st, lib.cuvhs_batch_last_error(self._h).decode())

    def results(self, items, keep):
        res = []
        for i, bufs in enumerate(keep):
            it = items[i]

            def json_text(it=it):
                jl = lib.cuvhs_batch_json(ctypes.byref(it), None, 0)
                jb = ctypes.create_string_buffer(int(jl) + 1)
                lib.cuvhs_batch_json(ctypes.byref(it), jb, jl + 1)
                return jb.value.decode()
            res.append(collect_result(bufs["out"], bufs, json_text))
        return res

    def decode(self, captures, pinned=False):
        """Decode [(samples, sample_rate_mhz), ...]; one DecodeResult per capture."""
        items, keep = self.prepare(captures, pinned)
        self.run(items)
        return self.results(items, keep)


def decode_file(in_path, out_base, sample_rate_mhz=28.0, device=0, overwrite=True, batch_fields=0,
                input_format="u8", dc_correct=False, system="NTSC"):
    cfg = Config()
    lib.cuvhs_default_config(ctypes.byref(cfg))
    cfg.system = Decoder.SYSTEMS[system.upper()]
    cfg.sample_rate_mhz = float(sample_rate_mhz)
    cfg.device = int(device)
    cfg.batch_fields = int(batch_fields)
    cfg.input_format = Decoder.FORMATS[input_format][0]
    cfg.dc_correct = 1 if dc_correct else 0
    st = lib.cuvhs_decode_file(ctypes.byref(cfg), str(in_path).encode(), str(out_base).encode(), 1 if overwrite else 0)
    if st != 0:
        raise CuvhsError(st, "cuvhs_decode_file failed")
