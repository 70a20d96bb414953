"""Python binding of the FP64 CPU oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, as the checker or the host-core baseline; the decoder never does.
The oracle restates the reference decoder (hunterschuler/cuVHS) in plain
C++ FP64 with the reference's tiling; its parity with the reference's own
CUDA build is pinned by the fixtures under tests/golden/.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
REF_HARNESS = os.path.join(HERE, "_ref", "ref_harness")
REF_CLI = os.path.join(HERE, "_ref", "cuvhs_ref")

F64_ARRAYS = ("linelocs_coarse", "linelocs", "demod", "demod05", "envelope", "chroma_prefilt")

_lib = None


def build():
    subprocess.check_call(["make", "-s", "-C", HERE, "oracle"])


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        L.oracle_create.restype = ctypes.c_void_p
        L.oracle_create.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_int]
        L.oracle_create_system.restype = ctypes.c_void_p
        L.oracle_create_system.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        for fn in ("oracle_field_width", "oracle_field_height", "oracle_lines_per_frame"):
            getattr(L, fn).argtypes = [ctypes.c_void_p]
        L.oracle_decode.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]
        L.oracle_luma.restype = ctypes.c_void_p
        L.oracle_luma.argtypes = [ctypes.c_void_p]
        L.oracle_chroma.restype = ctypes.c_void_p
        L.oracle_chroma.argtypes = [ctypes.c_void_p]
        L.oracle_json.restype = ctypes.c_char_p
        L.oracle_json.argtypes = [ctypes.c_void_p]
        L.oracle_num_fields.argtypes = [ctypes.c_void_p]
        L.oracle_num_chunks.argtypes = [ctypes.c_void_p]
        L.oracle_chunk_meta.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_longlong)]
        L.oracle_chunk_array.restype = ctypes.c_longlong
        L.oracle_chunk_array.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_void_p,
                                         ctypes.c_longlong]
        L.oracle_keep_signals.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.oracle_set_input.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.oracle_set_single_pass.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.oracle_destroy.argtypes = [ctypes.c_void_p]
        _lib = L
    return _lib


class Oracle:
    """One oracle decoder.  batch_fields is the reference's chunk size (its
    VRAM-derived batch; 3282 on a 180 GB B200 at 28 MHz)."""

    FORMATS = {"u8": (0, np.uint8), "s16": (1, np.int16), "u16": (2, np.uint16)}

    def __init__(self, sample_rate_mhz=28.0, batch_fields=3282, threads=0, keep_signals=False, input_format="u8",
                 dc_correct=False, system="NTSC", single_pass_lines=False):
        L = _load()
        self._h = L.oracle_create_system(float(sample_rate_mhz), int(batch_fields), int(threads),
                                         {"NTSC": 0, "PAL": 1}[system.upper()])
        self.field_shape = (L.oracle_field_height(self._h), L.oracle_field_width(self._h))
        self.lines_per_frame = L.oracle_lines_per_frame(self._h)
        if keep_signals:
            L.oracle_keep_signals(self._h, 1)
        fmt, self._dtype = self.FORMATS[input_format]
        L.oracle_set_input(self._h, fmt, 1 if dc_correct else 0)
        L.oracle_set_single_pass(self._h, 1 if single_pass_lines else 0)

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.oracle_destroy(self._h)
            self._h = None

    def decode(self, samples):
        L = _load()
        samples = np.ascontiguousarray(samples, self._dtype)
        n = L.oracle_decode(self._h, samples.ctypes.data, samples.size)
        self.n_fields = n
        P = ctypes.POINTER(ctypes.c_uint16)
        H, W = self.field_shape
        self.luma = np.ctypeslib.as_array(ctypes.cast(L.oracle_luma(self._h), P), (n * H * W,)).reshape(n, H, W).copy() \
            if n else np.zeros((0, H, W), np.uint16)
        self.chroma = np.ctypeslib.as_array(ctypes.cast(L.oracle_chroma(self._h), P), (n * H * W,)).reshape(n, H, W).copy() \
            if n else np.zeros((0, H, W), np.uint16)
        self.json = L.oracle_json(self._h).decode()
        return n

    @property
    def n_chunks(self):
        return _load().oracle_num_chunks(self._h)

    def chunk_meta(self, k):
        m = (ctypes.c_longlong * 6)()
        _load().oracle_chunk_meta(self._h, k, m)
        return dict(raw_offset=m[0], fields=m[1], spp=m[2], tiles=m[3], requested=m[4], next_raw_offset=m[5])

    def array(self, k, name):
        L = _load()
        cnt = L.oracle_chunk_array(self._h, k, name.encode(), None, 0)
        if cnt < 0:
            raise KeyError(name)
        dt = np.float64 if name in F64_ARRAYS else (np.int64 if name == "field_offsets" else np.int32)
        a = np.empty(cnt, dt)
        if cnt:
            L.oracle_chunk_array(self._h, k, name.encode(), a.ctypes.data, cnt)
        return a
