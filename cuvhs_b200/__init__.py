"""cuvhs_b200: B200-native VHS RF decoder (drop-in for the hunterschuler/cuVHS decode path).

The decoder is libcuvhs (CUDA sm_100a kernels + C++ host code behind a C ABI,
include/cuvhs.h) and the `cuvhs` CLI; this package binds the library for
Python callers and tests.
"""
from ._lib import (CLI_PATH, LIB_PATH, Batch, CuvhsError, DecodeResult, Decoder, EXPORTED, FIELD_H, FIELD_W,
                   decode_file, lib, SynthStream, synth_capture, synth_lines, synth_params,
                   synth_preemphasis)
from .workloads import WORKLOADS, batch_specs, make_batch_workload, make_workload, system_of

__all__ = ["Decoder", "Batch", "DecodeResult", "CuvhsError", "decode_file", "SynthStream", "synth_capture", "synth_lines", "synth_params",
           "synth_preemphasis", "lib",
           "LIB_PATH", "CLI_PATH", "EXPORTED", "FIELD_W", "FIELD_H", "WORKLOADS", "make_workload",
           "batch_specs", "make_batch_workload", "system_of"]
