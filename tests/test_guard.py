"""The FP64 guard band of the sync threshold decisions.

The reference compares FP64 sync samples with the pulse threshold; the decoder
computes sync in FP32 and re-evaluates in FP64 every sample its K1b writes
within the guard band (8 Hz) of the threshold.  Checked on the GPU against the
FP64 oracle:

* every threshold decision of the first two field slots (about a million
  samples per case) is the oracle's, including a capture whose sync tip sits
  1 Hz above the threshold (thousands of samples inside the band);
* outside the band the FP32 sync is within a quarter of the band of the FP64
  sync (the assumption the band rests on);
* the FP64 values the guard computes agree with the oracle's FP64 sync within
  1e-4 Hz, over thousands of samples listed with a 10-30 kHz band, and that
  wide band leaves the decode's outputs unchanged."""
import numpy as np
import pytest

import cuvhs_b200 as cv
from conftest import inside_fields, json_fields, rate_mhz, system, workload
from cuvhs_b200 import lib

GUARD_HZ = 8.0
FP64_TOL_HZ = 1e-4


def _oracle_signals(name):
    from oracle.oracle import Oracle
    o = Oracle(rate_mhz(name), keep_signals=True, system=system(name))
    o.decode(workload(name))
    return o


def _decode(name, **kw):
    """(result, debug arrays, ire0 Hz, pulse threshold Hz) of a debug decode."""
    with cv.Decoder(rate_mhz(name), debug=True, system=system(name), **kw) as d:
        r = d.decode_capture(workload(name))
        dbg = {k: d.debug_array(k) for k in ("sync", "guard_positions", "guard_values")}
        ire0, thr = lib.cuvhs_ire0_hz(d._h), lib.cuvhs_pulse_threshold_hz(d._h)
    return r, dbg, ire0, thr


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["small28", "dropouts28", "small358", "pal20_40", "tipthr28"])
def test_threshold_decisions_are_the_fp64_ones(name):
    r, dbg, ire0, thr = _decode(name)
    o = _oracle_signals(name)
    s64 = o.array(0, "demod05")
    n = dbg["sync"].size
    assert n > 0 and s64.size >= n
    mine = dbg["sync"] <= np.float32(thr - ire0)  # the comparison every later stage makes
    ref = s64[:n] <= thr                          # the reference's FP64 decision
    bad = np.flatnonzero(mine != ref)
    assert bad.size == 0, (name, bad[:10], s64[bad[:10]] - thr)
    # the band's premise: away from the threshold the FP32 error stays well inside it
    s32 = dbg["sync"].astype(np.float64) + ire0
    far = np.abs(s32 - thr) >= GUARD_HZ
    err = np.abs(s32[far] - s64[:n][far])
    assert err.max() < GUARD_HZ / 4, (name, float(err.max()))
    if name == "tipthr28":
        assert dbg["guard_positions"].size > 1000, dbg["guard_positions"].size


@pytest.mark.gpu
@pytest.mark.parametrize("name,band", [("small28", 3.0e4), ("small358", 3.0e4), ("pal20_40", 1.0e4)])
def test_guard_fp64_values_match_the_oracle(name, band):
    # the band lists a few thousand samples (the chunk's list holds 65,536)
    wide, dbg, _, _ = _decode(name, guard_band_hz=band)
    o = _oracle_signals(name)
    s64 = o.array(0, "demod05")
    pos, vals = dbg["guard_positions"], dbg["guard_values"]
    x = workload(name)
    keep = pos + 16384 < x.size  # analysis windows clear of the zero fill past the capture
    assert keep.sum() > 2000, keep.sum()
    diff = np.abs(vals[keep] - s64[pos[keep]])
    assert diff.max() < FP64_TOL_HZ, (name, float(diff.max()))
    # a wider band changes no output
    base, _, _, _ = _decode(name)
    assert json_fields(wide.json) == json_fields(base.json)
    inside = inside_fields([f["fileLoc"] for f in json_fields(base.json)], x.size, rate_mhz(name), system(name))
    for i in inside:
        for a, b in ((wide.luma[i], base.luma[i]), (wide.chroma[i], base.chroma[i])):
            assert np.abs(a.astype(np.int32) - b.astype(np.int32)).max() <= 1, i
