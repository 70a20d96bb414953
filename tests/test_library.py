"""Host-side checks that need no GPU: the C ABI exports, the synthesizer, the
CLI's argument handling and its failure paths."""
import ctypes
import hashlib
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, has_gpu

import cuvhs_b200 as cv


def declared_functions():
    names = []
    for h in ("cuvhs.h", "cuvhs_synth.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(cuvhs_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) >= 20
    lib = ctypes.CDLL(cv.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(cv.EXPORTED) == names


def test_synthesizer_is_seeded_and_thread_independent():
    a = cv.make_workload("small28")
    assert hashlib.md5(a.tobytes()).hexdigest() == "d0de38e166bc329e2c86f18cdce4e8b3"
    b = cv.make_workload("small28", threads=1)
    assert np.array_equal(a, b)
    c = cv.make_workload("small28", seed=8)
    assert not np.array_equal(a, c)


def test_synthesizer_spectrum():
    x = cv.make_workload("small28")[: 1 << 20].astype(np.float64) - 128
    X = np.abs(np.fft.rfft(x * np.hanning(x.size))) ** 2
    f = np.fft.rfftfreq(x.size, 1 / 28e6)
    carrier = X[(f > 3.3e6) & (f < 4.5e6)].sum()
    under = X[(f > 0.5e6) & (f < 0.8e6)].sum()
    assert carrier > 20 * X[(f > 8e6)].sum()
    assert under > 0.005 * carrier


def run_cli(*args):
    return subprocess.run([cv.CLI_PATH, *args], capture_output=True, text=True, timeout=60)


def test_cli_usage_errors(tmp_path):
    assert run_cli().returncode == 1
    assert run_cli("--bogus", "a", "b").returncode == 1
    r = run_cli("a", "b", "c")
    assert r.returncode == 1 and "Too many arguments" in r.stderr
    assert run_cli("--system", "SECAM", "a", "b").returncode == 1
    assert run_cli("--format", "f32", "a", "b").returncode == 1
    assert run_cli("-h").returncode == 0


def test_cli_refuses_existing_outputs(tmp_path):
    inp = tmp_path / "in.u8"
    inp.write_bytes(bytes(1000))
    base = tmp_path / "out"
    (tmp_path / "out.tbc").write_bytes(b"")
    r = run_cli("-f", "28", str(inp), str(base))
    assert r.returncode == 1
    assert "Output exists" in r.stderr


def test_cli_system_argument(tmp_path):
    """--system takes NTSC or PAL (case-insensitive, src/main.cpp:52-56); anything
    else is an argument error.  PAL passes parsing and fails here only on the
    missing input file."""
    r = run_cli("--overwrite", "--system", "SECAM", str(tmp_path / "x.u8"), str(tmp_path / "o"))
    assert r.returncode == 1 and "Unknown system" in r.stderr
    r = run_cli("--overwrite", "--system", "pal", str(tmp_path / "x.u8"), str(tmp_path / "o"))
    assert r.returncode == 1 and "Unknown system" not in r.stderr and "I/O error" in r.stderr


def test_oracle_16_bit_inputs_and_dc_correction():
    """The oracle's --format / --dc-correct restatement (src/io/raw_reader.cpp:71-99):
    s16 and u16 samples of the u8 capture's converted values decode to the same
    bytes; DC correction removes an added constant offset up to FP64 rounding."""
    from oracle.oracle import Oracle
    x = cv.make_workload("small28")
    v = (x.astype(np.int32) - 128) * 256
    outs = []
    for fmt, y, dc in (("u8", x, False), ("s16", v.astype(np.int16), False),
                       ("u16", (v + 32768).astype(np.uint16), False),
                       ("s16", np.clip(v + 2500, -32768, 32767).astype(np.int16), True)):
        o = Oracle(28.0, input_format=fmt, dc_correct=dc)
        o.decode(y)
        outs.append(o)
    for o in outs[1:3]:
        assert o.json == outs[0].json
        assert np.array_equal(o.luma, outs[0].luma) and np.array_equal(o.chroma, outs[0].chroma)
    assert outs[3].n_fields == outs[0].n_fields


def test_cli_missing_input_fails(tmp_path):
    r = run_cli("--overwrite", str(tmp_path / "nope.u8"), str(tmp_path / "o"))
    assert r.returncode == 1


@pytest.mark.skipif(has_gpu(), reason="checks the no-device error path")
def test_create_without_device_reports_error():
    with pytest.raises(cv.CuvhsError) as e:
        cv.Decoder(28.0)
    assert e.value.status == 2


def test_invalid_config_rejected():
    cfg = cv._lib.Config()
    cv.lib.cuvhs_default_config(ctypes.byref(cfg))
    cfg.system = 2  # neither NTSC (0) nor PAL (1)
    h = ctypes.c_void_p()
    assert cv.lib.cuvhs_create(ctypes.byref(cfg), ctypes.byref(h)) == 1
    cfg.system = 0
    cfg.input_format = 3
    assert cv.lib.cuvhs_create(ctypes.byref(cfg), ctypes.byref(h)) == 1
    cfg.input_format = 0
    cfg.sample_rate_mhz = 1.0
    assert cv.lib.cuvhs_create(ctypes.byref(cfg), ctypes.byref(h)) == 1
    assert cv.lib.cuvhs_create(None, ctypes.byref(h)) == 1


@pytest.mark.parametrize("name", ["small28", "dropouts28pal"])
def test_synth_tool_writes_the_workload_bytes(name, tmp_path):
    """cuvhs-synth (the synthesizer without the decoder, used where a process
    must not load libcuvhs) writes the same bytes as make_workload."""
    import subprocess
    from cuvhs_b200.workload_table import WORKLOADS
    tool = os.path.join(os.path.dirname(cv.CLI_PATH), "cuvhs-synth")
    out = tmp_path / "in.u8"
    subprocess.run([tool] + [f"{k}={v}" for k, v in WORKLOADS[name].items()] + [str(out)], check=True)
    assert np.array_equal(np.fromfile(out, np.uint8), cv.make_workload(name))


def test_synth_tool_rejects_unknown_parameters(tmp_path):
    import subprocess
    tool = os.path.join(os.path.dirname(cv.CLI_PATH), "cuvhs-synth")
    r = subprocess.run([tool, "no_such_field=1", str(tmp_path / "x.u8")], capture_output=True, text=True)
    assert r.returncode == 2 and "bad parameter" in r.stderr


def test_synth_stream_pieces_concatenate_to_the_capture():
    """The chunked synthesizer (cuvhs_synth_open/next/close), read in ragged
    pieces across several internal units, gives the one-piece capture's
    bytes -- with drift, dropouts and head switching, whose state carries
    across the pieces."""
    kw = dict(sample_rate_hz=40e6, n_fields=16, seed=5001, snr_db=36, jitter_bound=1.0, dropout_line_rate=0.002,
              headswitch_min=3, headswitch_max=8, speed_drift=0.002)
    whole = cv.synth_capture(**kw)
    s = cv.SynthStream(**kw)
    assert s.length == whole.size
    rng = np.random.default_rng(3)
    parts = []
    while s.position < s.length:
        buf = np.empty(int(rng.integers(1, 3_000_000)), np.uint8)
        got = s.read_into(buf)
        assert got > 0
        parts.append(buf[:got])
    s.close()
    assert np.array_equal(np.concatenate(parts), whole)
