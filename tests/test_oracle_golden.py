"""The FP64 oracle against the reference decoder's own B200 outputs.

Fixtures (tests/golden/, made by tests/golden/make_golden.py from the
reference compiled from its sources) hold the reference's .tbc.json, per-field
digests of its luma/chroma TBC, its sync pulses before and after validation,
line locations, field parity and dropouts for seeded synthetic captures."""
import hashlib

import numpy as np
import pytest

from conftest import golden, inside_fields, json_fields, oracle_decode, single_pass, system, workload

CASES = ["small28", "dropouts28", "plain40_28", "small28pal", "dropouts28pal", "small28_singlepass",
         "dropouts28_singlepass", "small28pal_singlepass"]


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference(name):
    g = golden(name)
    x = workload(name)
    assert hashlib.md5(x.tobytes()).hexdigest() == str(g["input_md5"])
    o = oracle_decode(name)
    mhz = float(g["sample_rate_mhz"])
    locs = [f["fileLoc"] for f in json_fields(g["json_text"])]
    inside = inside_fields(locs, x.size, mhz, system(name))
    assert len(inside) >= len(locs) - 1
    # .tbc.json: the video parameters and every field inside the capture
    # identical (parity, phase IDs, file locations, dropouts); with the
    # validated line locations the whole text is identical, the field past the
    # end of the capture included
    ofields, gfields = json_fields(o.json), json_fields(g["json_text"])
    assert len(ofields) == len(gfields)
    assert o.json.split('"fields"')[0] == g["json_text"].split('"fields"')[0]
    for i in inside:
        assert ofields[i] == gfields[i], i
    if not single_pass(name):
        assert o.json == g["json_text"]
    # luma and chroma bit-identical on every field inside the capture
    for i in inside:
        assert hashlib.md5(o.luma[i].tobytes()).hexdigest() == str(g["luma_md5"][i]), i
        assert hashlib.md5(o.chroma[i].tobytes()).hexdigest() == str(g["chroma_md5"][i]), i
    assert np.array_equal(o.luma[0, ::16], g["luma_rows_f0"])
    # integer intermediates
    assert np.array_equal(o.array(0, "field_offsets"), g["field_offsets"])
    assert np.array_equal(o.array(0, "is_first"), g["is_first"])
    assert np.array_equal(o.array(0, "do_count"), g["do_count"])
    P = len(g["field_offsets"])
    for pre in ("k2", "k2b"):
        cnt = o.array(0, f"{pre}_pulse_count")
        off = np.concatenate([[0], np.cumsum(g[f"{pre}_count"])])
        for f in inside:
            assert cnt[f] == g[f"{pre}_count"][f], (pre, f)
            for part in ["starts", "lengths"] + (["types"] if pre == "k2b" else []):
                mine = o.array(0, f"{pre}_pulse_{part}").reshape(P, 800)[f, :cnt[f]]
                assert np.array_equal(mine, g[f"{pre}_{part}"][off[f]:off[f + 1]]), (pre, part, f)
    lpf, rows = o.lines_per_frame, o.field_shape[0] + 1  # the lines the resamplers read
    ll = o.array(0, "linelocs").reshape(P, lpf)
    llc = o.array(0, "linelocs_coarse").reshape(P, lpf)
    for f in inside:
        assert np.array_equal(llc[f, :rows], g["linelocs_coarse"][f, :rows])
        assert np.abs(ll[f, :rows] - g["linelocs"][f, :rows]).max() < 1e-6
