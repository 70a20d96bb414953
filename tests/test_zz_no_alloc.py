"""cuvhs_dropouts_noalloc: dropout detection and concealment for callers that
cannot allocate device memory (code under CUDA-graph stream capture, real-time
capture loops that must not block in an allocator, hosts whose device memory
another allocator owns).  Its scratch is a fixed device array inside the
library, so the tests check it against the decoder's own dropout stage
(cuvhs_decode_capture, which uses context-allocated scratch):

* on the unconcealed luma and chroma planes the stage entry points produce,
  two calls in a row must conceal them into exactly the decoder's planes and
  give exactly its dropout lists -- the second call reuses the array the first
  one left behind;
* after cudaDeviceReset the array is looked up again in the new context (a
  fresh process, so the reset ends no one else's context).

This file runs last in the suite and also passes alone in a fresh process."""
import ctypes
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

import cuvhs_b200 as cv
from cuvhs_b200 import lib, stages

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _u16(t):
    return t.cpu().numpy().view(np.uint16)


@pytest.mark.gpu
def test_dropouts_noalloc_matches_decoder_twice():
    import torch

    x = cv.make_workload("dropouts28")
    with cv.Decoder(28.0, debug=True) as d:
        r = d.decode_capture(x)
        cnt = d.debug_array("do_count")
        lines, sx, ex = (d.debug_array(k) for k in ("do_lines", "do_starts", "do_ends"))
        nf = min(d.batch_fields, x.size // d.samples_per_field)
    # the same chunk through the stage entry points: planes before concealment
    with cv.Decoder(28.0) as s:
        n_read = min(nf * s.tile_stride, x.size)
        T = min(n_read // s.samples_per_field, nf)
        raw = torch.from_numpy(x).cuda()
        video, sync, env = stages.fm_demod(s, raw, T, n_read)
        offs, _ = stages.discover_vsyncs(s, sync, T, nf)
        starts, lengths, counts = stages.sync_pulses(s, sync, T, offs)
        ll, _ = stages.line_locations(s, 0, offs, starts, lengths, counts)
        dll = torch.from_numpy(ll).cuda()
        stages.hsync_refine(s, sync, dll)
        luma = stages.tbc_resample(s, video, dll)
        chroma, _ = stages.chroma_decode(s, raw, dll, n_read)
        torch.cuda.synchronize()
        spp = s.tile_stride
    fields = len(offs)
    assert fields == r.n_fields and cnt[:fields].sum() > 0, (fields, r.n_fields, cnt)
    # concealment must change the planes, or the comparison below proves nothing
    assert not np.array_equal(_u16(luma), r.luma[:fields])
    assert not np.array_equal(_u16(chroma), r.chroma[:fields])

    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream(dev)
    for call in range(2):
        d_luma = luma.clone()
        d_chroma = chroma.clone()
        d_cnt = torch.full((fields,), -1, dtype=torch.int32, device=dev)
        outs = [torch.full((fields * 512,), -7, dtype=torch.int32, device=dev) for _ in range(3)]
        st = lib.cuvhs_dropouts_noalloc(env.data_ptr(), dll.data_ptr(), fields, spp, d_luma.data_ptr(),
                                        d_chroma.data_ptr(), d_cnt.data_ptr(), outs[0].data_ptr(),
                                        outs[1].data_ptr(), outs[2].data_ptr(), ctypes.c_void_p(stream.cuda_stream))
        assert st == 0, call
        torch.cuda.synchronize()
        got = d_cnt.cpu().numpy()
        assert np.array_equal(got, cnt[:fields]), (call, got, cnt[:fields])
        for f in range(fields):
            n = got[f]
            for mine, ref in zip(outs, (lines, sx, ex)):
                assert np.array_equal(mine.cpu().numpy()[f * 512:f * 512 + n], ref[f * 512:f * 512 + n]), (call, f)
        assert np.array_equal(_u16(d_luma), r.luma[:fields]), call
        assert np.array_equal(_u16(d_chroma), r.chroma[:fields]), call


@pytest.mark.gpu
def test_dropouts_noalloc_rejects_oversize_and_bad_arguments():
    import torch

    dev = torch.device("cuda:0")
    t = torch.zeros(16, dtype=torch.int32, device=dev)
    p = t.data_ptr()
    # 503,740-sample slots need 152 partial sums each: 100000 fields exceed the fixed scratch
    assert lib.cuvhs_dropouts_noalloc(p, p, 100000, 503740, p, p, p, p, p, p, None) == 5
    assert lib.cuvhs_dropouts_noalloc(None, p, 1, 503740, p, p, p, p, p, p, None) == 1
    assert lib.cuvhs_dropouts_noalloc(p, p, 0, 503740, p, p, p, p, p, p, None) == 1


# Runs in a child process: decode with the context API, then call the entry
# point on buffers from the CUDA runtime, reset the device (ending this
# process's own context) and call it again on new buffers.
_RESET_CHILD = textwrap.dedent("""
    import ctypes, sys
    import numpy as np
    sys.path.insert(0, sys.argv[1])
    import cuvhs_b200 as cv
    from cuvhs_b200 import lib
    rt = ctypes.CDLL("libcudart.so.12")  # the runtime libcuvhs already loaded

    def ok(e, what):
        assert e == 0, (what, e)

    x = cv.make_workload("dropouts28")
    with cv.Decoder(28.0, debug=True) as d:
        d.decode_capture(x)
        env = d.debug_array("envelope")  # the chunk's first two field slots
        ll = d.debug_array("linelocs")
        cnt = d.debug_array("do_count")
        spans = [d.debug_array(k) for k in ("do_lines", "do_starts", "do_ends")]
        spp = d.tile_stride
    fields = env.size // spp
    plane = np.zeros((fields, 263, 910), np.uint16)

    def dev_copy(a):
        p = ctypes.c_void_p()
        ok(rt.cudaMalloc(ctypes.byref(p), ctypes.c_size_t(a.nbytes)), "cudaMalloc")
        ok(rt.cudaMemcpy(p, a.ctypes.data_as(ctypes.c_void_p), ctypes.c_size_t(a.nbytes), 1), "H2D")
        return p

    def host(p, a):
        ok(rt.cudaMemcpy(a.ctypes.data_as(ctypes.c_void_p), p, ctypes.c_size_t(a.nbytes), 2), "D2H")
        return a

    def call():
        bufs = [dev_copy(a) for a in (env, np.ascontiguousarray(ll[:fields * 525]), plane, plane,
                                      np.zeros(fields, np.int32), *(np.zeros(fields * 512, np.int32),) * 3)]
        st = lib.cuvhs_dropouts_noalloc(bufs[0], bufs[1], fields, spp, bufs[2], bufs[3], bufs[4], bufs[5],
                                        bufs[6], bufs[7], None)
        assert st == 0, st
        ok(rt.cudaDeviceSynchronize(), "sync")
        res = [host(bufs[4], np.zeros(fields, np.int32))] + [host(b, np.zeros(fields * 512, np.int32))
                                                             for b in bufs[5:8]]
        for b in bufs:
            ok(rt.cudaFree(b), "cudaFree")
        return res

    first = call()
    ok(rt.cudaDeviceReset(), "cudaDeviceReset")
    second = call()
    assert np.array_equal(first[0], cnt[:fields]) and cnt[:fields].sum() > 0, (first[0], cnt[:fields])
    for a, b in zip(first, second):
        assert np.array_equal(a, b)
    for f in range(fields):
        n = first[0][f]
        for mine, ref in zip(first[1:], spans):
            assert np.array_equal(mine[f * 512:f * 512 + n], ref[f * 512:f * 512 + n]), f
    print("reset ok", int(cnt[:fields].sum()))
""")


@pytest.mark.gpu
def test_dropouts_noalloc_after_device_reset():
    out = subprocess.run([sys.executable, "-c", _RESET_CHILD, ROOT], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-4000:]
    assert "reset ok" in out.stdout
