"""One long capture decoded as independent segments (one per GPU, or one after
another on one GPU) and joined into exactly the single-pass decode.

The reference decodes a capture as a chain of chunks (Pipeline::run,
src/pipeline/pipeline.cu:2626-2713): each chunk starts where the previous one
predicted the next field (its next_raw_offset) and inherits the state the
previous chunk left -- the last field's parity (pipeline.cu:2575), the
line-location history (pipeline.h:92-97) and the chroma track and phase cycle
(chroma_decode.h:9-15).  A chunk's output is a function of (capture, start
offset, field count, incoming state) alone, so a segment that starts its own
chain partway into the capture produces exactly the single-pass chunks as soon
as its chain and state meet the single-pass ones.

A split therefore runs in two steps:

1. every segment runs its own chunk chain from a start `halo` samples before
   its split point (the first segment from 0, fresh state), recording each
   chunk's start, next offset and incoming and outgoing state;
2. the joins, in capture order: from the end of the joined prefix (its next
   offset and state), chunks are re-decoded one at a time ("replayed") until
   the prefix reaches a chunk of the next segment that starts at the same
   offset with the same incoming state; that chunk and every later one of the
   segment are then the single-pass chunks and are kept as they are.

No collective is needed on the data path: segments exchange a few bytes of
chain position and state, and each GPU's fields go to host memory at their
field index.  A join normally replays one or two chunks (the first segment
chunk starts at a different offset than the single-pass chain, and the
line-location history is kept relative to the chunk it was found in).
"""
from dataclasses import dataclass
from typing import Callable, List, Optional

import numpy as np


@dataclass
class ChunkRecord:
    """One chunk of a chain: where it started, where the next one starts, the
    state it met and the state it left, and its output (any object)."""
    raw_offset: int
    next_offset: int
    fields: int
    state_in: tuple
    state_out: tuple
    output: object = None


def plan_segments(n_samples: int, parts: int, first_field: int, field_period: float, batch_fields: int,
                  samples_per_line: int) -> List[tuple]:
    """(decode start, stop) of each segment.  The single-pass chain starts
    chunk k about ten lines before field k * batch_fields (every full chunk
    holds batch_fields fields), so segment r starts there for the k that puts
    it nearest to r / parts of the capture, predicting field positions from
    the first field's location and the nominal field period: when the
    prediction holds (constant tape speed), the segment's chain meets the
    single-pass chain after one chunk.  A segment stops where the next one
    starts; the first starts at 0."""
    parts = max(1, int(parts))
    step = batch_fields * field_period
    starts = [0]
    for r in range(1, parts):
        k = max(1, int(round((n_samples * r / parts - first_field) / step)))
        g = int(round(first_field + k * step)) - 10 * samples_per_line
        starts.append(min(max(g, starts[-1] + 1), n_samples))
    stops = starts[1:] + [n_samples]
    return list(zip(starts, stops))


def field_period(sample_rate_hz: float, pal: bool = False) -> float:
    """Nominal samples per field: the capture rate over the field rate."""
    return sample_rate_hz / (50.0 if pal else 60000.0 / 1001.0)


def run_chain(decode_chunk: Callable, get_state: Callable, n_samples: int, samples_per_field: int,
              batch_fields: int, start: int, stop: int, after_first: Optional[Callable] = None) -> List[ChunkRecord]:
    """The chunk loop from `start` with the decoder's current state, over the
    chunks that start before `stop` (Pipeline::run's loop).
    decode_chunk(raw_offset, num_fields) -> (output, fields, next_offset);
    after_first(), if given, runs once after the first chunk (to amend the
    decoder's state)."""
    chunks = []
    raw = int(start)
    while raw < stop:
        remaining = (n_samples - raw) // samples_per_field
        if remaining <= 0:
            break
        nf = min(batch_fields, remaining)
        st_in = get_state()
        out, fields, nxt = decode_chunk(raw, nf)
        chunks.append(ChunkRecord(raw, int(nxt), int(fields), st_in, get_state(), out))
        if fields == 0:
            break
        if after_first is not None and len(chunks) == 1:
            after_first()
        raw = int(nxt)
    return chunks


def join(prefix: List[ChunkRecord], tail: List[ChunkRecord], replay: Callable, n_samples: int,
         samples_per_field: int, initial=None):
    """The single-pass chain over prefix + tail.  `prefix` is exact (it starts
    the capture, or was joined already); tail's chunks are kept from the first
    one whose start offset and incoming state equal the chain's, and chunks
    before that are replayed: replay(raw_offset, state) -> ChunkRecord, decoded
    with that incoming state.  `initial` = (offset, state) when prefix is
    empty.  Returns (chunks, replayed count)."""
    out = list(prefix)
    if out:
        offset, state = out[-1].next_offset, out[-1].state_out
        if out[-1].fields == 0:
            return out, 0
    else:
        offset, state = initial
    where = {c.raw_offset: k for k, c in enumerate(tail)}
    replayed = 0
    while True:
        k = where.get(offset)
        if k is not None and tail[k].state_in == state:
            out.extend(tail[k:])
            return out, replayed
        if (n_samples - offset) // samples_per_field <= 0:
            return out, replayed
        c = replay(offset, state)
        replayed += 1
        out.append(c)
        if c.fields == 0:
            return out, replayed
        offset, state = c.next_offset, c.state_out


def join_all(segments: List[List[ChunkRecord]], replay: Callable, n_samples: int, samples_per_field: int):
    """Join every segment in capture order; returns (chunks, replays per join)."""
    chain = list(segments[0])
    counts = []
    for seg in segments[1:]:
        chain, r = join(chain, seg, replay, n_samples, samples_per_field)
        counts.append(r)
    return chain, counts


# ------------------------------------------------------------ decoder binding

def _gpu_chain_fns(dec, x):
    """decode_chunk / get_state / set_state callables over a Decoder and a capture."""
    def decode_chunk(raw, nf):
        res, nxt = dec.decode_chunk(x[raw:], raw, nf)
        return res, res.n_fields, nxt

    def get_state():
        # The chroma phase cycle position is kept mod 8 (chroma_decode.cu:1000)
        # but indexes a table that repeats every four fields (:672), so two
        # chains whose positions differ by four decode every later field alike:
        # the state compares (and is replayed) by its position mod 4.
        t = dec.get_state().as_tuple()
        return t[:-1] + (t[-1] % 4,)

    def set_state(t):
        from ._lib import State
        st = State(*t)
        dec.set_state(st)
    return decode_chunk, get_state, set_state


def decode_segment(dec, x, start, stop, batch_fields, chroma_threshold=None):
    """One segment's chain on `dec` from a fresh state.  The chroma decode's
    track-error threshold is set once, from the capture's first field
    (chroma_decode.cu:684-743), and carried unchanged; a segment that starts
    mid-capture measures its own on its first chunk, so with
    `chroma_threshold` (the capture's) it takes the capture's value after
    that chunk, which lets its chain's state meet the single-pass one."""
    decode_chunk, get_state, set_state = _gpu_chain_fns(dec, x)
    dec.reset()
    after_first = None
    if chroma_threshold is not None:
        def after_first():
            st = dec.get_state()
            st.chroma_threshold = chroma_threshold
            dec.set_state(st)
    return run_chain(decode_chunk, get_state, x.size, dec.samples_per_field, batch_fields, start, stop,
                     after_first)


def replayer(dec, x):
    """replay(raw_offset, state) on `dec`: one chunk with the given incoming state."""
    decode_chunk, get_state, set_state = _gpu_chain_fns(dec, x)

    def replay(raw, state):
        set_state(state)
        nf = min(dec.batch_fields, (x.size - raw) // dec.samples_per_field)
        out, fields, nxt = decode_chunk(raw, nf)
        return ChunkRecord(raw, int(nxt), int(fields), state, get_state(), out)
    return replay


def merge_results(dec, chunks: List[ChunkRecord]):
    """The chunks' outputs as one DecodeResult with the capture's .tbc.json."""
    import ctypes
    from ._lib import DecodeResult, FieldInfo, Output, lib
    results = [c.output for c in chunks if c.output is not None and c.output.n_fields > 0]
    shape = dec.field_shape
    luma = np.concatenate([r.luma for r in results]) if results else np.zeros((0,) + shape, np.uint16)
    chroma = np.concatenate([r.chroma for r in results]) if results else np.zeros((0,) + shape, np.uint16)
    file_loc = np.concatenate([r.file_loc for r in results]) if results else np.zeros(0, np.uint64)
    first = np.concatenate([r.is_first_field for r in results]) if results else np.zeros(0, np.int32)
    phase = np.concatenate([r.field_phase_id for r in results]) if results else np.zeros(0, np.int32)
    dropouts = [d for r in results for d in r.dropouts]
    n = len(file_loc)
    fi = (FieldInfo * max(n, 1))()
    dl, ds, de = [], [], []
    off = 0
    for i in range(n):
        fi[i].file_loc = int(file_loc[i])
        fi[i].is_first_field = int(first[i])
        fi[i].field_phase_id = int(phase[i])
        fi[i].dropout_count = len(dropouts[i][0])
        fi[i].dropout_offset = off
        off += len(dropouts[i][0])
        dl.append(dropouts[i][0])
        ds.append(dropouts[i][1])
        de.append(dropouts[i][2])
    cat = (lambda a: np.ascontiguousarray(np.concatenate(a), np.int32) if a else np.zeros(1, np.int32))
    dl, ds, de = cat(dl), cat(ds), cat(de)
    out = Output()
    out.fields = ctypes.addressof(fi)
    out.fields_out = n
    out.dropout_line, out.dropout_startx, out.dropout_endx = dl.ctypes.data, ds.ctypes.data, de.ctypes.data
    out.dropouts_out = off
    out.max_fields = max(n, 1)
    out.max_dropouts = max(off, 1)
    jl = lib.cuvhs_json(dec._h, ctypes.byref(out), None, 0)
    jb = ctypes.create_string_buffer(int(jl) + 1)
    lib.cuvhs_json(dec._h, ctypes.byref(out), jb, jl + 1)
    return DecodeResult(luma=luma, chroma=chroma, file_loc=file_loc, is_first_field=first, field_phase_id=phase,
                        dropouts=dropouts, json=jb.value.decode())


def capture_start(dec, x):
    """The capture's first chunk, decoded on `dec` (state reset before and
    after): (first field location, chroma track-error threshold)."""
    dec.reset()
    nf = max(1, min(dec.batch_fields, x.size // dec.samples_per_field))
    res, _ = dec.decode_chunk(x, 0, nf)
    thr = dec.get_state().chroma_threshold
    dec.reset()
    return (int(res.file_loc[0]) if res.n_fields else 0), thr


def plan_for(dec, x, parts, first_field):
    pal = dec.lines_per_frame != 525
    spl = dec.samples_per_field // (313 if pal else 263)
    fs = spl * (15625.0 if pal else 15734.264)
    return plan_segments(x.size, parts, first_field, field_period(fs, pal), dec.batch_fields, spl)


def decode_split(x, sample_rate_mhz, parts=2, batch_fields=0, device=0, **decoder_kw):
    """Decode capture `x` as `parts` segments one after another on one GPU and
    join them: the same result as one Decoder.decode_capture with the same
    batch_fields.  Returns (result, replayed chunks per join, chunks per segment)."""
    from ._lib import Decoder
    with Decoder(sample_rate_mhz, device=device, batch_fields=batch_fields, **decoder_kw) as dec:
        spf = dec.samples_per_field
        first_field, thr = capture_start(dec, x)
        plan = plan_for(dec, x, parts, first_field)
        segs = [decode_segment(dec, x, a, b, dec.batch_fields, None if k == 0 else thr)
                for k, (a, b) in enumerate(plan)]
        chain, replays = join_all(segs, replayer(dec, x), x.size, spf)
        return merge_results(dec, chain), replays, [len(s) for s in segs]


def join_distributed(records: List[ChunkRecord], replay: Callable, n_samples: int, samples_per_field: int,
                     group=None):
    """The joins of a split whose segment k was decoded on rank k
    (torch.distributed; gloo or nccl).  Each rank joins its own segment to the
    end of the segment before it, replaying on its own device; no field data
    moves.  Ranks first assume that every earlier segment keeps its own chain
    end (the normal case: a join replays a chunk or two and keeps the rest),
    then exchange the ends their joins really produced and redo any join whose
    assumed start was wrong, until no end changes (at most world rounds).
    Every rank takes the same collective steps.  Returns (this rank's chunks,
    index of its first field in the capture, chunks replayed here)."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)

    def end_of(chunks, fallback):
        return (chunks[-1].next_offset, chunks[-1].state_out, chunks[-1].fields) if chunks else fallback

    def gather(obj):
        allv = [None] * world
        dist.all_gather_object(allv, obj, group=group)
        return allv

    # ends as decoded: the first guess of every predecessor's joined end
    ends = gather(end_of(records, None))
    kept, replayed, used = list(records), 0, None
    for _ in range(world):
        if rank == 0:
            kept, replayed, used = list(records), 0, None
        else:
            # the last segment before this one whose chain reaches a known end
            prev = next((ends[k] for k in range(rank - 1, -1, -1) if ends[k] is not None), None)
            want = None if prev is None else (prev[0], prev[1])
            if want != used:
                if want is None or prev[2] == 0:
                    kept, replayed = [], 0  # the capture ended before this segment
                else:
                    kept, replayed = join([], records, replay, n_samples, samples_per_field, initial=want)
                used = want
        new_ends = gather(end_of(kept, None) if rank > 0 else end_of(records, None))
        changed = any(new_ends[k] != ends[k] for k in range(world))
        ends = new_ends
        if not changed:
            break
    counts = gather(sum(c.fields for c in kept))
    return kept, int(sum(counts[:rank])), replayed


def max_time_throughput(units: float, seconds: float, group=None, device=None) -> float:
    """Whole-job throughput of ranks that each processed `units` in their own
    `seconds`: the units of all ranks over the slowest rank's time (what a
    multi-GPU step takes).  Without an initialised process group: units / seconds."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(units) / float(seconds)
    if device is None:
        device = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    u = torch.tensor([float(units)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    dist.all_reduce(u, group=group)
    return float(u[0]) / float(t[0])

