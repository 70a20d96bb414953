"""Multi-process checks on CPU (gloo ranks), running the package's own split,
join and reduction code (cuvhs_b200.shard):

* one long capture split into segments, one per rank, each decoding its own
  chunk chain and joining it to the segment before it, gives exactly the
  single-pass chain -- with a stand-in chunk decoder that has the real one's
  properties: chunks start where the previous chunk predicted the next field,
  decode a fixed number of fields, and carry a state (field parity and a
  chunk-relative position) into the next chunk's output;
* the multi-GPU throughput is the units of all ranks over the slowest rank's time."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from cuvhs_b200 import shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


class FakeTape:
    """Fields at irregular positions.  A chunk at `raw` decodes the next nf
    fields starting at or after raw; each field's output depends on the
    incoming state (parity, position of the previous field relative to the
    chunk that found it); every fifth field fixes the parity by itself, as a
    field's own blanking pattern does."""

    def __init__(self, n_fields=240, spf=1000, seed=5, drift=0.0):
        rng = np.random.default_rng(seed)
        self.spf = spf
        i = np.arange(n_fields)
        # per-field jitter; `drift` stretches the spacing slowly (tape speed)
        speed = 1.0 + drift * np.sin(2 * np.pi * i / n_fields)
        self.pos = (300 + np.cumsum(spf * speed) - spf + rng.integers(-40, 41, n_fields)).astype(np.int64)
        self.n_samples = int(self.pos[-1] + spf // 2)
        self.state = (1, -1.0)

    def plan(self, parts):
        return shard.plan_segments(self.n_samples, parts, int(self.pos[0]), float(self.spf), 16, 20)

    def reset(self):
        self.state = (1, -1.0)

    def get_state(self):
        return self.state

    def set_state(self, st):
        self.state = st

    def decode_chunk(self, raw, nf):
        idx = np.flatnonzero(self.pos >= raw)[:nf]
        if idx.size == 0:
            return [], 0, raw
        parity, rel = self.state
        out = []
        for i in idx:
            parity = int(i % 2) if i % 5 == 0 else 1 - parity
            out.append((int(i), parity, rel))
            rel = float(self.pos[i] - raw) / 7.0
        self.state = (parity, rel)
        mean = (self.pos[idx[-1]] - self.pos[idx[0]]) // max(1, idx.size - 1) if idx.size > 1 else self.spf
        return out, int(idx.size), int(self.pos[idx[-1]] + mean - 300)

    def chain(self, start=0, stop=None):
        return shard.run_chain(self.decode_chunk, self.get_state, self.n_samples, self.spf, 16, start,
                               self.n_samples if stop is None else stop)

    def replay(self, raw, state):
        self.set_state(state)
        out, fields, nxt = self.decode_chunk(raw, min(16, (self.n_samples - raw) // self.spf))
        return shard.ChunkRecord(raw, nxt, fields, state, self.get_state(), out)


def _outputs(chunks):
    return [f for c in chunks for f in c.output]


def _split_worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    tape = FakeTape()
    a, b = tape.plan(world)[rank]
    tape.reset()
    mine = tape.chain(a, b)
    kept, first_field, replayed = shard.join_distributed(mine, tape.replay, tape.n_samples, tape.spf)
    outs = [None] * world
    dist.all_gather_object(outs, (first_field, _outputs(kept), replayed))
    value = shard.max_time_throughput(units=10.0 * (rank + 1), seconds=[2.0, 5.0, 3.0][rank])
    if rank == 0:
        q.put((outs, value))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_split_capture_over_ranks_equals_the_single_chain(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_split_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    outs, value = q.get(timeout=120)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    tape = FakeTape()
    tape.reset()
    single = _outputs(tape.chain())
    joined = [f for _, o, _ in outs for f in o]
    assert joined == single
    # each rank's first field index is the number of fields kept before it
    assert [fi for fi, _, _ in outs] == list(np.cumsum([0] + [len(o) for _, o, _ in outs[:-1]]))
    assert all(r <= 2 for _, _, r in outs), [r for _, _, r in outs]
    # the reduction: all ranks' units over the slowest rank's seconds
    assert abs(value - sum(10.0 * (r + 1) for r in range(world)) / 5.0) < 1e-9


@pytest.mark.parametrize("drift", [0.0, 0.02])
def test_single_process_join_replays_until_chain_and_state_meet(drift):
    """Constant speed: every join replays at most two chunks.  With the field
    spacing drifting the predicted boundaries miss and the joins replay
    more, but the joined chain is still exactly the single one."""
    tape = FakeTape(drift=drift)
    tape.reset()
    single = tape.chain()
    segs = []
    for a, b in tape.plan(4):
        tape.reset()
        segs.append(tape.chain(a, b))
    chain, replays = shard.join_all(segs, tape.replay, tape.n_samples, tape.spf)
    assert _outputs(chain) == _outputs(single)
    assert [c.raw_offset for c in chain] == [c.raw_offset for c in single]
    assert len(replays) == 3
    if drift == 0.0:
        assert max(replays) <= 2, replays
