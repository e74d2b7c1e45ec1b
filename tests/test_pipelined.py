"""The pipelined render loop: Driver::next_block split into collect / admit /
advance / more (src/driver.rs:434-642) and the backend's render split into
begin / end, so the host prepares block n + 1 while the device renders
block n. Both splits must leave every call and argument the serial loop
makes unchanged: the block inputs, the continuation answers and the WAV
file are the same, byte for byte.
"""
import ctypes as C
import struct

import numpy as np
import pytest

from kestrel_b200 import host as H
from kestrel_b200 import native as N
from kestrel_b200.render import render_file

gpu = pytest.mark.gpu


def _spec(workload, **over):
    cfg, bs, ms = H.config_workload(workload, seed=7)
    for k, v in over.items():
        setattr(ms if hasattr(ms, k) else cfg, k, v)
    return cfg, bs, ms


def _vlq(v):
    out = [v & 0x7F]
    v >>= 7
    while v:
        out.append((v & 0x7F) | 0x80)
        v >>= 7
    return bytes(reversed(out))


def _sound_cc_file(path, notes=160):
    """A one-track file whose notes ride on changing sound controllers
    (CC71 / CC74), so blocks carry params variants."""
    t = b""
    for i in range(notes):
        ch = i % 3
        t += _vlq(0) + bytes([0xB0 | ch, 74, (i * 37) % 128])
        t += _vlq(0) + bytes([0xB0 | ch, 71, (i * 11) % 128])
        t += _vlq(0) + bytes([0x90 | ch, 30 + (i * 7) % 60, 90])
        t += _vlq(24) + bytes([0x80 | ch, 30 + (i * 7) % 60, 0])
    t += _vlq(0) + b"\xff\x2f\x00"
    path.write_bytes(b"MThd" + struct.pack(">IHHh", 6, 0, 1, 96) + b"MTrk" + struct.pack(">I", len(t)) + t)
    return path


def _same_inputs(x, y):
    assert np.array_equal(x.gates, y.gates) and np.array_equal(x.chan, y.chan)
    assert (x.bend, x.gain, x.variant) == (y.bend, y.gain, y.variant)
    assert np.array_equal(x.cmds, y.cmds)
    assert len(x.variants) == len(y.variants)
    for (i, a), (j, b) in zip(x.variants, y.variants):
        assert i == j and np.array_equal(a, b)
    assert (x.live, x.want, x.take) == (y.live, y.want, y.take)


def _decay(live, blk, cap):
    # a stand-in backend: admitted voices join, a quarter of the pool ends
    return min(cap, live + len(blk.cmds)) * 3 // 4


@pytest.mark.parametrize("workload,over", [
    ("plain", dict(notes=3000, seconds=1.0, max_voices=400)),
    ("black", dict(notes=20000, seconds=1.0, cluster_lo=50, cluster_hi=400, program_period_s=0.2)),
    ("smf", {}),
])
def test_split_driver_equals_prepare_finish(tmp_path, workload, over):
    if workload == "smf":
        cfg, bs, _ = _spec("black")
        ms = _sound_cc_file(tmp_path / "cc.mid")
    else:
        cfg, bs, ms = _spec(workload, **over)
    bank = H.Bank(bs, cfg)
    a, b = H.Driver(cfg, bank, ms), H.Driver(cfg, bank, ms)
    # serial: prepare(n), render, finish(n)
    serial, live = [], 0
    while True:
        blk = a.prepare(live)
        live = _decay(live, blk, cfg.max_voices)
        more = a.finish(live)
        serial.append((blk, more))
        if not more:
            break
    assert len(serial) > 8
    # pipelined: collect(n + 1) comes before more(n), and so does admit(n + 1)
    # whenever its admission cannot depend on the live count
    piped, live, early = [], 0, 0
    b.collect()
    blk = b.admit(live)
    b.advance()
    while True:
        b.collect()
        nxt = b.admit(0) if b.admit_ready() else None
        live = _decay(live, blk, cfg.max_voices)
        more = b.more_after(live)
        piped.append((blk, more))
        if not more:
            break
        if nxt is not None:
            nxt.live = live       # the caller's live count, which admission did not need
            blk, early = nxt, early + 1
        else:
            blk = b.admit(live)
        b.advance()
    assert len(piped) == len(serial) and early > 0
    for (x, mx), (y, my) in zip(serial, piped):
        _same_inputs(x, y)
        assert mx == my
    if workload == "smf":
        assert any(x.variants for x, _ in serial)


class _AsyncOracle:
    """The CPU reference backend behind the asynchronous calls, so the
    pipelined loop's ordering is checked without a GPU. Like the CUDA
    backend, it stages a block's inputs and applies them (the spawn
    included) only when that block begins."""

    spawn_deferred = True

    def __init__(self, cfg, bank):
        from oracle.binding import OracleSynth
        self.o = OracleSynth(cfg, bank.pool, bank.params)
        self.block_frames = cfg.block_frames
        self.held = None
        self.staged = None

    def feed_raw(self, kb, variants):
        vs = []
        for idx, addr, n in variants:
            vs.append((idx, np.frombuffer((C.c_char * (n * N.PARAMS_DTYPE.itemsize)).from_address(addr),
                                          dtype=N.PARAMS_DTYPE).copy()))
        gates = np.ctypeslib.as_array(kb.gates, shape=(kb.n_gates,)).copy()
        chan = np.ctypeslib.as_array(kb.chan, shape=(kb.n_chan,)).copy()
        if kb.n_cmds:
            raw = (C.c_char * (kb.n_cmds * N.SPAWN_DTYPE.itemsize)).from_address(kb.cmds)
            cmds = np.frombuffer(raw, dtype=N.SPAWN_DTYPE).copy()
        else:
            cmds = np.zeros(0, N.SPAWN_DTYPE)
        self.staged = (vs, gates, chan, bool(kb.bend), bool(kb.gain), bool(kb.variant), cmds)

    def render_begin(self):
        assert self.held is None and self.staged is not None
        vs, gates, chan, bend, gain, variant, cmds = self.staged
        self.staged = None
        for idx, data in vs:
            self.o.set_params_variant(idx, data)
        self.o.set_gates(gates)
        self.o.set_channels(chan, bend, gain, variant)
        self.o.spawn(cmds)
        self.held = self.o.render()

    def render_end(self, out):
        out[:] = self.held
        self.held = None
        return out

    def stats(self):
        # the previous block's stats until render_end, as kc_stats reports
        return self.o.stats() if self.held is None else self._last

    def close(self):
        self.o.close()


def _tracking_async(cfg, bank):
    s = _AsyncOracle(cfg, bank)
    s._last = s.o.stats()
    orig_begin = s.render_begin

    def begin():
        s._last = s.o.stats()
        orig_begin()
    s.render_begin = begin
    return s


def _oracle(cfg, bank):
    from oracle.binding import OracleSynth
    return OracleSynth(cfg, bank.pool, bank.params)


@pytest.mark.parametrize("source", ["synthetic", "smf"])
def test_pipelined_loop_equals_serial_on_cpu(tmp_path, source):
    cfg, bs, ms = _spec("black", notes=6000, seconds=0.6, cluster_lo=50, cluster_hi=300, program_period_s=0.2,
                        max_voices=4096, max_steal_percent=5)
    if source == "smf":
        ms = _sound_cc_file(tmp_path / "cc.mid", notes=60)
    a = render_file(tmp_path / "serial.wav", cfg, bs, ms, backend=_oracle)
    b = render_file(tmp_path / "piped.wav", cfg, bs, ms, backend=_tracking_async)
    assert not a.pipelined and b.pipelined and b.phases is not None
    assert (a.blocks, a.peak_voices, a.clipped) == (b.blocks, b.peak_voices, b.clipped)
    # blocks admitted while the one before rendered, and (with clusters over
    # the steal budget) blocks that waited for it
    assert b.phases["early_blocks"] > 0
    if source == "synthetic":
        assert b.phases["early_blocks"] < b.blocks - 1
    assert (tmp_path / "serial.wav").read_bytes() == (tmp_path / "piped.wav").read_bytes()


@gpu
@pytest.mark.parametrize("workload,over,seconds", [
    ("plain", {}, 2.0),
    ("black", dict(notes=200000, seconds=2.0, cluster_lo=200, cluster_hi=4000), 0.0),
    ("smf", {}, 0.0),
])
def test_cuda_pipelined_render_equals_serial(tmp_path, workload, over, seconds):
    if workload == "smf":
        cfg, bs, _ = _spec("black")
        ms = _sound_cc_file(tmp_path / "cc.mid")
    else:
        cfg, bs, ms = _spec(workload, **over)
    a = render_file(tmp_path / "serial.wav", cfg, bs, ms, pipelined=False, max_seconds=seconds)
    b = render_file(tmp_path / "piped.wav", cfg, bs, ms, pipelined=True, max_seconds=seconds)
    assert b.pipelined and a.blocks == b.blocks and a.peak_voices == b.peak_voices
    assert (tmp_path / "serial.wav").read_bytes() == (tmp_path / "piped.wav").read_bytes()


@gpu
def test_render_begin_end_contract():
    from kestrel_b200.backend import CudaSynth
    cfg, bs, ms = _spec("plain", notes=20000, seconds=1.0)
    bank = H.Bank(bs, cfg)
    drv = H.Driver(cfg, bank, ms)
    a = CudaSynth(cfg, bank.pool, bank.params, bank.regions, bank.max_sample_len)
    b = CudaSynth(cfg, bank.pool, bank.params, bank.regions, bank.max_sample_len)
    # a: the serial render; its blocks' inputs are recorded
    blocks, ref = [], []
    for _ in range(10):
        blk = drv.prepare(a.stats().active_voices)
        H.feed(a, blk)
        ref.append(a.render().copy())
        drv.finish(a.stats().active_voices)
        blocks.append(blk)
    out = np.empty(cfg.block_frames * 2, np.float32)
    with pytest.raises(N.KestrelError):
        b.render_end(out)           # nothing in flight
    # b: block i + 1's inputs are staged while block i is in flight
    H.feed(b, blocks[0])
    b.render_begin()
    assert b.pending
    with pytest.raises(N.KestrelError):
        b.render_begin()            # one block at a time
    with pytest.raises(N.KestrelError):
        b.clone()
    got = []
    for i in range(10):
        if i + 1 < 10:
            b.set_gates(np.zeros_like(blocks[i + 1].gates))
            H.feed(b, blocks[i + 1])
        got.append(b.render_end().copy())
        assert not b.pending
        if i + 1 < 10:
            b.render_begin()
    for x, y in zip(ref, got):
        assert np.array_equal(x, y)
    assert a.stats() == b.stats()
    a.close()
    b.close()


@pytest.mark.parametrize("workload,over", [
    ("steal", dict(notes=2_000_000, seconds=1.2, max_voices=50000)),
    ("black", dict(notes=400_000, seconds=1.5, program_period_s=0.3)),
    ("smf", {}),
])
def test_read_ahead_leaves_the_blocks_unchanged(tmp_path, workload, over):
    """The event source on its own thread (and, with no program draws, the
    onset windows on another) yields the driver the same blocks."""
    if workload == "smf":
        cfg, bs, _ = _spec("black")
        ms = _sound_cc_file(tmp_path / "cc.mid")
    else:
        cfg, bs, ms = _spec(workload, **over)
    bank = H.Bank(bs, cfg, H.options(read_ahead=0))
    a = H.Driver(cfg, bank, ms)
    bank.opt.read_ahead = 1
    b = H.Driver(cfg, bank, ms)
    live = 0
    for _ in range(16):
        x, y = a.prepare(live), b.prepare(live)
        _same_inputs(x, y)
        live = _decay(live, x, cfg.max_voices)
        assert a.finish(live) == b.finish(live)
    a.close()
    b.close()


def test_block_csv_rows_match_between_the_loops(tmp_path):
    """`--block-csv`: the same rows from the serial and the pipelined loop;
    admission never takes more than it queued, the drop count accumulates
    want - take, and the energies bound each other."""
    import csv as pycsv
    cfg, bs, ms = _spec("black", notes=30000, seconds=0.5, cluster_lo=500, cluster_hi=3000, max_voices=2048,
                        admit_rule=N.ADMIT_LOUDEST)
    render_file(tmp_path / "a.wav", cfg, bs, ms, backend=_oracle, block_csv=tmp_path / "a.csv")
    render_file(tmp_path / "b.wav", cfg, bs, ms, backend=_tracking_async, block_csv=tmp_path / "b.csv")
    assert (tmp_path / "a.csv").read_text() == (tmp_path / "b.csv").read_text()
    rows = list(pycsv.DictReader(open(tmp_path / "a.csv")))
    assert [int(r["block"]) for r in rows] == list(range(1, len(rows) + 1))
    dropped = 0
    for r in rows:
        want, take = int(r["want"]), int(r["take"])
        assert take <= want and int(r["take_e"]) <= int(r["want_e"])
        dropped += want - take
        assert int(r["dropped"]) == dropped
        assert 0.0 <= float(r["rms"]) <= float(r["peak"]) <= 1.0
    assert dropped > 0 and any(int(r["stolen"]) > 0 for r in rows)
