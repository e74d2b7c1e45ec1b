"""The host driver (C++ restatement of src/driver.rs) on CPU.

Checks the invariants the reference states for Driver::next_block: admission
takes Config::admit_take of the queued candidates (src/config.rs:120-131,
src/driver.rs:557-585), note ids are handed out in candidate order and never
reused (src/driver.rs:805-823), gate rows only ever count up, the controller
flags are false when a control sat at unity (src/voice.rs:600-616), and the
whole stream is a pure function of its seed.
"""
import numpy as np
import pytest

from kestrel_b200 import host as H
from kestrel_b200 import native as N
from oracle.binding import OracleSynth, lib as olib


def _ids(cmds):
    return (cmds["note_id_hi"].astype(np.uint64) << np.uint64(32)) | cmds["note_id_lo"]


def _small(workload, **over):
    cfg, bs, ms = H.config_workload(workload, seed=3)
    for k, v in over.items():
        if hasattr(cfg, k):
            setattr(cfg, k, v)
        elif hasattr(ms, k):
            setattr(ms, k, v)
        else:
            setattr(bs, k, v)
    return cfg, bs, ms


def test_driver_is_deterministic():
    cfg, bs, ms = _small("black", notes=20000, seconds=2.0)
    bank = H.Bank(bs, cfg)
    a, b = H.Driver(cfg, bank, ms), H.Driver(cfg, bank, ms)
    live = 0
    for _ in range(12):
        x, y = a.prepare(live), b.prepare(live)
        assert np.array_equal(x.cmds, y.cmds) and np.array_equal(x.gates, y.gates)
        assert np.array_equal(x.chan, y.chan) and (x.bend, x.gain) == (y.bend, y.gain)
        live = min(cfg.max_voices, live + len(x.cmds))
        a.finish(live)
        b.finish(live)


def test_admission_and_ids():
    cfg, bs, ms = _small("plain", max_voices=300, notes=40000, seconds=3.0)
    bank = H.Bank(bs, cfg)
    drv = H.Driver(cfg, bank, ms)
    orc = OracleSynth(cfg, bank.pool, bank.params)
    last_id = 0
    prev_gates = None
    saturated = 0
    for _ in range(30):
        live = orc.stats().active_voices
        blk = drv.prepare(live)
        assert blk.take == olib().ko_admit_take(cfg, live, blk.want)
        assert len(blk.cmds) == blk.take
        saturated += blk.take < blk.want
        ids = _ids(blk.cmds)
        if ids.size:
            assert len(np.unique(ids)) == ids.size
            assert ids.min() > last_id  # fresh ids every block
            last_id = int(ids.max())
        g = blk.gates.reshape(-1, 2048)
        assert np.all(np.diff(g.astype(np.int64), axis=0) >= 0)  # tiles only count up
        if prev_gates is not None:
            assert np.all(g[0] >= prev_gates[-1])
        prev_gates = g
        assert not blk.bend and not blk.gain  # no controllers in this workload
        H.feed(orc, blk)
        orc.render()
        drv.finish(orc.stats().active_voices)
    assert saturated > 0  # the small pool made admission choose


def test_black_workload_controllers_and_presets():
    cfg, bs, ms = _small("black", notes=50000, seconds=3.0)
    bank = H.Bank(bs, cfg)
    assert bank.presets == 128 and bank.regions == 128 * 128
    drv = H.Driver(cfg, bank, ms)
    blk = None
    regions = set()
    live = 0
    for _ in range(20):
        blk = drv.prepare(live)
        regions.update(int(r) for r in blk.cmds["region"])
        live = min(cfg.max_voices, live + len(blk.cmds))
        drv.finish(live)
    assert blk.bend and blk.gain  # pitch bend and CC7/CC11 curves every 10 ms
    ch = blk.chan.reshape(-1, 16, 4)
    assert len(np.unique(ch[:, :, 0])) > 1
    assert len({r // 128 for r in regions}) > 4  # program changes spread the presets


def test_bank_matches_the_configured_generators():
    cfg, bs, ms = H.config_workload("plain")
    bank = H.Bank(bs, cfg)
    assert bank.pool_rate == 48000 and bank.max_sample_len == 35666  # 32768 @ 44.1k resampled
    p = bank.params[0]
    assert p["attack_rate"] == pytest.approx(1.0 / (0.005 * 48000), rel=1e-3)   # 5 ms
    assert p["sustain"] == pytest.approx(10 ** (-60 / 200), rel=1e-4)             # -6 dB
    assert p["decay_coef"] == pytest.approx(10 ** (-5 / (0.2 * 48000)), rel=1e-6)  # 200 ms to -100 dB
    assert p["release_coef"] == pytest.approx(10 ** (-5 / (0.3 * 48000)), rel=1e-6)
    assert p["flags"] == 1  # 8 kHz lowpass on
