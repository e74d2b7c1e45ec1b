"""The output stage: limiters, clamp_block and the WAV writer.

The limiter tests are the reference's own (src/limiter.rs:473-705), restated
against the C++ restatement: the follower's quiet and loud behaviour, the
brickwall's ceiling guarantee with violent transients, its fast recovery,
true-peak detection catching inter-sample overshoot, the sustained stage
steadying the gain without reintroducing pumping, and determinism. The WAV
tests check the header (src/wav.rs:63-79), pcm16 rounding, and the size
fields patched at finish.
"""
import struct

import numpy as np
import pytest

from kestrel_b200 import host as H


def _brick(ceiling_db=0.0, release=60.0, sustain=400.0, true_peak=True):
    return H.Limiter(H.LIMITER_BRICKWALL, 48000, ceiling_db, 2.0, release, sustain, true_peak)


def test_quiet_signal_passes_through_scaled():
    lim = H.Limiter(H.LIMITER_OMNI, 48000)
    buf = np.full(48000 * 6, 0.1, np.float32)
    lim.process(buf)
    assert np.all(np.abs(buf[-1000:] - 0.125) < 0.005)


def test_loud_signal_is_pulled_down():
    lim = H.Limiter(H.LIMITER_OMNI, 48000)
    buf = np.full(48000 * 2, 8.0, np.float32)
    lim.process(buf)
    assert np.all(np.abs(buf[-100:]) <= 1.0)


def test_omni_is_deterministic_across_identical_input():
    def make():
        lim = H.Limiter(H.LIMITER_OMNI, 48000)
        buf = (np.sin(np.arange(8192, dtype=np.float32) * np.float32(0.01)) * np.float32(3.0)).astype(np.float32)
        return lim.process(buf).copy()
    assert make().tobytes() == make().tobytes()


@pytest.mark.parametrize("ceiling", [1.0, 0.5])
def test_brickwall_never_exceeds_the_ceiling(ceiling):
    bw = _brick(ceiling_db=20 * np.log10(ceiling))
    t = np.arange(48000 * 2) // 2
    buf = (np.sin(t * 0.05) * 40.0 + np.where(t % 977 == 0, 300.0, 0.0)).astype(np.float32)
    bw.process(buf)  # limiter, then clamp_block
    assert float(np.max(np.abs(buf))) <= ceiling + 1e-4
    assert bw.clipped == 0  # the clamp never had to move a sample


def _burst():
    t = np.arange(48000 * 2) // 2
    return np.where((t >= 4800) & (t < 4848), 60.0, 0.5).astype(np.float32)


def _level(buf, sec):
    a = int(sec * 48000) * 2
    return float(np.max(np.abs(buf[a:a + 4800])))


def test_brickwall_recovers_quickly_after_a_transient():
    buf = _burst()
    _brick().process(buf)
    assert abs(_level(buf, 0.02) - 0.5) < 0.02
    assert abs(_level(buf, 0.35) - 0.5) < 0.02


def test_true_peak_detection_catches_intersample_overshoot():
    t = (np.arange(48000 * 2) // 2).astype(np.float64)
    src = (np.sin(t * np.pi / 2 + np.pi / 4) * np.sqrt(2.0)).astype(np.float32)
    tp, sp = src.copy(), src.copy()
    # clamp_block pins both at 1.0 in the end: compare the limiters before it
    a, b = _brick(sustain=400.0, true_peak=True), _brick(sustain=400.0, true_peak=False)
    a.process(tp)
    b.process(sp)
    assert float(np.max(np.abs(tp))) < float(np.max(np.abs(sp))) - 0.05


def test_brickwall_is_deterministic():
    def run():
        buf = (np.sin(np.arange(8192, dtype=np.float32) * np.float32(0.017)) * np.float32(9.0)).astype(np.float32)
        return _brick().process(buf).copy()
    assert run().tobytes() == run().tobytes()


def _wobble(sustain_ms):
    t = (np.arange(48000 * 2 * 2) // 2) / 48000.0
    src = ((np.sin(t * 1000.0 * 2 * np.pi) + np.sin(t * 1050.0 * 2 * np.pi)) * 20.0).astype(np.float32)
    buf = src.copy()
    bw = _brick(release=5.0, sustain=sustain_ms)
    d = bw.latency * 2
    bw.process(buf)
    start = src.size // 2
    k = np.arange(start, src.size - d)
    k = k[np.abs(src[k]) > 4.0]
    assert k.size > 10000
    g = buf[k + d].astype(np.float64) / src[k].astype(np.float64)
    return g.std() / g.mean()


def test_the_sustained_stage_holds_the_gain_steady_on_a_loud_passage():
    assert _wobble(400.0) < _wobble(0.0) * 0.85


def test_the_sustained_stage_does_not_reintroduce_pumping():
    buf = _burst()
    _brick(sustain=400.0).process(buf)
    assert abs(_level(buf, 0.35) - 0.5) < 0.02


def test_limiter_config_ranges_are_validated():
    for bad in (dict(ceiling_db=1.0), dict(lookahead_ms=0.01), dict(release_ms=0.0), dict(sustain_ms=20000.0)):
        kw = dict(ceiling_db=0.0, lookahead_ms=2.0, release_ms=60.0, sustain_ms=0.0)
        kw.update(bad)
        with pytest.raises(ValueError):
            H.Limiter(H.LIMITER_BRICKWALL, 48000, **kw)


def test_clamp_block_counts_what_it_moves():
    x = np.array([0.5, 1.5, -2.0, 1.0, -1.0], np.float32)
    n = H.lib().kh_clamp_block(x.ctypes.data, x.size)
    assert n == 2 and x.tolist() == [0.5, 1.0, -1.0, 1.0, -1.0]


@pytest.mark.parametrize("fmt", [H.WAV_PCM16, H.WAV_FLOAT32])
def test_wav_header_and_payload(tmp_path, fmt):
    p = tmp_path / "out.wav"
    w = H.WavWriter(p, 48000, 2, fmt)
    blocks = [np.array([0.5, -0.5, 1.5, -1.5, 0.0, 2.0 ** -16], np.float32), np.array([0.25, -0.25], np.float32)]
    for b in blocks:
        w.write(b)
    n = w.finish()
    raw = p.read_bytes()
    riff, size, wave, fmt_id, fmt_len, tag, ch, sr, byte_rate, align, bits, data_id, data_len = struct.unpack(
        "<4sI4s4sIHHIIHH4sI", raw[:44])
    width = 2 if fmt == H.WAV_PCM16 else 4
    assert (riff, wave, fmt_id, data_id) == (b"RIFF", b"WAVE", b"fmt ", b"data")
    assert (fmt_len, ch, sr, align, bits) == (16, 2, 48000, 2 * width, 8 * width)
    assert tag == (1 if fmt == H.WAV_PCM16 else 3)
    assert byte_rate == 48000 * 2 * width
    assert data_len == n == 8 * width and size == 36 + n and len(raw) == 44 + n
    x = np.concatenate(blocks)
    if fmt == H.WAV_PCM16:
        got = np.frombuffer(raw[44:], "<i2")
        want = np.round(np.clip(x, -1, 1) * np.float32(32767)).astype(np.int16)
        assert got.tolist() == want.tolist()
        assert got[2] == 32767 and got[3] == -32767
    else:
        assert np.frombuffer(raw[44:], "<f4").tobytes() == x.tobytes()
