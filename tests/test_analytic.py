"""Closed-form answers the reference states, through both backends.

Kestrel's README (README.md:32-38) says the backend was developed against
tests that are not distributed: phase-accumulator precision tests, envelope
curves checked against analytically computed ones, null tests and
byte-for-byte determinism. The parity tests elsewhere compare the CUDA backend
with the CPU restatement (oracle/cpu_synth.cpp); this file pins BOTH of them to
answers that need neither, each derived from a statement of the reference:

* a single note of the test kit's default soundfont renders to exactly the
  sample (src/testkit.rs:318-348 `simple_sf2`, src/testkit.rs:616-627
  `single_note_midi`, src/cpu.rs:508-512), loaded from an .sf2 file and
  driven from a .mid file;
* the interpolation fraction is `lo as f32 * 2^-32` (src/fixed.rs:205-211);
* the 32.32 phase after N frames is start + N * step, wrapped into the loop
  (src/fixed.rs:185-203, src/cpu.rs:592-601), up to 2^24 frames, where an f32
  accumulator would be off by hundreds of samples (src/fixed.rs:213-224);
* the envelope: the attack adds its rate per frame, the decay and release
  multiply (or subtract) towards the target or the floor, and each stage
  changes on the frame the closed form crosses its threshold
  (src/cpu.rs:512-549);
* the biquad's impulse response is the f64 recursion's within a stated bound
  (src/cpu.rs:564-572);
* a non-looping voice dies on the frame its phase reaches the sample's end
  (src/cpu.rs:499-506);
* nearest interpolation reads the tap under the phase, and Catmull-Rom
  follows its polynomial over the four taps advance_index picks, across the
  loop seam (src/cpu.rs:240-302);
* the steal set is the `need` smallest keys -- note ids under Oldest,
  (level quantised to 16 bits, id) under Quietest -- each victim stopping at
  id % span + 1 and fading out, and compaction keeps the survivors' order
  (src/cpu.rs:213-221, 330-391, 84-117).

Every case runs on the oracle (CPU suite) and on the CUDA backend (marked
gpu). One voice sounds at a time, with gain 1.0 unless stated, so the output
block is the voice's own sample: the mix adds nothing to it on either side.
"""
from __future__ import annotations

import math
import struct

import numpy as np
import pytest

from kestrel_b200 import host as H
from kestrel_b200 import native as N
from oracle.binding import OracleSynth

F32 = np.float32
BACKENDS = [pytest.param("oracle", id="oracle"), pytest.param("cuda", id="cuda", marks=pytest.mark.gpu)]
SLOT = 60  # channel 0, key 60


def make_backend(kind, cfg, pool, params):
    if kind == "oracle":
        return OracleSynth(cfg, pool, params)
    from kestrel_b200.backend import CudaSynth
    return CudaSynth(cfg, pool, params, 1, max(int(pool.size), 1))


def tap(v):
    """CpuSynth::fetch (src/cpu.rs:187-194) of an i16 sample: v / 32767 in
    f32, clamped at -1."""
    return np.maximum(F32(v) * F32(1.0 / 32767.0), F32(-1.0))


def instant_params(**kw):
    """A RegionParams with make_params' instant envelope (src/bank.rs:876-954
    for -12000 timecents): full level on the first frame, sustain 1.0, no
    filter. Keyword arguments override fields."""
    p = np.zeros(1, N.PARAMS_DTYPE)
    p["attack_rate"], p["attack_end"] = 1.0, 1.0
    p["decay_coef"] = F32(10.0) ** F32(-100.0 / 20.0)
    p["decay_target"], p["sustain"] = 1.0, 1.0
    p["release_coef"] = F32(10.0) ** F32(-100.0 / 20.0)
    p["b0"] = 1.0
    for k, v in kw.items():
        p[k] = v
    return p


def one_voice(length, step=1 << 32, phase=0, loop=None, **kw):
    """One SpawnCmd (src/voice.rs:22-57) for sample 0 of the pool."""
    c = np.zeros(1, N.SPAWN_DTYPE)
    c["phase_hi"], c["phase_lo"] = phase >> 32, phase & 0xFFFFFFFF
    c["step_hi"], c["step_lo"] = step >> 32, step & 0xFFFFFFFF
    c["smp_len"] = length
    if loop is not None:
        c["loop_start"], c["loop_end"] = loop
        c["flags"] = N.VF_LOOP
    c["gate_slot"], c["ordinal"] = SLOT, 1
    c["note_id_lo"] = 1
    c["gain_l"], c["gain_r"] = 1.0, 1.0
    for k, v in kw.items():
        c[k] = v
    return c


def render(kind, cfg, pool, params, cmd, blocks, release_at=None):
    """Spawn `cmd` at the start of block 0 and render `blocks` blocks with no
    controllers. With `release_at`, the note's gate row carries its ordinal
    from the first gate tile starting at or after that absolute frame. Returns
    (left channel, right channel, pool fields after the last block)."""
    s = make_backend(kind, cfg, pool, params)
    bf, gf = cfg.block_frames, cfg.gate_frames
    tiles = bf // gf
    chan = np.zeros(tiles * 64, np.uint32)
    outs = []
    try:
        for b in range(blocks):
            gates = np.zeros((tiles, N.GATE_SLOTS), np.uint32)
            if release_at is not None:
                starts = b * bf + np.arange(tiles) * gf
                gates[starts >= release_at, SLOT] = 1
            s.set_gates(gates.reshape(-1))
            s.set_channels(chan, False, False, False)
            s.spawn(cmd if b == 0 else cmd[:0])
            outs.append(s.render().copy())
        fields = s.read_pool()
    finally:
        s.close()
    out = np.concatenate(outs).reshape(-1, 2)
    return out[:, 0], out[:, 1], fields


# ---- src/testkit.rs:318-348: the default soundfont's note is the sample ------------------------

def sine_cycles(freq, rate, cycles, amp):
    """testkit::sine_cycles (src/testkit.rs:19-28)."""
    per = int(round(rate / freq))
    i = np.arange(per * cycles)
    v = np.round(np.sin(i / per * 2.0 * math.pi) * amp * 32767.0)
    return np.clip(v, -32767.0, 32767.0).astype(np.int16)


def vlq(v):
    out = [v & 0x7F]
    v >>= 7
    while v:
        out.append((v & 0x7F) | 0x80)
        v >>= 7
    return bytes(reversed(out))


def single_note_smf(key, vel, off_tick, ppq=960, us_per_qn=500_000):
    """testkit::single_note_midi (src/testkit.rs:616-627): a tempo track and
    one note from tick 0 to `off_tick`."""
    tempo = vlq(0) + b"\xff\x51\x03" + us_per_qn.to_bytes(3, "big") + vlq(0) + b"\xff\x2f\x00"
    note = vlq(0) + bytes([0x90, key, vel]) + vlq(off_tick) + bytes([0x80, key, 0]) + vlq(0) + b"\xff\x2f\x00"
    data = b"MThd" + struct.pack(">IHHh", 6, 1, 2, ppq)
    for t in (tempo, note):
        data += b"MTrk" + struct.pack(">I", len(t)) + t
    return data


@pytest.mark.parametrize("kind", BACKENDS)
def test_default_soundfont_note_renders_exactly_the_sample(kind, tmp_path):
    from test_sf2 import build_sf2

    rate = 48000
    smp = sine_cycles(440.0, rate, 20, 0.5)
    n = smp.size
    # simple_sf2: one looped sine (root 69) and a zone with sampleModes 1 and
    # an instant attack, decay and release at full sustain.
    zone = [(54, 1), (34, -12000), (36, -12000), (37, 0), (38, -12000), (53, 0)]
    sf2, _ = build_sf2([dict(data=smp, rate=rate, root=69, loop=(0, n))], [[zone]],
                       [dict(bank=0, program=0, zones=[[(41, 0)]])])
    (tmp_path / "simple.sf2").write_bytes(sf2)
    # The note is released at tick 961 = 0.5005208 s = frame 24025 (960 ticks
    # per quarter at 120 bpm: 25 frames per tick), inside the gate tile that
    # starts at 24000; the gate row of the next tile (24032) carries it.
    (tmp_path / "note.mid").write_bytes(single_note_smf(69, 127, 961))

    cfg = N.default_config(max_voices=64)
    bank = H.Bank(tmp_path / "simple.sf2", cfg)
    drv = H.Driver(cfg, bank, tmp_path / "note.mid")
    s = make_backend(kind, cfg, bank.pool, bank.params)
    blocks, cmds = [], []
    try:
        for _ in range(7):
            blk = drv.prepare(s.stats().active_voices)
            cmds.append(blk.cmds)
            H.feed(s, blk)
            blocks.append(s.render().copy())
            drv.finish(s.stats().active_voices)
    finally:
        s.close()
        drv.close()
    spawned = np.concatenate(cmds)
    assert spawned.size == 1 and spawned["step_hi"][0] == 1 and spawned["step_lo"][0] == 0
    assert bank.params[spawned["params"][0]]["flags"] == 0  # 13500 cents: no filter (src/bank.rs:931-938)
    out = np.concatenate(blocks).reshape(-1, 2)
    t_rel = 24032
    f = np.arange(out.shape[0])
    x = tap(smp[f % n])
    for ch, g in ((0, spawned["gain_l"][0]), (1, spawned["gain_r"][0])):
        want = np.where(f < t_rel, x * F32(g), F32(0.0)).astype(F32)
        np.testing.assert_array_equal(out[:, ch], want, err_msg=f"channel {ch}")
    assert np.abs(out[:t_rel]).max() > 0.3


# ---- src/fixed.rs:205-211: frac is lo as f32 * 2^-32 ----------------------------------------------

@pytest.mark.parametrize("kind", BACKENDS)
def test_interpolation_fraction_is_the_shader_expression(kind):
    # A voice that never moves (step 0) sits between tap 3 (0.0) and tap 4
    # (1.0): linear interpolation then outputs the fraction itself.
    pool = np.zeros(64, np.int16)
    pool[4] = 32767
    cfg = N.default_config(max_voices=8, block_frames=256, gate_frames=32)
    for lo in (0, 1, 0x4000_0000, 0x8000_0000, 0xFFFF_FFFF):
        left, right, _ = render(kind, cfg, pool, instant_params(), one_voice(56, step=0, phase=(3 << 32) | lo), 1)
        want = F32(lo) * F32(1.0 / 4294967296.0)
        assert np.all(left == want) and np.all(right == want), (hex(lo), left[:4], want)


# ---- src/fixed.rs:185-224, src/cpu.rs:592-601: the 32.32 phase in closed form ---------------------

def closed_phase(start, step, frames, ls, le):
    """Phase after `frames` frames: start + frames * step in exact integers,
    the integer part wrapped into [ls, le) the way the per-frame wrap leaves
    it (no step spans the loop, so the wrap is a modulo)."""
    p = start + frames * step
    hi, lo = p >> 32, p & 0xFFFFFFFF
    if hi >= le:
        hi = ls + (hi - ls) % (le - ls)
    return hi, lo


@pytest.mark.parametrize("kind", BACKENDS)
def test_phase_and_interpolation_follow_the_closed_form(kind):
    # A ramp (every sample distinct, as testkit::ramp, src/testkit.rs:30-39)
    # looped over [1000, 5000), read at a fractional step of about sqrt(2).
    L, ls, le = 5000, 1000, 5000
    i = np.arange(L)
    ramp = np.round((i / (L - 1) * 2.0 - 1.0) * 32767.0).astype(np.int16)
    pool = np.concatenate([ramp, np.zeros(8, np.int16)])
    step = 0x1_6A09_E667
    start = (123 << 32) | 0x9ABC_DEF0
    cfg = N.default_config(max_voices=8)
    blocks = 5
    left, right, fields = render(kind, cfg, pool, instant_params(), one_voice(L, step, start, loop=(ls, le)), blocks)
    frames = blocks * cfg.block_frames
    hi, lo = closed_phase(start, step, frames, ls, le)
    assert fields.shape[1] == 1
    assert (int(fields[N.FIELD["phase_hi"], 0]), int(fields[N.FIELD["phase_lo"], 0])) == (hi, lo)
    # Every frame's output: the reference's linear interpolation between the
    # phase's tap and its loop-aware neighbour, at frac = lo as f32 * 2^-32.
    ph = [closed_phase(start, step, f, ls, le) for f in range(frames)]
    idx = np.array([p[0] for p in ph], np.int64)
    fr = np.array([p[1] for p in ph], np.uint64).astype(F32) * F32(1.0 / 4294967296.0)
    nxt = np.where(idx + 1 < le, idx + 1, ls + (idx + 1 - ls) % (le - ls))
    s0, s1 = tap(ramp[idx]), tap(ramp[nxt])
    want = (s0 + (s1 - s0) * fr).astype(F32)
    np.testing.assert_array_equal(left, want)
    np.testing.assert_array_equal(right, want)


@pytest.mark.parametrize("kind", BACKENDS)
def test_phase_does_not_drift_over_2_24_frames(kind):
    # src/fixed.rs:185-224: the 44.1 -> 48 kHz step (the worst common ratio)
    # accumulated for 2^24 frames, where an f32 accumulator is off by
    # hundreds of samples. The 32.32 phase must be the exact integer sum,
    # wrapped into the loop.
    step = int((44100.0 / 48000.0) * 2**32)  # Fixed::from_f64 truncates
    L, ls, le = 40000, 8000, 40000
    pool = np.zeros(L + 8, np.int16)
    cfg = N.default_config(max_voices=8)
    blocks = (1 << 24) // cfg.block_frames
    start = 17 << 32
    _, _, fields = render(kind, cfg, pool, instant_params(), one_voice(L, step, start, loop=(ls, le)), blocks)
    hi, lo = closed_phase(start, step, blocks * cfg.block_frames, ls, le)
    assert (int(fields[N.FIELD["phase_hi"], 0]), int(fields[N.FIELD["phase_lo"], 0])) == (hi, lo)
    # The f32 accumulator the module replaces (src/fixed.rs:213-224) would be
    # more than 100 samples away from the exact position at this point.
    exact = (1 << 24) * step / 2**32
    acc, step32 = F32(0.0), F32(step / 2**32)
    for _ in range(1 << 10):  # 2^24 f32 adds, 2^14 at a time
        acc = np.cumsum(np.concatenate([[acc], np.full(1 << 14, step32, F32)]), dtype=F32)[-1]
    assert abs(float(acc) - exact) > 100.0


# ---- src/cpu.rs:512-549: envelope curves ----------------------------------------------------------

DC_POOL = np.full(64, 32767, np.int16)  # tap 1.0 everywhere: the output is the level


def transition(values, threshold):
    """First index whose value is <= threshold (the reference's stage test)."""
    hit = np.nonzero(np.asarray(values) <= threshold)[0]
    return int(hit[0]) if hit.size else None


@pytest.mark.parametrize("kind", BACKENDS)
def test_attack_ramp_and_power_of_two_curves_are_exact(kind):
    # Attack rate 2^-10 to attack_end 1.0: level (f + 1) * 2^-10, every sum
    # exact, reaching 1.0 (decay) on frame 1023. Exponential decay by 0.5 to
    # target 0.25: 0.5 on frame 1024, 0.25 <= target on frame 1025, which
    # sets the sustain level 0.75. Released at frame 2048: 0.375, 0.1875, ...
    # until 0.75 * 2^-17 <= 1e-5 kills the voice (0 from then on).
    p = instant_params(attack_rate=2.0**-10, attack_end=1.0, decay_coef=0.5, decay_target=0.25, sustain=0.75,
                       release_coef=0.5)
    cfg = N.default_config(max_voices=8)
    left, right, fields = render(kind, cfg, DC_POOL, p, one_voice(56, loop=(0, 56)), 2, release_at=2048)
    want = np.zeros(2 * cfg.block_frames, F32)
    want[:1024] = (np.arange(1024) + 1) * 2.0**-10
    want[1024], want[1025:2048] = 0.5, 0.75
    k = np.arange(1, 17)
    want[2047 + k] = 0.75 * 0.5**k
    np.testing.assert_array_equal(left, want)
    np.testing.assert_array_equal(right, want)
    assert fields.shape[1] == 0  # dead on frame 2064, compacted away


@pytest.mark.parametrize("kind", BACKENDS)
def test_attack_ramp_at_a_real_rate(kind):
    # A 5 ms attack (240 frames) with a 2.05 ms hold (98.4 frames): rate
    # 1/240, attack_end 1 + 98.4/240 (src/bank.rs:886-887). The level after
    # n frames is the rounded running sum, within n half-ulps of n / 240; the
    # output is min(level, 1) (src/cpu.rs:555), so the hold plays at full
    # level. The stage changes on the first frame whose exact n * rate reaches
    # attack_end (checked to be far from the rounding), which a decay by 0.5
    # to a 0.25 sustain makes visible: 1.0 on that frame, then 0.5, then 0.25.
    rate = F32(1.0) / F32(240.0)
    end = F32(1.0) + F32(98.4) * rate
    p = instant_params(attack_rate=rate, attack_end=end, decay_coef=0.5, decay_target=0.25, sustain=0.25)
    cfg = N.default_config(max_voices=8, block_frames=1024)
    left, _, _ = render(kind, cfg, DC_POOL, p, one_voice(56, loop=(0, 56)), 1)
    n_exact = math.ceil(float(end) / float(rate))
    margin = min(abs(n * float(rate) - float(end)) for n in (n_exact - 1, n_exact))
    assert margin > n_exact * 2.0**-24 * 2
    f = n_exact - 1  # the frame on which the n_exact-th addition lands
    k = np.arange(1, f + 1)
    exact = k * float(rate)
    assert np.all(np.abs(left[:f] - np.minimum(exact, 1.0)) <= k * 2.0**-24 * 2)
    assert left[f] == 1.0 and left[f + 1] == 0.5 and np.all(left[f + 2:] == 0.25)


@pytest.mark.parametrize("kind", BACKENDS)
def test_exponential_decay_and_release_match_the_closed_form(kind):
    # make_params' curves (src/bank.rs:894-904): a 180 ms decay to -6 dB
    # sustain and a 45 ms release to the 1e-5 floor at 48 kHz. Closed form
    # level(n) = start * coef^n; each frame's multiply rounds once, so the
    # f32 level stays within n * 2^-24 relative, and both transitions land on
    # the closed form's crossing frame (its distance from the threshold is
    # checked to exceed that bound).
    dc = F32(10.0) ** F32(-100.0 / (20.0 * 0.180 * 48000))
    rc = F32(10.0) ** F32(-100.0 / (20.0 * 0.045 * 48000))
    sus, floor = F32(10.0 ** (-60 / 200.0)), F32(1e-5)
    p = instant_params(decay_coef=dc, decay_target=sus, sustain=sus, release_coef=rc)
    cfg = N.default_config(max_voices=8)
    rel = 4096  # the gate tile starting at frame 4096
    left, _, fields = render(kind, cfg, DC_POOL, p, one_voice(56, loop=(0, 56)), 2, release_at=rel)

    def crossing(start, coef, thr, limit):
        v = float(start) * float(coef) ** np.arange(1, limit + 1, dtype=np.float64)
        n = transition(v, float(thr)) + 1
        prev, at = float(start) * float(coef) ** (n - 1), float(start) * float(coef) ** n
        assert min(prev - float(thr), float(thr) - at) > n * 2.0**-23 * float(thr), "margin"
        return n, v

    n_d, v_d = crossing(1.0, dc, sus, 2000)
    assert left[0] == 1.0  # instant attack
    k = np.arange(1, n_d)
    assert np.all(np.abs(left[k] - v_d[k - 1]) <= k * 2.0**-24 * v_d[k - 1])
    assert left[n_d] == sus and np.all(left[n_d:rel] == sus)  # decay -> sustain on the crossing frame
    n_r, v_r = crossing(sus, rc, floor, 4096)
    k = np.arange(1, n_r)
    seg = left[rel + k - 1]
    assert np.all(np.abs(seg - v_r[k - 1]) <= k * 2.0**-24 * v_r[k - 1])
    assert left[rel + n_r - 1] == 0.0 and np.all(left[rel + n_r - 1:] == 0.0)  # release -> dead
    assert left[rel + n_r - 2] > floor
    assert fields.shape[1] == 0


@pytest.mark.parametrize("kind", BACKENDS)
def test_linear_curves_subtract_exactly(kind):
    # EnvelopeCurve::Linear (src/cpu.rs:522-527, 538-543) with power-of-two
    # coefficients: every subtraction is exact, so level(n) = start - n * coef
    # on every frame and the transitions land on the exact crossing frames.
    dc, rc = 2.0**-13, 2.0**-12
    sus, floor = F32(10.0 ** (-60 / 200.0)), F32(1e-5)
    p = instant_params(decay_coef=dc, decay_target=sus, sustain=sus, release_coef=rc)
    cfg = N.default_config(max_voices=8, decay_curve=N.CURVE_LINEAR, release_curve=N.CURVE_LINEAR)
    rel = 8192
    left, _, fields = render(kind, cfg, DC_POOL, p, one_voice(56, loop=(0, 56)), 3, release_at=rel)
    n_d = math.ceil((1.0 - float(sus)) / dc)
    k = np.arange(1, n_d)
    np.testing.assert_array_equal(left[k], (1.0 - k * dc).astype(F32))
    assert left[n_d] == sus and np.all(left[n_d:rel] == sus)
    n_r = math.ceil((float(sus) - float(floor)) / rc)
    k = np.arange(1, n_r)
    np.testing.assert_array_equal(left[rel + k - 1], (float(sus) - k * rc).astype(F32))
    assert np.all(left[rel + n_r - 1:] == 0.0)
    assert fields.shape[1] == 0


# ---- src/cpu.rs:564-572: the biquad's impulse response ---------------------------------------------

@pytest.mark.parametrize("kind", BACKENDS)
@pytest.mark.parametrize("fc,q_cb", [(2000.0, 0.0), (8000.0, 30.0), (300.0, 120.0)])
def test_biquad_impulse_response_matches_the_f64_recursion(kind, fc, q_cb):
    # A one-sample impulse of full scale, read at unity step under an instant
    # envelope, through biquad_lowpass(fc, Q) (src/bank.rs:963-979): the
    # output is the filter's impulse response. Against the same coefficients
    # recursed in f64, the f32 transposed-direct-form response stays within
    # 1e-6 absolute over its first 512 frames. The sample is not looped and is
    # 600 frames long, so the voice dies on frame 600 (src/cpu.rs:499-506).
    b0, b1, a1, a2 = (F32(x) for x in H.biquad_lowpass(fc, q_cb, 48000.0))
    p = instant_params(b0=b0, b1=b1, a1=a1, a2=a2, flags=N.RP_FILTER)
    pool = np.zeros(608, np.int16)
    pool[0] = 32767
    cfg = N.default_config(max_voices=8, block_frames=1024)
    left, _, fields = render(kind, cfg, pool, p, one_voice(600), 1)
    h = np.zeros(600)
    z1 = z2 = 0.0
    for i in range(600):
        x = 1.0 if i == 0 else 0.0
        y = float(b0) * x + z1
        z1 = float(b1) * x - float(a1) * y + z2
        z2 = float(b0) * x - float(a2) * y
        h[i] = y
    assert np.max(np.abs(left[:512] - h[:512])) <= 1e-6
    assert abs(left[0] - float(b0)) == 0.0  # y0 = b0 * 1.0
    assert np.all(left[600:] == 0.0)  # idx 600 >= len: dead before its envelope step
    assert fields.shape[1] == 0


@pytest.mark.parametrize("kind", BACKENDS)
def test_end_of_sample_kill_frame(kind):
    # A non-looping 1000-frame sample at a step of 1.25: the voice renders
    # while floor(f * 1.25) < 1000, i.e. frames 0..799, and dies on frame 800
    # (src/cpu.rs:499-506); its last frames interpolate towards the clamped
    # final sample (src/cpu.rs:261-276).
    L = 1000
    pool = np.concatenate([np.full(L, 16384, np.int16), np.zeros(8, np.int16)])
    cfg = N.default_config(max_voices=8, block_frames=1024)
    left, _, fields = render(kind, cfg, pool, instant_params(), one_voice(L, step=(5 << 32) // 4), 1)
    x = tap(16384)
    assert np.all(left[:800] == x) and np.all(left[800:] == 0.0)
    assert fields.shape[1] == 0


# ---- src/cpu.rs:240-302: nearest and Catmull-Rom, loop-aware neighbours ---------------------------

def _ramp_voice(cfg_interp, kind, blocks=2):
    L, ls, le = 3000, 1000, 3000
    ramp = (-30000 + 20 * np.arange(L)).astype(np.int16)  # exactly linear in i16
    pool = np.concatenate([ramp, np.zeros(8, np.int16)])
    step, start = 0x1_3C6E_F372, (5 << 32) | 0x2468_ACE0
    cfg = N.default_config(max_voices=8, interpolation=cfg_interp)
    left, _, fields = render(kind, cfg, pool, instant_params(), one_voice(L, step, start, loop=(ls, le)), blocks)
    frames = blocks * cfg.block_frames
    ph = [closed_phase(start, step, f, ls, le) for f in range(frames)]
    idx = np.array([p[0] for p in ph], np.int64)
    fr = np.array([p[1] for p in ph], np.uint64).astype(F32) * F32(1.0 / 4294967296.0)
    return left, fields, ramp, idx, fr, (ls, le), (start, step, frames)


@pytest.mark.parametrize("kind", BACKENDS)
def test_nearest_reads_the_tap_under_the_phase(kind):
    left, fields, ramp, idx, _, (ls, le), (start, step, frames) = _ramp_voice(N.INTERP_NEAREST, kind)
    np.testing.assert_array_equal(left, tap(ramp[idx]))
    assert (int(fields[N.FIELD["phase_hi"], 0]), int(fields[N.FIELD["phase_lo"], 0])) == \
        closed_phase(start, step, frames, ls, le)


@pytest.mark.parametrize("kind", BACKENDS)
def test_catmull_rom_follows_its_polynomial_across_the_loop_seam(kind):
    # Every frame against catmull_rom (src/cpu.rs:295-302) of the four taps
    # advance_index picks (src/cpu.rs:240-259: index - 1, + 1, + 2, wrapped
    # into [loop_start, loop_end)), evaluated in f64: within 4e-6 (a few f32
    # roundings of values up to 2). On the exactly linear stretch of the ramp
    # the polynomial is the straight line; across the seam it blends the
    # loop's end into its start.
    left, _, ramp, idx, fr, (ls, le), _ = _ramp_voice(N.INTERP_CUBIC, kind)

    def nb(i, off):
        raw = i + off
        return np.where(raw >= le, ls + (raw - ls) % (le - ls), np.maximum(raw, 0))

    t = [tap(ramp[nb(idx, o)]).astype(np.float64) for o in (-1, 0, 1, 2)]
    f = fr.astype(np.float64)
    a = -0.5 * t[0] + 1.5 * t[1] - 1.5 * t[2] + 0.5 * t[3]
    b = t[0] - 2.5 * t[1] + 2.0 * t[2] - 0.5 * t[3]
    c = -0.5 * t[0] + 0.5 * t[2]
    want = ((a * f + b) * f + c) * f + t[1]
    assert np.max(np.abs(left - want)) <= 4e-6
    seam = (idx >= le - 2) | (idx < ls + 1)
    assert seam.sum() > 10  # the seam was crossed
    lin = ~seam
    line = t[1] + (t[2] - t[1]) * f
    assert np.max(np.abs(left[lin] - line[lin])) <= 4e-6


# ---- src/cpu.rs:330-391: the steal set ------------------------------------------------------------

def _steal_run(kind, rule, params, which_params):
    """64 sustained voices (note ids 1..64) fill a 64-voice pool in block 0;
    block 1 spawns 10 more (ids 65..74), so 10 must be stolen (max_steal 16).
    Every voice is full scale at gain 2^-7, so the block's sums are exact."""
    cfg = N.default_config(max_voices=64, max_steal_percent=25, steal_rule=rule, sort_voices=0)
    ids = np.arange(1, 75)
    cmds = np.concatenate([one_voice(56, loop=(0, 56), note_id_lo=i, gain_l=2.0**-7, gain_r=2.0**-7,
                                     params=which_params(i)) for i in ids])
    s = make_backend(kind, cfg, DC_POOL, params)
    tiles = cfg.block_frames // cfg.gate_frames
    outs, live_ids = [], []
    try:
        for b, batch in enumerate((cmds[:64], cmds[64:])):
            s.set_gates(np.zeros(tiles * N.GATE_SLOTS, np.uint32))
            s.set_channels(np.zeros(tiles * 64, np.uint32), False, False, False)
            s.spawn(batch)
            outs.append(s.render().copy().reshape(-1, 2)[:, 0])
            live_ids.append(s.read_pool()[N.FIELD["note_lo"]].astype(np.int64))
        st = s.stats()
    finally:
        s.close()
    return outs, live_ids, st, cfg


@pytest.mark.parametrize("kind", BACKENDS)
def test_oldest_rule_steals_the_lowest_note_ids(kind):
    outs, live, st, cfg = _steal_run(kind, N.STEAL_OLDEST, instant_params(), lambda i: 0)
    assert (st.stolen, st.dropped, st.active_voices) == (10, 0, 64)
    # Victims are ids 1..10: each stops at frame id % span + 1 and fades over
    # steal_fade_frames, then is compacted away; the survivors keep their order.
    np.testing.assert_array_equal(live[1], np.arange(11, 75))
    span = cfg.block_frames - cfg.steal_fade_frames
    assert all(i % span + 1 == i + 1 for i in range(1, 11))
    assert outs[1][0] == F32(74 * 2.0**-7)           # every voice at full level on frame 0
    assert np.all(outs[1][10 + 96:] == F32(64 * 2.0**-7))  # the last victim (id 10) is silent from frame 106
    # id 1 stops at frame 2 (stop_rel 2): d = f + 1 - 2 is 0 on frame 1 and 1 on frame 2
    assert outs[1][1] == outs[1][0] and outs[1][2] < outs[1][1]


@pytest.mark.parametrize("kind", BACKENDS)
def test_quietest_rule_steals_the_lowest_levels_then_ids(kind):
    # Four sustain levels; a voice's steal key is its level quantised to 16
    # bits above its note id (src/cpu.rs:213-221), so the victims are the 10
    # smallest (level, id) pairs.
    sus = np.array([0.75, 0.25, 1.0, 0.5], np.float32)
    params = np.concatenate([instant_params(decay_target=s, sustain=s) for s in sus])
    pick = lambda i: (i * 7) % 4
    outs, live, st, _ = _steal_run(kind, N.STEAL_QUIETEST, params, pick)
    assert (st.stolen, st.dropped, st.active_voices) == (10, 0, 64)
    q = {i: int(np.float32(sus[pick(i)]) * np.float32(65535.0)) for i in range(1, 65)}
    victims = sorted(range(1, 65), key=lambda i: (q[i], i))[:10]
    assert all(sus[pick(i)] == np.float32(0.25) for i in victims)
    want = [i for i in range(1, 65) if i not in victims] + list(range(65, 75))
    np.testing.assert_array_equal(live[1], want)
