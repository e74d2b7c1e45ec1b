"""The reference's own known-answer tests, restated against this library.

Kestrel ships no golden vectors for the backend path (its tests/ directory is
not distributed, README.md:33-39), only in-module unit tests. Each test here
restates one of them (cited) against the C++ restatements in this repository
-- the oracle (oracle/cpu_synth.cpp) and the host side
(kestrel_b200/csrc/host) -- so they are pinned to the reference's stated
behaviour wherever the reference pins it.
"""
import math

import numpy as np
import pytest

from kestrel_b200 import host as H
from oracle import binding as O

FRAC_ONE = 1 << 32


# ---- src/fixed.rs:116-167 --------------------------------------------------------
# The module's other two tests -- frac_matches_shader_expression (:147-153)
# and f32_phase_would_have_failed (:155-166) -- are restated through both
# backends' render paths in tests/test_analytic.py, where the fraction and the
# 32.32 phase come out of the oracle's and the device's own arithmetic.

def test_fixed_round_trip_unity():  # fixed.rs:119-126
    f = O.lib().ko_fixed_from_f64(1.0)
    assert f >> 32 == 1 and f & 0xFFFFFFFF == 0
    assert np.float32(f & 0xFFFFFFFF) * np.float32(1.0 / 4294967296.0) == 0.0


def test_fixed_accumulates_without_drift():  # fixed.rs:127-145
    ratio = 44100.0 / 48000.0
    step = O.lib().ko_fixed_from_f64(ratio)
    p = 0
    for _ in range(1000):
        p = (p + step) & 0xFFFFFFFFFFFFFFFF
    assert abs(p / FRAC_ONE - ratio * 1000.0) < 1e-6
    n = 1_000_000_000
    total = step * n
    err = total / FRAC_ONE - ratio * n
    assert abs(err) < 1.0


# ---- our own checks of src/fixed.rs:72-113 ------------------------------------------
# The reference has no unit test for Fixed::scale or bend_factor. These assert
# what their doc comments state (src/fixed.rs:72-82: truncating, saturating
# 8.24 scaling; :98-100: the 8.24 factor of a bend, BEND_ONE for a non-finite
# bend) against the oracle's restatement.

def test_fixed_scale_truncates_and_saturates():  # Fixed::scale, fixed.rs:83-90
    s = O.lib().ko_fixed_scale
    assert s(1 << 32, 1 << 24) == 1 << 32
    assert s(3 << 32, (1 << 24) // 2) == (3 << 32) // 2
    assert s((1 << 64) - 1, 0xFFFFFFFF) == (1 << 64) - 1
    v, f = 0x123456789ABCDEF, 0x01234567
    assert s(v, f) == (v * f) >> 24


def test_bend_factor():  # bend_factor, fixed.rs:101-113
    b = O.lib().ko_bend_factor
    assert b(0.0) == 1 << 24
    assert b(12.0) == 2 << 24
    assert b(float("nan")) == 1 << 24
    assert b(1e9) == 0xFFFFFFFF


# ---- src/voice.rs:660-766 (gate table) ------------------------------------------

def _gates():
    return H.GateTable(64, 16)  # cfg() of voice.rs:664-671: block 64, gate tile 16


def test_gate_rows_reflect_state_at_tile_start():  # voice.rs:673-688
    g = _gates()
    assert g.tiles == 4
    g.begin_block()
    assert g.note_on(0, 60, 0) == 1
    g.note_off(0, 60, 40)
    g.end_block()
    s = H.GateTable.slot(0, 60)
    assert [int(g.row(t)[s]) for t in range(4)] == [0, 0, 0, 1]


def test_pedal_defers_note_offs():  # voice.rs:690-710
    g = _gates()
    s = H.GateTable.slot(0, 60)
    g.begin_block()
    g.note_on(0, 60, 0)
    g.set_sustain(0, True, 0)
    g.note_off(0, 60, 16)
    g.end_block()
    assert g.row(3)[s] == 0
    assert g.sounding() == 1
    g.begin_block()
    g.set_sustain(0, False, 16)
    g.end_block()
    assert g.row(1)[s] == 0
    assert g.row(2)[s] == 1
    assert g.sounding() == 0


def test_restrike_under_pedal():  # voice.rs:716-739
    g = _gates()
    s = H.GateTable.slot(0, 60)
    g.begin_block()
    g.set_sustain(0, True, 0)
    g.note_on(0, 60, 0)
    g.note_off(0, 60, 0)
    g.note_on(0, 60, 16)
    g.note_off(0, 60, 16)
    g.note_off(0, 60, 16)
    g.end_block()
    assert g.sounding() == 2
    g.begin_block()
    g.set_sustain(0, False, 0)
    g.end_block()
    assert g.row(3)[s] == 2
    assert g.sounding() == 0


def test_unmatched_note_off_does_not_pre_release():  # voice.rs:740-750
    g = _gates()
    g.begin_block()
    g.note_off(0, 60, 0)
    assert g.note_on(0, 60, 16) == 1
    g.end_block()
    assert g.row(3)[H.GateTable.slot(0, 60)] == 0


def test_retrigger_releases_in_order():  # voice.rs:752-765
    g = _gates()
    g.begin_block()
    a = g.note_on(0, 60, 0)
    b = g.note_on(0, 60, 0)
    g.note_off(0, 60, 16)
    g.end_block()
    assert (a, b) == (1, 2)
    r = g.row(3)[H.GateTable.slot(0, 60)]
    assert a <= r < b


def test_sostenuto_holds_only_what_was_sounding():  # voice.rs:350-378 semantics
    g = _gates()
    s1, s2 = H.GateTable.slot(0, 60), H.GateTable.slot(0, 62)
    g.begin_block()
    g.note_on(0, 60, 0)
    g.set_sostenuto(0, True, 0)
    g.note_on(0, 62, 0)
    g.note_off(0, 60, 16)  # caught by sostenuto: held
    g.note_off(0, 62, 16)  # struck after: damps
    g.end_block()
    assert g.row(3)[s1] == 0 and g.row(3)[s2] == 1
    g.begin_block()
    g.set_sostenuto(0, False, 0)
    g.end_block()
    assert g.row(0)[s1] == 0 and g.row(1)[s1] == 1


# ---- src/voice.rs:132-210 (admission keys) ----------------------------------------

def test_mix48_is_a_bijection_on_a_range():
    vals = [H.mix48(i) for i in range(1 << 14)]
    assert len(set(vals)) == len(vals)
    assert all(v < (1 << 48) for v in vals)


def test_rank_gain_q():
    assert H.rank_gain_q(0.0, 0.0) == 0
    assert H.rank_gain_q(float("nan"), 1.0) == 0
    assert H.rank_gain_q(0.5, 0.5) < H.rank_gain_q(1.0, 1.0) < H.rank_gain_q(4.0, 4.0)
    g = np.float32(1.0) + np.float32(1.0)
    assert H.rank_gain_q(1.0, 1.0) == (int(g.view(np.uint32)) >> 16) & 0x7FFF


# ---- src/bank.rs:981-1035 --------------------------------------------------------

def test_velocity_curve_is_sane():  # bank.rs:985-992
    assert H.velocity_atten_cb(127, 100.0) < 0.01
    cb = H.velocity_atten_cb(64, 100.0)
    assert 100.0 <= cb < 140.0
    assert H.velocity_atten_cb(1, 100.0) >= 800.0


def test_amp_veltrack_scales_the_velocity_curve():  # bank.rs:994-1014
    for vel in [1, 40, 64, 100, 127]:
        assert H.velocity_atten_cb(vel, 0.0) == 0.0
    for vel in [1, 40, 64, 100]:
        half = H.velocity_atten_cb(vel, 50.0)
        assert 0.0 < half < H.velocity_atten_cb(vel, 100.0)
    assert H.velocity_atten_cb(127, 50.0) < 0.01
    assert H.velocity_atten_cb(127, -100.0) >= 960.0
    assert H.velocity_atten_cb(1, -100.0) < 0.01


def test_lowpass_is_unity_at_dc():  # bank.rs:1016-1027
    b0, b1, a1, a2 = H.biquad_lowpass(1000.0, 0.0, 48000.0)
    h = (2.0 * b0 + b1) / (1.0 + a1 + a2)
    assert abs(h - 1.0) < 0.02
    b0, b1, a1, a2 = H.biquad_lowpass(1000.0, 120.0, 48000.0)
    assert (2.0 * b0 + b1) / (1.0 + a1 + a2) < h


def test_timecents_round_trip():  # bank.rs:1029-1034
    assert H.timecents_to_secs(-12000.0) == 0.0
    assert abs(H.timecents_to_secs(0.0) - 1.0) < 1e-6
    assert abs(H.timecents_to_secs(1200.0) - 2.0) < 1e-5


# ---- src/resample.rs:109-171 -------------------------------------------------------

def test_resample_dc_survives():  # resample.rs:113-122
    src = np.full(4000, 10000, np.int16)
    out = H.resample_i16(src, 48000.0 / 44100.0)
    assert out.size == round(4000.0 * 48000.0 / 44100.0)
    assert np.all(np.abs(out[200:-200].astype(np.int32) - 10000) < 60)


def test_resample_sine_keeps_its_frequency():  # resample.rs:124-145
    n = 44100
    t = np.arange(n) / 44100.0
    src = np.trunc(16000.0 * np.sin(2.0 * np.pi * 1000.0 * t)).astype(np.int16)  # `as i16` truncates
    out = H.resample_i16(src, 48000.0 / 44100.0)
    w = out[1000:47000]
    crossings = int(np.sum((w[:-1] < 0) != (w[1:] < 0)))
    freq = crossings / 2.0 / (46000.0 / 48000.0)
    assert abs(freq - 1000.0) < 5.0


def test_resample_upsampling_does_not_clip_headroom():  # resample.rs:148-161
    t = np.arange(2000) / 44100.0
    src = np.trunc(26000.0 * np.sin(2.0 * np.pi * 440.0 * t)).astype(np.int16)
    out = H.resample_i16(src, 2.0)
    assert np.all(np.abs(out.astype(np.int32)) < 32000)


def test_resample_extreme_input_saturates_instead_of_wrapping():  # resample.rs:163-170
    src = np.where(np.arange(500) % 2 == 0, 32767, -32768).astype(np.int16)
    out = H.resample_i16(src, 2.0)
    assert out.dtype == np.int16 and out.size == 1000


def test_resample_identity_ratio_is_a_copy():  # resample.rs:102-107
    src = np.arange(-500, 500, dtype=np.int16)
    assert np.array_equal(H.resample_i16(src, 1.0), src)


# ---- src/config.rs arithmetic --------------------------------------------------------

def test_config_arithmetic():  # config.rs:120-131, 534-552
    from kestrel_b200 import native as N
    L = O.lib()
    c = N.default_config(max_voices=1000, max_steal_percent=25)
    assert L.ko_max_steal(c) == 250
    assert L.ko_pool_slots(c) == 1250
    assert L.ko_steal_span(c) == 4096 - 96
    assert L.ko_admit_take(c, 0, 500) == 500
    assert L.ko_admit_take(c, 900, 500) == 350  # need = min(400, 900, 250) = 250; take = min(500, 1000-650)
    c2 = N.default_config(max_voices=10, max_steal_percent=1)
    assert L.ko_max_steal(c2) == 1  # at least one


# ---- src/cpu.rs:295-302 ------------------------------------------------------------

def test_catmull_rom_endpoints():
    cr = O.lib().ko_catmull_rom
    assert cr(0.1, 0.2, 0.7, 0.9, 0.0) == np.float32(0.2)
    # interpolates a straight line exactly at t = 0.5 within f32 rounding
    assert abs(cr(0.0, 1.0, 2.0, 3.0, 0.5) - 1.5) < 1e-6
