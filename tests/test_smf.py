"""Standard MIDI files: the streaming parser and track merger (src/midi.rs)
and the driver reading a file.

Known answers follow the reference's parser (src/midi.rs:126-374): running
status, note-on with velocity 0 as a note-off, meta and SysEx skipped, the
end-of-track meta, ties between tracks broken by track index, SMPTE
division, chunk walking that stops at zero padding. End to end, the
synthetic workloads written out as files (the way MidiWriter writes them,
src/midi.rs:439-506) drive the driver to exactly the block inputs the
in-memory stream does.
"""
import struct

import numpy as np
import pytest

from kestrel_b200 import host as H
from kestrel_b200 import native as N


def vlq(v):
    out = [v & 0x7F]
    v >>= 7
    while v:
        out.append((v & 0x7F) | 0x80)
        v >>= 7
    return bytes(reversed(out))


def smf(tracks, division=96, fmt=1, pad=b""):
    data = b"MThd" + struct.pack(">IHHh", 6, fmt, len(tracks), division)
    for t in tracks:
        data += b"MTrk" + struct.pack(">I", len(t)) + t
    return data + pad


def events(path):
    return H.read_smf(path)[1]


def test_running_status_velocity_zero_and_meta(tmp_path):
    t = (vlq(0) + bytes([0x90, 60, 100]) + vlq(10) + bytes([62, 90])      # running status: another note-on
         + vlq(0) + bytes([0xFF, 0x01, 3]) + b"abc"                         # text meta clears running status
         + vlq(5) + bytes([0x90, 60, 0])                                    # velocity 0: a note-off
         + vlq(1) + bytes([0xF0, 2, 0x7E, 0xF7])                            # SysEx, skipped
         + vlq(2) + bytes([0xB3, 7, 99]) + vlq(0) + bytes([0xC3, 5])
         + vlq(0) + bytes([0xE3, 0x00, 0x40])                               # bend centre
         + vlq(0) + bytes([0xE3, 0x7F, 0x7F])                               # bend max
         + vlq(3) + bytes([0xFF, 0x51, 3, 0x07, 0xA1, 0x20])               # tempo 500000
         + vlq(0) + bytes([0xFF, 0x2F, 0]) + bytes([0x90, 1, 1]))          # after end of track: ignored
    p = tmp_path / "a.mid"
    p.write_bytes(smf([t]))
    ev = events(p)
    kinds = [(e[0], e[1]) for e in ev]
    assert kinds == [(0, "note_on"), (10, "note_on"), (10, "other"), (15, "note_off"), (16, "other"), (18, "cc"),
                     (18, "program"), (18, "pitch_bend"), (18, "pitch_bend"), (21, "tempo"), (21, "other")]
    assert ev[1][3:5] == (62, 90) and ev[3][3] == 60
    assert ev[5][2:5] == (3, 7, 99) and ev[6][3] == 5
    assert ev[7][5] == 0 and ev[8][5] == 8191 and ev[9][6] == 500000


def test_data_before_any_status_ends_the_track(tmp_path):
    p = tmp_path / "b.mid"
    p.write_bytes(smf([vlq(0) + bytes([60, 100]) + vlq(0) + bytes([0x90, 61, 1])]))
    assert events(p) == []


def test_tracks_merge_by_tick_then_track_index(tmp_path):
    t0 = vlq(5) + bytes([0x90, 1, 1]) + vlq(0) + bytes([0x90, 2, 1]) + vlq(0) + bytes([0xFF, 0x2F, 0])
    t1 = vlq(0) + bytes([0x91, 3, 1]) + vlq(5) + bytes([0x91, 4, 1]) + vlq(0) + bytes([0xFF, 0x2F, 0])
    p = tmp_path / "c.mid"
    p.write_bytes(smf([t0, t1]))
    info, ev = H.read_smf(p)
    assert info[:3] == (1, 2, 96)
    notes = [(e[0], e[3]) for e in ev if e[1] == "note_on"]
    assert notes == [(0, 3), (5, 1), (5, 2), (5, 4)]


def test_smpte_division_and_zero_padding(tmp_path):
    t = vlq(0) + bytes([0x90, 60, 1]) + vlq(0) + bytes([0xFF, 0x2F, 0])
    div = -((25 << 8)) | 40  # 25 fps x 40 ticks per frame
    p = tmp_path / "d.mid"
    p.write_bytes(smf([t], division=div, fmt=0, pad=bytes(64)))
    info, ev = H.read_smf(p)
    assert info == (0, 1, 0, 25, 40)
    assert [e[1] for e in ev] == ["note_on", "other"]


def test_not_a_midi_file(tmp_path):
    p = tmp_path / "e.mid"
    p.write_bytes(b"RIFF" + bytes(20))
    with pytest.raises(RuntimeError, match="not a standard MIDI file"):
        H.read_smf(p)


def test_written_file_header_is_midiwriter_format(tmp_path):
    spec = H.midi_spec(notes=50, seconds=1.0, seed=3)
    p = tmp_path / "w.mid"
    H.write_synthetic_midi(spec, p)
    raw = p.read_bytes()
    assert raw[:14] == b"MThd" + struct.pack(">IHHH", 6, 1, 1, 9600)
    assert raw[14:18] == b"MTrk" and raw.endswith(bytes([0, 0xFF, 0x2F, 0]))
    info, ev = H.read_smf(p)
    ons = sum(1 for e in ev if e[1] == "note_on")
    assert 0 < ons <= 50 and ons == sum(1 for e in ev if e[1] == "note_off")  # every note ends
    assert all(a[0] <= b[0] for a, b in zip(ev, ev[1:]))


@pytest.mark.parametrize("workload,blocks", [("plain", 60), ("black", 30)])
def test_driver_over_the_written_file_matches_the_stream(tmp_path, workload, blocks):
    cfg, bs, ms = H.config_workload(workload, seed=9)
    if workload == "black":
        ms.notes, ms.seconds = 200_000, 6.0  # same shape, a file of a few MB
    p = tmp_path / f"{workload}.mid"
    H.write_synthetic_midi(ms, p)
    bank = H.Bank(bs, cfg)
    d1, d2 = H.Driver(cfg, bank, ms), H.Driver(cfg, bank, p)
    live = 0
    for b in range(blocks):
        x, y = d1.prepare(live), d2.prepare(live)
        for f in ("gates", "chan", "cmds"):
            assert np.array_equal(getattr(x, f), getattr(y, f)), (b, f)
        assert (x.bend, x.gain, x.variant) == (y.bend, y.gain, y.variant)
        assert [i for i, _ in x.variants] == [i for i, _ in y.variants]
        live = min(live + len(x.cmds), cfg.max_voices) * 3 // 4
        assert d1.finish(live) == d2.finish(live)
    assert live > 0
