"""The file readers on damaged input: seeded mutations (truncation, byte
and size-field corruption, insertion) of small valid SoundFont 2, SFZ, WAV
and standard MIDI files either load or are refused with an error -- never
a crash, a hang or a runaway allocation. The loaders read files a user
hands in, so they must hold up against anything.
"""
import random
import struct

import pytest

from kestrel_b200 import host as H
from kestrel_b200 import native as N

import test_sf2 as T2
import test_sfz as TZ
import test_smf as TS


def _mutate(rng, b):
    b = bytearray(b)
    k = rng.randint(0, 3)
    if k == 0 and len(b) > 1:
        b = b[:rng.randint(0, len(b) - 1)]
    elif k == 1:
        for _ in range(rng.randint(1, 8)):
            i = rng.randrange(len(b))
            b[i] = rng.randrange(256)
    elif k == 2:
        for _ in range(rng.randint(1, 4)):
            i = rng.randrange(max(len(b) - 4, 1))
            b[i:i + 4] = struct.pack("<I", rng.choice([0, 1, 0xFFFFFFFF, 0x7FFFFFFF, rng.randrange(1 << 32)]))
    else:
        i = rng.randrange(len(b))
        b[i:i] = bytes(rng.randrange(256) for _ in range(rng.randint(1, 16)))
    return bytes(b)


@pytest.mark.parametrize("fmt", ["sf2", "wav", "sfz", "mid"])
def test_damaged_files_load_or_are_refused(tmp_path, fmt):
    rng = random.Random({"sf2": 11, "wav": 12, "sfz": 13, "mid": 14}[fmt])
    cfg = N.default_config(max_voices=4096)
    samples = [dict(data=T2._sine(300, 1), root=60), dict(data=T2._sine(200, 2))]
    inst = [[(48, 50)], [(43, 40 << 8 | 20), (54, 1), (53, 0)], [(53, 1)]]
    sf2, _ = T2.build_sf2(samples, [inst], [dict(bank=0, program=0, zones=[[(48, 3)], [(41, 0)]])])
    wav = TZ.wav_bytes(TZ.tone(500), smpl=(60, 0, (10, 400)))
    sfz = (b"<global> volume=-3\n<group> lokey=c3 hikey=c5\n<region> sample=s.wav key=c4 "
           b"loop_mode=loop_continuous\n<region> sample=s.wav lovel=1 hivel=64 tune=20\n")
    mid = TS.smf([TS.vlq(0) + b"\x90\x3c\x40" + TS.vlq(96) + b"\x80\x3c\x00" + TS.vlq(0) + b"\xff\x2f\x00"])
    loaded = refused = 0
    for it in range(150):
        try:
            if fmt == "sf2":
                (tmp_path / "f.sf2").write_bytes(_mutate(rng, sf2))
                H.Bank(tmp_path / "f.sf2", cfg, H.options(resample_pool=it % 2))
            elif fmt == "wav":
                (tmp_path / "s.wav").write_bytes(_mutate(rng, wav))
                (tmp_path / "i.sfz").write_bytes(sfz)
                H.Bank(tmp_path / "i.sfz", cfg, H.options(resample_pool=it % 2))
            elif fmt == "sfz":
                (tmp_path / "s.wav").write_bytes(wav)
                (tmp_path / "i.sfz").write_bytes(_mutate(rng, sfz))
                H.Bank(tmp_path / "i.sfz", cfg)
            else:
                (tmp_path / "m.mid").write_bytes(_mutate(rng, mid))
                H.read_smf(tmp_path / "m.mid")
            loaded += 1
        except (RuntimeError, OSError, ValueError):
            refused += 1
    assert loaded + refused == 150 and loaded > 0


def test_driver_over_damaged_midi_files(tmp_path):
    """The block driver over damaged MIDI files with programs, controllers,
    tempo changes and bends: each opens and runs, or is refused."""
    rng = random.Random(21)
    cfg, bs, _ = H.config_workload("plain", seed=1)
    bank = H.Bank(bs, cfg)
    tr = b""
    for i in range(40):
        tr += TS.vlq(5) + bytes([0xC0 | (i % 16), i % 128]) + TS.vlq(0) + bytes([0xB0 | (i % 16), 7, 100])
        tr += TS.vlq(0) + b"\xff\x51\x03" + struct.pack(">I", 300000 + i * 1000)[1:]
        tr += TS.vlq(3) + bytes([0x90 | (i % 16), 30 + i, 90]) + TS.vlq(0) + bytes([0xE0 | (i % 16), 0, 64 + i])
        tr += TS.vlq(7) + bytes([0x80 | (i % 16), 30 + i, 0])
    tr += TS.vlq(0) + b"\xff\x2f\x00"
    mid = TS.smf([tr, TS.vlq(0) + b"\xff\x2f\x00"])
    ran = 0
    for _ in range(60):
        (tmp_path / "m.mid").write_bytes(_mutate(rng, mid))
        try:
            drv = H.Driver(cfg, bank, tmp_path / "m.mid")
        except RuntimeError:
            continue
        live = 0
        for _ in range(40):
            blk = drv.prepare(live)
            live = min(cfg.max_voices, live + len(blk.cmds)) // 2
            if not drv.finish(live):
                break
        drv.close()
        ran += 1
    assert ran > 40
