"""SFZ instruments (src/sfz.rs) and the WAV reader they load samples with
(src/wav.rs:160-356).

The reference's own unit tests (note names, values with spaces,
src/sfz.rs:683-698) are restated as known answers; the rest builds SFZ
files and WAVs here and checks what the loader made of them against the
rules of src/sfz.rs written out by hand: inheritance from <global>,
<master> and <group>, the `key` alias collapsing at the level that wrote
it, positional <control> default paths, #include, every opcode the loader
reads, the WAV formats and the smpl chunk, stereo files as two hard-panned
regions, and each refusal. A bank loaded from SFZ renders through the CUDA
backend like the CPU reference.
"""
import ctypes as C
import struct

import numpy as np
import pytest

from kestrel_b200 import host as H
from kestrel_b200 import native as N

gpu = pytest.mark.gpu


def wav_bytes(frames, rate=48000, bits=16, fmt="pcm", channels=1, smpl=None, extensible=False):
    """frames: float array in [-1, 1], shape (n,) or (n, channels)."""
    x = np.asarray(frames, np.float64).reshape(len(frames), channels)
    if fmt == "float":
        data = x.astype("<f4" if bits == 32 else "<f8").tobytes()
        tag = 3
    elif bits == 8:
        data = np.clip(np.round(x * 127 + 128), 0, 255).astype(np.uint8).tobytes()
        tag = 1
    elif bits == 24:
        v = np.clip(np.round(x * 8388607), -8388608, 8388607).astype("<i4")
        data = b"".join(int(q).to_bytes(4, "little", signed=True)[:3] for q in v.reshape(-1))
        tag = 1
    else:
        scale, dt = {16: (32767, "<i2"), 32: (2147483647, "<i4")}[bits]
        data = np.clip(np.round(x * scale), -scale - 1, scale).astype(dt).tobytes()
        tag = 1
    block = channels * bits // 8
    if extensible:
        fmt_chunk = struct.pack("<HHIIHHHHI", 0xFFFE, channels, rate, rate * block, block, bits, 22, bits, 0) + \
            struct.pack("<H", tag) + b"\x00\x00\x00\x00\x10\x00\x80\x00\x00\xaa\x00\x38\x9b\x71"
    else:
        fmt_chunk = struct.pack("<HHIIHH", tag, channels, rate, rate * block, block, bits)
    body = b"WAVE" + b"fmt " + struct.pack("<I", len(fmt_chunk)) + fmt_chunk
    if smpl:
        # src/wav.rs:283-296 reads the note and its pitch fraction at bytes
        # 20 and 24 of the chunk (where the format's own layout keeps the
        # SMPTE fields; its unity note sits at 12): written where it reads them
        root, frac, loop = smpl
        s = struct.pack("<9I", 0, 0, 0, 0, 0, root, frac, 1 if loop else 0, 0)
        if loop:
            s += struct.pack("<6I", 0, 0, loop[0], loop[1], 0, 0)
        body += b"smpl" + struct.pack("<I", len(s)) + s
    body += b"LIST" + struct.pack("<I", 5) + b"INFOx\x00"  # an odd chunk the reader skips with its pad byte
    body += b"data" + struct.pack("<I", len(data)) + data + (b"\x00" if len(data) % 2 else b"")
    return b"RIFF" + struct.pack("<I", len(body)) + body


def f32_to_i16(x):
    """WavData::channel_i16: clamp to [-1, 1], * 32767, round half away from zero."""
    v = np.clip(np.asarray(x, np.float32), np.float32(-1), np.float32(1)) * np.float32(32767)
    return (np.sign(v) * np.floor(np.abs(v) + np.float32(0.5))).astype(np.int16)


def tone(n, seed=0):
    rng = np.random.default_rng(seed)
    return np.clip(np.sin(np.arange(n) * 0.05) * 0.6 + rng.normal(0, 0.05, n), -1, 1)


def _cfg():
    return N.default_config(max_voices=4096)


def load(path, resample=0):
    return H.Bank(path, _cfg(), H.options(resample_pool=resample))


def test_note_names_and_values_with_spaces():
    """src/sfz.rs:687-698, plus flats, case, and non-notes."""
    lib = H.lib()
    got = {}
    for name in ["c4", "a4", "c#4", "c-1", "eb3", "B3", "bb3", "G9", "x4", "c", "c#", "4"]:
        v = C.c_int32()
        got[name] = v.value if lib.kh_sfz_note_name(name.encode(), C.byref(v)) == 0 else None
    assert got == {"c4": 60, "a4": 69, "c#4": 61, "c-1": 0, "eb3": 51, "B3": 59, "bb3": 58, "G9": 127, "x4": None,
                   "c": None, "c#": None, "4": None}
    s = "My Sample Name.wav lokey=30"
    assert s[:lib.kh_sfz_value_end(s.encode())].strip() == "My Sample Name.wav"
    assert lib.kh_sfz_value_end(b"60") == 2
    assert lib.kh_sfz_value_end(b"a.wav <region>") == 5


@pytest.mark.parametrize("bits,fmt,ext", [(8, "pcm", False), (16, "pcm", False), (24, "pcm", False),
                                          (32, "pcm", False), (32, "float", False), (64, "float", False),
                                          (16, "pcm", True)])
def test_wav_formats_decode_into_the_pool(tmp_path, bits, fmt, ext):
    x = tone(1001, seed=bits)
    (tmp_path / "s.wav").write_bytes(wav_bytes(x, bits=bits, fmt=fmt, extensible=ext))
    (tmp_path / "i.sfz").write_text("<region> sample=s.wav\n")
    b = load(tmp_path / "i.sfz")
    raw = (tmp_path / "s.wav").read_bytes()
    data = raw[raw.index(b"data") + 8:]
    if fmt == "float":
        dec = np.frombuffer(data[:1001 * bits // 8], "<f4" if bits == 32 else "<f8").astype(np.float32)
    elif bits == 8:
        dec = (np.frombuffer(data[:1001], np.uint8).astype(np.float32) - np.float32(128)) / np.float32(128)
    elif bits == 24:
        q = np.frombuffer(data[:3003], np.uint8).reshape(-1, 3).astype(np.int32)
        v = (q[:, 0] << 8 | q[:, 1] << 16 | q[:, 2] << 24) >> 8
        dec = v.astype(np.float32) / np.float32(8388608)
    else:
        dt, sc = {16: ("<i2", 32768), 32: ("<i4", 2147483648)}[bits]
        dec = np.frombuffer(data[:1001 * bits // 8], dt).astype(np.float32) / np.float32(sc)
    si = b.sample_info(0)
    assert si["len"] == 1001 and si["rate"] == 48000 and si["root_key"] == 60
    assert np.array_equal(b.pool[:1001], f32_to_i16(dec))
    # no smpl loop: the loop spans the whole sample, and a region without
    # loop_mode follows it (src/sfz.rs:466-467, 590-599)
    assert (si["loop_start"], si["loop_end"]) == (0, 1000) and b.region_info(0)["loop_mode"] == 1


def test_smpl_chunk_root_tuning_and_loop(tmp_path):
    (tmp_path / "s.wav").write_bytes(wav_bytes(tone(2000), smpl=(64, 0x80000000, (100, 900))))
    (tmp_path / "i.sfz").write_text("<region> sample=s.wav\n<region> sample=s.wav pitch_keycenter=70 "
                                    "loop_mode=no_loop\n")
    b = load(tmp_path / "i.sfz")
    si = b.sample_info(0)
    assert (si["root_key"], si["correction_cents"], si["loop_start"], si["loop_end"]) == (64, 50.0, 100, 900)
    assert b.n_samples == 1                       # read once, used twice
    r0, r1 = b.region_info(0), b.region_info(1)
    assert r0["root_key_override"] == 64 and r0["loop_mode"] == 1   # the WAV's loop turns looping on
    assert r1["root_key_override"] == 70 and r1["loop_mode"] == 0
    # a chunk with the unity note at byte 12 and zero SMPTE fields reads as
    # note 0, as the reference reads it
    c = struct.pack("<9I", 0, 0, 0, 64, 0, 0, 0, 0, 0)
    raw = (tmp_path / "s.wav").read_bytes()
    a = raw.index(b"smpl")
    n = struct.unpack("<I", raw[a + 4:a + 8])[0]
    body = raw[12:a] + b"smpl" + struct.pack("<I", len(c)) + c + raw[a + 8 + n:]
    (tmp_path / "t.wav").write_bytes(b"RIFF" + struct.pack("<I", len(body) + 4) + b"WAVE" + body)
    (tmp_path / "t.sfz").write_text("<region> sample=t.wav\n")
    assert load(tmp_path / "t.sfz").sample_info(0)["root_key"] == 0


def test_inheritance_aliases_and_control_paths(tmp_path):
    for d in ("a", "b"):
        (tmp_path / d).mkdir()
    (tmp_path / "a" / "x.wav").write_bytes(wav_bytes(tone(500, 1)))
    (tmp_path / "b" / "x.wav").write_bytes(wav_bytes(tone(700, 2)))
    (tmp_path / "b" / "Mixed Case.WAV").write_bytes(wav_bytes(tone(300, 3)))
    (tmp_path / "inc.sfz").write_text("<region> sample=x.wav lovel=10 hivel=20 // an included region\n")
    (tmp_path / "i.sfz").write_text("""
// header comment
<global> volume=-6 pan=20 amplfo_depth=3
<control> default_path=a\\
<group> lokey=0 hikey=127 tune=12.6
<region> sample=x.wav key=c4
<region> sample=x.wav key=60 pitch_keycenter=62 lokey=55
<master> transpose=-3 <group> hikey=90
<region> sample=x.wav
<master>
<region> sample=x.wav
<control> default_path=b/
#include "inc.sfz"
<region> sample=mixed case.wav end=-1
<region> sample=mixed case.wav loopmode=loop_sustain
<region> lokey=1
<global>
<region> sample=missing.wav
<effect> type=reverb <weird> x=1
""")
    b = load(tmp_path / "i.sfz")
    regs = [b.region_info(i) for i in range(b.regions)]
    assert len(regs) == 6
    # key=c4 expands at the region, over the group's lokey/hikey
    assert (regs[0]["key_lo"], regs[0]["key_hi"], regs[0]["root_key_override"]) == (60, 60, 60)
    # an explicit sibling at the same level wins over the alias
    assert (regs[1]["key_lo"], regs[1]["key_hi"], regs[1]["root_key_override"]) == (55, 60, 62)
    for r in regs[:4]:
        assert r["attenuation_cb"] == 60.0 and r["pan"] == pytest.approx(0.2)
    assert [r["fine_tune"] for r in regs[:2]] == [13, 13]
    # a <master> replaces the one before it and clears the group
    assert (regs[2]["coarse_tune"], regs[2]["key_hi"], regs[2]["fine_tune"]) == (-3, 90, 0)
    assert (regs[3]["coarse_tune"], regs[3]["key_hi"]) == (0, 127)
    # <control> default_path governs the regions after it: a/ then b/
    lens = [b.sample_info(r["sample"])["len"] for r in regs]
    assert lens[:4] == [500] * 4 and lens[4] == 700
    assert (regs[4]["vel_lo"], regs[4]["vel_hi"]) == (10, 20)
    # case-insensitive file names; end=-1 disables; loopmode alias
    assert lens[5] == 300 and regs[5]["loop_mode"] == 2
    rep = "\n".join(b.report)
    assert "missing.wav" in rep and "<weird>" in rep and "amplfo_* (not implemented)" in rep
    assert b.presets == 1 and b.preset_info(0) == (0, 0, list(range(6)))


def test_every_opcode_the_loader_reads(tmp_path):
    (tmp_path / "s.wav").write_bytes(wav_bytes(tone(4410), rate=44100, smpl=(60, 0, (441, 4000))))
    (tmp_path / "st.wav").write_bytes(wav_bytes(np.stack([tone(900, 5), tone(900, 6)], 1), channels=2))
    (tmp_path / "i.sfz").write_text("""
<region> sample=s.wav lovel=5 hivel=300 transpose=200 pitch_keytrack=50.4 amp_veltrack=-150
  ampeg_delay=0.1 ampeg_attack=0.02 ampeg_hold=0.3 ampeg_decay=1.5 ampeg_sustain=50 ampeg_release=0.7
  cutoff=1000 resonance=3 fil_veltrack=12000 offset=-5 end=4000 loop_start=500 loop_end=3900
  group=2 off_by=2 loop_mode=loop_continuous
<region> sample=s.wav cutoff=1000 fil_type=hpf_2p group=2 off_by=3 offset=7 loop_mode=one_shot
<region> sample=st.wav pan=-30
""")
    b = H.Bank(tmp_path / "i.sfz", _cfg(), H.options(resample_pool=1))
    r0, r1 = b.region_info(0), b.region_info(1)
    assert (r0["vel_lo"], r0["vel_hi"], r0["coarse_tune"], r0["scale_tuning"]) == (5, 127, 127, 50)
    assert r0["scale_tuning"] == 50
    assert (r0["delay"], r0["attack"], r0["hold"], r0["decay"], r0["sustain"], r0["release"]) == \
        pytest.approx((0.1, 0.02, 0.3, 1.5, 0.5, 0.7))
    assert r0["filter_fc_cents"] == pytest.approx(1200 * np.log2(1000 / 8.176), rel=1e-6)
    assert r0["filter_q_cb"] == 30.0 and r0["exclusive_class"] == 2 and r0["addr_start"] == 0
    # absolute positions in source frames, against the sample's points taken back to the source rate
    si = b.sample_info(r0["sample"])
    ratio = np.float32(48000 / 44100)
    src = lambda v: int(np.floor(np.float32(v) / ratio + np.float32(0.5)))
    assert si["rate"] == 48000 and si["resample_ratio"] == pytest.approx(float(ratio))
    assert r0["addr_end"] == 4000 - src(si["len"])
    assert r0["addr_loop_start"] == 500 - src(si["loop_start"]) and r0["addr_loop_end"] == 3900 - src(si["loop_end"])
    assert r0["loop_mode"] == 1 and r1["loop_mode"] == 0
    # a non-lowpass type turns the filter off; a cross-group off_by is reported, not approximated
    assert r1["filter_fc_cents"] == 13500.0 and r1["exclusive_class"] == 0 and r1["addr_start"] == 7
    assert any("off_by (cross-group" in x for x in b.report)
    # a stereo file: two samples, two regions panned hard, the region's own pan overridden
    r2, r3 = b.region_info(2), b.region_info(3)
    assert (r2["pan"], r3["pan"]) == (-1.0, 1.0) and r2["sample"] != r3["sample"]
    assert b.regions == 4 and b.n_samples == 3


def test_refusals(tmp_path):
    (tmp_path / "none.sfz").write_text("<group> volume=1\n")
    with pytest.raises(RuntimeError, match="no <region> sections"):
        load(tmp_path / "none.sfz")
    (tmp_path / "bad.sfz").write_text("<region> sample=gone.wav\n<region> lokey=3\n")
    with pytest.raises(RuntimeError, match="every region was unusable"):
        load(tmp_path / "bad.sfz")
    (tmp_path / "x.wav").write_bytes(b"RIFF\x04\x00\x00\x00WAVX")
    (tmp_path / "fmt.sfz").write_text("<region> sample=x.wav\n")
    with pytest.raises(RuntimeError, match="every region was unusable"):
        load(tmp_path / "fmt.sfz")
    (tmp_path / "loop.sfz").write_text('#include "loop.sfz"\n<region> sample=x.wav\n')
    with pytest.raises(RuntimeError):
        load(tmp_path / "loop.sfz")
    with pytest.raises(RuntimeError, match="unrecognised soundfont extension"):
        H.Bank(tmp_path / "a.txt", _cfg())


def _sfz_kit(tmp_path):
    """Eight looped sample files over the keyboard, one stereo."""
    lines = []
    for i in range(8):
        n = 6000 + 500 * i
        if i == 3:
            data = wav_bytes(np.stack([tone(n, 20 + i), tone(n, 40 + i)], 1), rate=44100, channels=2,
                             smpl=(36 + 12 * (i % 6), 0, (n // 2, n - 1)))
        else:
            data = wav_bytes(tone(n, 20 + i), rate=44100 if i % 2 else 48000,
                             smpl=(36 + 12 * (i % 6), 0, (n // 2, n - 1)))
        (tmp_path / f"s{i}.wav").write_bytes(data)
        lines.append(f"<region> sample=s{i}.wav lokey={16 * i} hikey={16 * i + 15} pitch_keycenter={16 * i + 8} "
                     f"ampeg_release=0.2 cutoff={2000 + 1000 * i} resonance=2 volume=-3")
    (tmp_path / "kit.sfz").write_text("<global> ampeg_attack=0.005 ampeg_decay=0.4 ampeg_sustain=60\n" +
                                      "\n".join(lines) + "\n")
    return tmp_path / "kit.sfz"


def _oracle(cfg, bank):
    from oracle.binding import OracleSynth
    return OracleSynth(cfg, bank.pool, bank.params)


def test_sfz_kit_renders_on_the_cpu_reference(tmp_path):
    from kestrel_b200.render import render_file
    kit = _sfz_kit(tmp_path)
    cfg, _, ms = H.config_workload("plain", seed=9)
    ms.notes, ms.seconds = 3000, 1.0
    st = render_file(tmp_path / "o.wav", cfg, kit, ms, backend=_oracle, max_seconds=0.6)
    x = np.frombuffer((tmp_path / "o.wav").read_bytes()[44:], "<f4")
    assert st.blocks > 3 and np.any(x != 0) and np.max(np.abs(x)) <= 1.0


@gpu
def test_sfz_kit_cuda_nulls_against_the_cpu_reference(tmp_path):
    from kestrel_b200.render import render_file
    kit = _sfz_kit(tmp_path)
    cfg, _, ms = H.config_workload("plain", seed=9)
    ms.notes, ms.seconds = 20000, 2.0
    a = render_file(tmp_path / "cuda.wav", cfg, kit, ms, max_seconds=2.0)
    b = render_file(tmp_path / "cpu.wav", cfg, kit, ms, backend=_oracle, max_seconds=2.0)
    assert a.blocks == b.blocks
    x = np.frombuffer((tmp_path / "cuda.wav").read_bytes()[44:], "<f4").astype(np.float64)
    y = np.frombuffer((tmp_path / "cpu.wav").read_bytes()[44:], "<f4").astype(np.float64)
    d = float(np.max(np.abs(x - y)))
    assert d == 0.0 or 20 * np.log10(d) <= -100.0
