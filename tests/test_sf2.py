"""SoundFont 2 files (src/sf2.rs:145-505): the RIFF walk, the pdta records,
preset and instrument flattening, and the pool build that reads only the
used samples.

The checker is a Python restatement of the flattening rules written here
from the same source (global zones, preset offsets, absolute-only
generators, range intersection, ROM and out-of-range samples skipped), run
on hand-built and randomly generated files. The synthetic banks, which are
now written in the test kit's SF2 layout and loaded by the same code, must
come back byte-identical through a file on disk.
"""
import random
import struct

import numpy as np
import pytest

from kestrel_b200 import host as H
from kestrel_b200 import native as N

ABSOLUTE_ONLY = {0, 1, 2, 3, 4, 12, 45, 50, 53, 54, 57, 58, 46, 47, 41, 43, 44}


def default_gens():
    g = [0] * 60
    g[8] = 13500
    for op in (21, 23, 25, 26, 27, 28, 30, 33, 34, 35, 36, 38):
        g[op] = -12000
    g[43] = 0x7F00
    g[44] = 0x7F00
    g[46] = -1
    g[47] = -1
    g[56] = 100
    g[58] = -1
    return g


def i16(x):
    return ((x + 0x8000) & 0xFFFF) - 0x8000


# ---- a writer with the format's freedom (global zones, several zones per preset) ----

def chunk(cid, payload):
    return cid + struct.pack("<I", len(payload)) + payload + (b"\0" if len(payload) % 2 else b"")


def name20(s):
    return s.encode()[:19].ljust(20, b"\0")


def build_sf2(samples, instruments, presets, info=b"", smpl_pad=46, extra=b""):
    """samples: list of dict(data (int16 array), rate, root, corr, loop=(s, e), rom=False)
    instruments: list of lists of zones; a zone is a list of (op, amount), with
    (53, sid) last when it is not a global zone.
    presets: list of dict(bank, program, zones: list of lists of (op, amount))."""
    smpl = b""
    ranges = []
    frames = 0
    for s in samples:
        d = np.asarray(s["data"], np.int16)
        ranges.append((frames, frames + len(d)))
        smpl += d.astype("<i2").tobytes() + b"\0\0" * smpl_pad
        frames += len(d) + smpl_pad
    phdr = pbag = pgen = inst = ibag = igen = shdr = b""
    for p in presets:
        phdr += name20("p") + struct.pack("<HHHIII", p["program"], p["bank"], len(pbag) // 4, 0, 0, 0)
        for z in p["zones"]:
            pbag += struct.pack("<HH", len(pgen) // 4, 0)
            for op, amt in z:
                pgen += struct.pack("<HH", op, amt & 0xFFFF)
    phdr += name20("EOP") + struct.pack("<HHHIII", 0, 0, len(pbag) // 4, 0, 0, 0)
    pbag += struct.pack("<HH", len(pgen) // 4, 0)
    pgen += struct.pack("<HH", 0, 0)
    for zones in instruments:
        inst += name20("i") + struct.pack("<H", len(ibag) // 4)
        for z in zones:
            ibag += struct.pack("<HH", len(igen) // 4, 0)
            for op, amt in z:
                igen += struct.pack("<HH", op, amt & 0xFFFF)
    inst += name20("EOI") + struct.pack("<H", len(ibag) // 4)
    ibag += struct.pack("<HH", len(igen) // 4, 0)
    igen += struct.pack("<HH", 0, 0)
    for s, (a, b) in zip(samples, ranges):
        ls, le = s.get("loop", (0, b - a))
        stype = 0x8001 if s.get("rom") else 1
        end = b + s.get("end_extra", 0)
        shdr += name20("s") + struct.pack("<IIIIIBbHH", a, end, a + ls, a + le, s.get("rate", 48000),
                                          s.get("root", 60), s.get("corr", 0), 0, stype)
    shdr += name20("EOS") + b"\0" * 26
    sdta = b"sdta" + chunk(b"smpl", smpl)
    pdta = b"pdta" + b"".join(chunk(c, d) for c, d in [
        (b"phdr", phdr), (b"pbag", pbag), (b"pmod", b"\0" * 10), (b"pgen", pgen), (b"inst", inst),
        (b"ibag", ibag), (b"imod", b"\0" * 10), (b"igen", igen), (b"shdr", shdr)])
    body = b"sfbk" + chunk(b"LIST", b"INFO" + chunk(b"ifil", b"\2\0\1\0") + info) + chunk(b"LIST", sdta) + \
        chunk(b"LIST", pdta) + extra
    return b"RIFF" + struct.pack("<I", len(body)) + body, ranges


# ---- the flattening, restated (src/sf2.rs:309-467) -------------------------------------

def range_of(g, is_set, op):
    if not is_set:
        return (0, 127)
    raw = g[op] & 0xFFFF
    lo, hi = raw & 0xFF, raw >> 8
    return (hi, lo) if lo > hi else (lo, hi)


def flatten(samples, instruments, presets, smpl_frames, ranges):
    regions, out_presets, used = [], [], set()
    for p in presets:
        pglob, pglob_set = [0] * 60, [False] * 60
        first = True
        ids = []
        for z in p["zones"]:
            zone, zset, inst = [0] * 60, [False] * 60, None
            for op, amt in z:
                if op == 41:
                    inst = amt & 0xFFFF
                elif op < 60:
                    zone[op], zset[op] = i16(amt), True
            if inst is None:
                if first:
                    pglob, pglob_set = zone, zset
                first = False
                continue
            first = False
            pg, ps = list(pglob), list(pglob_set)
            for i in range(60):
                if zset[i]:
                    pg[i], ps[i] = zone[i], True
            pk, pv = range_of(pg, ps[43], 43), range_of(pg, ps[44], 44)
            if inst >= len(instruments) or not instruments[inst]:
                continue
            iglob = default_gens()
            ifirst = True
            for iz in instruments[inst]:
                ig, sid = list(iglob), None
                for op, amt in iz:
                    if op == 53:
                        sid = amt & 0xFFFF
                    elif op < 60:
                        ig[op] = i16(amt)
                if sid is None:
                    if ifirst:
                        iglob = ig
                    ifirst = False
                    continue
                ifirst = False
                if sid >= len(samples):
                    continue
                s = samples[sid]
                a, b = ranges[sid]
                b += s.get("end_extra", 0)
                if s.get("rom") or b <= a or b > smpl_frames:
                    continue
                ik, iv = range_of(ig, True, 43), range_of(ig, True, 44)
                k = (max(pk[0], ik[0]), min(pk[1], ik[1]))
                v = (max(pv[0], iv[0]), min(pv[1], iv[1]))
                if k[0] > k[1] or v[0] > v[1]:
                    continue
                f = list(ig)
                for op in range(60):
                    if ps[op] and op not in ABSOLUTE_ONLY:
                        f[op] = max(-32768, min(32767, f[op] + pg[op]))
                used.add(sid)
                ids.append(len(regions))
                regions.append((sid, k, v, f))
        if ids:
            out_presets.append((p["bank"], p["program"], ids))
    return regions, out_presets, sorted(used)


def _smpl_frames(ranges, pad=46):
    return ranges[-1][1] + pad if ranges else 0


def expect_region(sid_dense, k, v, f):
    tc = lambda x: 0.0 if x <= -12000 else 2.0 ** (x / 1200.0)
    return {
        "sample": sid_dense, "key_lo": k[0], "key_hi": k[1], "vel_lo": v[0], "vel_hi": v[1],
        "root_key_override": f[58], "fixed_key": f[46], "fixed_vel": f[47], "coarse_tune": f[51],
        "fine_tune": f[52], "scale_tuning": f[56], "keynum_to_hold": f[39], "keynum_to_decay": f[40],
        "loop_mode": {1: 1, 3: 2}.get(f[54] & 3, 0), "exclusive_class": max(0, min(255, f[57])),
        "attenuation_cb": float(f[48]), "pan": max(-1.0, min(1.0, f[17] / 500.0)),
        "addr_start": f[0] + f[4] * 32768, "addr_end": f[1] + f[12] * 32768,
        "addr_loop_start": f[2] + f[45] * 32768, "addr_loop_end": f[3] + f[50] * 32768,
        "delay": tc(f[33]), "attack": tc(f[34]), "hold": tc(f[35]), "decay": tc(f[36]),
        "sustain": 10.0 ** (-max(float(f[37]), 0.0) / 200.0), "release": tc(f[38]),
        "filter_fc_cents": float(f[8]), "filter_q_cb": float(f[9]),
    }


def check_bank(bank, samples, instruments, presets, data, ranges):
    regions, exp_presets, used = flatten(samples, instruments, presets, _smpl_frames(ranges), ranges)
    dense = {sid: i for i, sid in enumerate(used)}
    assert bank.regions == len(regions)
    assert bank.presets == len(exp_presets)
    for i, (sid, k, v, f) in enumerate(regions):
        got = bank.region_info(i)
        exp = expect_region(dense[sid], k, v, f)
        for key, val in exp.items():
            if isinstance(val, float):
                assert got[key] == pytest.approx(val, rel=2e-6, abs=1e-12), (i, key)
            else:
                assert got[key] == val, (i, key, got[key], val)
    for i, (b, p, ids) in enumerate(exp_presets):
        assert bank.preset_info(i) == (b, p, ids)
    # the pool holds each used sample once, in id order, then 8 guard frames
    pool = bank.pool
    assert bank.n_samples == len(used)
    pos = 0
    for j, sid in enumerate(used):
        si = bank.sample_info(j)
        d = np.asarray(samples[sid]["data"], np.int16)
        assert si["start"] == pos and si["len"] == len(d)
        assert np.array_equal(pool[pos:pos + len(d)], d)
        assert not pool[pos + len(d):pos + len(d) + 8].any()
        ls, le = samples[sid].get("loop", (0, len(d)))
        assert si["loop_start"] == min(ls, max(len(d) - 1, 0)) and si["loop_end"] == min(le, len(d))
        assert si["root_key"] == min(samples[sid].get("root", 60), 127)
        assert si["correction_cents"] == samples[sid].get("corr", 0)
        pos += len(d) + 8
    assert pos == len(pool)
    return regions


def _cfg():
    return N.default_config(max_voices=4096)


def _load(tmp_path, data, name="t.sf2", **opt):
    p = tmp_path / name
    p.write_bytes(data)
    return H.Bank(p, _cfg(), H.options(resample_pool=0, **opt))


def _sine(n, seed):
    rng = np.random.default_rng(seed)
    return (rng.integers(-20000, 20000, n)).astype(np.int16)


def test_rich_soundfont(tmp_path):
    """Key splits, pan, an envelope, a filter, a preset-level attenuation
    offset on a second preset (the test kit's rich soundfont)."""
    samples = [dict(data=_sine(4800, 1), rate=48000, root=57, loop=(0, 4096)),
               dict(data=_sine(2048, 2), rate=48000, root=69),
               dict(data=_sine(4096, 3), rate=48000, root=81)]
    zones = [
        [(43, 59 << 8), (44, 127 << 8), (54, 1), (34, -3000), (36, 1200), (37, 200), (38, 0), (17, -400), (53, 0)],
        [(43, 71 << 8 | 60), (44, 127 << 8), (34, -12000), (36, -12000), (37, 0), (38, -1200), (8, 8000), (53, 1)],
        [(43, 127 << 8 | 72), (44, 127 << 8), (34, -12000), (36, 600), (37, 100), (38, -600), (17, 400), (48, 100),
         (53, 2)],
    ]
    presets = [dict(bank=0, program=0, zones=[[(41, 0)]]),
               dict(bank=0, program=1, zones=[[(48, 200), (41, 0)]])]
    data, ranges = build_sf2(samples, [zones], presets)
    bank = _load(tmp_path, data)
    regions = check_bank(bank, samples, [zones], presets, data, ranges)
    assert len(regions) == 6
    assert bank.region_info(5)["attenuation_cb"] == 300.0   # 100 + the preset's 200
    assert bank.region_info(0)["pan"] == pytest.approx(-0.8)
    assert bank.region_info(1)["filter_fc_cents"] == 8000.0


def test_global_zones_and_absolute_only_generators(tmp_path):
    samples = [dict(data=_sine(1000, 4), root=60), dict(data=_sine(1500, 5), root=64)]
    inst = [
        [(48, 50), (38, -1200), (57, 3)],                         # instrument global zone
        [(43, 40 << 8 | 20), (54, 3), (53, 0)],
        [(43, 90 << 8 | 41), (48, 10), (53, 1)],
        [(48, 999)],                                              # a later sampleless zone: skipped
    ]
    presets = [dict(bank=1, program=7, zones=[
        [(48, 20), (43, 60 << 8 | 30), (58, 99), (54, 1), (0, 123)],  # preset global zone
        [(52, 5), (41, 0)],
        [(44, 64 << 8), (41, 0)],
        [(48, 7)],                                                # not first: not global, skipped
    ])]
    data, ranges = build_sf2(samples, [inst], presets)
    bank = _load(tmp_path, data)
    regions = check_bank(bank, samples, [inst], presets, data, ranges)
    r0 = bank.region_info(0)
    assert (r0["key_lo"], r0["key_hi"]) == (30, 40)              # preset range intersects the zone's
    assert r0["attenuation_cb"] == 70.0                           # 50 inherited + 20 preset offset
    assert r0["root_key_override"] == -1 and r0["addr_start"] == 0  # absolute-only at preset level
    assert r0["loop_mode"] == 2 and r0["exclusive_class"] == 3
    assert len(regions) == 4


def test_rom_and_out_of_range_samples_are_skipped(tmp_path):
    samples = [dict(data=_sine(500, 6), rom=True), dict(data=_sine(600, 7)),
               dict(data=_sine(700, 8), end_extra=10_000_000), dict(data=_sine(800, 9))]
    inst = [[(53, 0)], [(53, 1)], [(53, 2)], [(53, 3)], [(53, 40)]]
    presets = [dict(bank=0, program=0, zones=[[(41, 0)]])]
    data, ranges = build_sf2(samples, [inst], presets)
    bank = _load(tmp_path, data)
    check_bank(bank, samples, [inst], presets, data, ranges)
    assert bank.regions == 2 and bank.n_samples == 2


@pytest.mark.parametrize("seed", range(12))
def test_random_soundfonts_flatten_as_restated(tmp_path, seed):
    rng = random.Random(seed)
    samples = [dict(data=_sine(rng.randint(16, 3000), seed * 100 + i), root=rng.randint(0, 140),
                    corr=rng.randint(-50, 50), rom=rng.random() < 0.1,
                    loop=(rng.randint(0, 40), rng.randint(0, 4000)))
               for i in range(rng.randint(1, 8))]
    ops = [8, 9, 17, 33, 34, 35, 36, 37, 38, 39, 40, 48, 51, 52, 56, 0, 1, 2, 3, 4, 12, 45, 50, 54, 57, 58, 46, 47]

    def gens(k):
        out = []
        for _ in range(k):
            op = rng.choice(ops + [43, 44])
            if op in (43, 44):
                lo, hi = rng.randint(0, 127), rng.randint(0, 127)
                out.append((op, hi << 8 | lo))
            else:
                out.append((op, rng.randint(-15000, 15000)))
        return out

    instruments = []
    for _ in range(rng.randint(1, 4)):
        zones = []
        if rng.random() < 0.5:
            zones.append(gens(rng.randint(0, 4)))
        for _ in range(rng.randint(0, 5)):
            zones.append(gens(rng.randint(0, 5)) + [(53, rng.randint(0, len(samples)))])
        instruments.append(zones)
    presets = []
    for p in range(rng.randint(1, 4)):
        zones = []
        if rng.random() < 0.5:
            zones.append(gens(rng.randint(0, 4)))
        for _ in range(rng.randint(1, 4)):
            zones.append(gens(rng.randint(0, 4)) + [(41, rng.randint(0, len(instruments)))])
        presets.append(dict(bank=rng.randint(0, 2), program=rng.randint(0, 127), zones=zones))
    data, ranges = build_sf2(samples, instruments, presets)
    regions, exp_presets, _ = flatten(samples, instruments, presets, _smpl_frames(ranges), ranges)
    if not exp_presets:
        with pytest.raises(RuntimeError, match="no usable presets"):
            _load(tmp_path, data)
        return
    bank = _load(tmp_path, data)
    check_bank(bank, samples, instruments, presets, data, ranges)


@pytest.mark.parametrize("presets,random_gens", [(1, 0), (128, 1)])
@pytest.mark.parametrize("resample", [0, 1])
def test_synthetic_bank_through_a_file_is_identical(tmp_path, presets, random_gens, resample):
    cfg = _cfg()
    spec = H.bank_spec(presets=presets, random_generators=random_gens, seed=11, sample_frames=6000,
                       loop_frames=2000)
    a = H.Bank(spec, cfg, H.options(resample_pool=resample))
    H.write_synthetic_sf2(spec, tmp_path / "synth.sf2")
    b = H.Bank(tmp_path / "synth.sf2", cfg, H.options(resample_pool=resample))
    assert np.array_equal(a.pool, b.pool)
    assert a.params.tobytes() == b.params.tobytes()
    assert (a.regions, a.presets, a.n_samples) == (b.regions, b.presets, b.n_samples)
    for i in range(0, a.regions, 97):
        assert a.region_info(i) == b.region_info(i)
    if random_gens:
        # the presets' own generators arrive as preset-level offsets
        assert len({b.region_info(p * 128)["attack"] for p in range(presets)}) > presets // 2


def test_chunk_walk_pads_odd_chunks_and_clamps_sizes(tmp_path):
    samples = [dict(data=_sine(300, 10))]
    inst = [[(53, 0)]]
    presets = [dict(bank=0, program=0, zones=[[(41, 0)]])]
    # an odd INFO sub-chunk (no ZSTR padding) and an unknown trailing chunk
    data, ranges = build_sf2(samples, [inst], presets, info=chunk(b"INAM", b"odd"), extra=chunk(b"junk", b"x" * 5))
    bank = _load(tmp_path, data)
    check_bank(bank, samples, [inst], presets, data, ranges)
    # a RIFF size larger than the file and a truncated tail are clamped, not fatal
    big = data[:4] + struct.pack("<I", 0x7FFFFFFF) + data[8:] + b"LIS"
    check_bank(_load(tmp_path, big, "big.sf2"), samples, [inst], presets, data, ranges)


@pytest.mark.parametrize("mutate,msg", [
    (lambda d: b"RIFX" + d[4:], "not a RIFF file"),
    (lambda d: d[:8] + b"sfbx" + d[12:], "expected sfbk"),
    (lambda d: d.replace(b"smpl", b"smpX", 1), "no smpl chunk"),
    (lambda d: d.replace(b"igen", b"igeX", 1), "pdta is missing igen"),
])
def test_unusable_files_are_refused(tmp_path, mutate, msg):
    samples = [dict(data=_sine(300, 11))]
    data, _ = build_sf2(samples, [[[(53, 0)]]], [dict(bank=0, program=0, zones=[[(41, 0)]])])
    with pytest.raises(RuntimeError, match=msg):
        _load(tmp_path, mutate(data))


def test_no_presets_and_no_usable_presets(tmp_path):
    samples = [dict(data=_sine(300, 12))]
    data, _ = build_sf2(samples, [[[(53, 0)]]], [])
    with pytest.raises(RuntimeError, match="no presets"):
        _load(tmp_path, data)
    data, _ = build_sf2(samples, [[[(53, 5)]]], [dict(bank=0, program=0, zones=[[(41, 0)]])])
    with pytest.raises(RuntimeError, match="no usable presets"):
        _load(tmp_path, data)
    with pytest.raises(RuntimeError, match="opening"):
        H.Bank(tmp_path / "missing.sf2", _cfg())


def test_resampled_file_pool_matches_the_resampler(tmp_path):
    """A 44.1 kHz sample is pooled at the output rate through resample_i16,
    loop points scaled and rounded (src/sf2.rs:650-666)."""
    d = _sine(4410, 13)
    samples = [dict(data=d, rate=44100, loop=(1000, 4000))]
    data, _ = build_sf2(samples, [[[(53, 0)]]], [dict(bank=0, program=0, zones=[[(41, 0)]])])
    p = tmp_path / "r.sf2"
    p.write_bytes(data)
    bank = H.Bank(p, _cfg(), H.options(resample_pool=1))
    si = bank.sample_info(0)
    ratio = 48000 / 44100
    assert si["rate"] == 48000 and si["len"] == int(np.floor(4410 * ratio + 0.5))
    assert si["loop_start"] == int(np.floor(1000 * ratio + 0.5)) and si["loop_end"] == int(np.floor(4000 * ratio + 0.5))
    assert bank.pool_rate == 48000


def _oracle(cfg, bank):
    from oracle.binding import OracleSynth
    return OracleSynth(cfg, bank.pool, bank.params)


def _render_from_files(tmp_path, backend):
    from kestrel_b200.render import render_file
    cfg, bs, ms = H.config_workload("black", seed=4)
    ms.notes, ms.seconds = 20000, 0.5
    H.write_synthetic_sf2(bs, tmp_path / "bank.sf2")
    H.write_synthetic_midi(ms, tmp_path / "song.mid")
    a = render_file(tmp_path / "mem.wav", cfg, bs, ms, backend=backend)
    b = render_file(tmp_path / "file.wav", cfg, tmp_path / "bank.sf2", tmp_path / "song.mid", backend=backend)
    assert a.blocks == b.blocks and a.blocks > 5
    assert (tmp_path / "mem.wav").read_bytes() == (tmp_path / "file.wav").read_bytes()


def test_rendering_from_sf2_and_midi_files_matches_the_synthetic_inputs(tmp_path):
    """gen-assets then render: the 128-preset bank and its stream, written to
    .sf2 and .mid files and read back, render the same WAV bytes."""
    _render_from_files(tmp_path, _oracle)


@pytest.mark.gpu
def test_cuda_render_from_sf2_and_midi_files(tmp_path):
    from kestrel_b200.render import cuda_backend
    _render_from_files(tmp_path, cuda_backend)
