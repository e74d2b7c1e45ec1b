"""The host side that feeds a backend: synthetic banks, MIDI and the driver.

Binds libkestrel_host.so (include/kestrel_host.h), the C++ restatement of
Kestrel's driver (src/driver.rs), bank (src/bank.rs) and SF2 flattening
(src/sf2.rs). ``run_blocks`` is Driver::next_block's loop
(src/bin/kestrel.rs:311-365 calls it once per block): prepare the block's
inputs, hand them to a backend in the reference's call order, render.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import native as N

HOST_LIB_PATH = Path(__file__).resolve().parent / "libkestrel_host.so"


class KhOptions(C.Structure):
    _fields_ = [("master_volume", C.c_float), ("filter_enabled", C.c_uint32), ("max_layers", C.c_uint32),
                ("default_channel_volume", C.c_uint32), ("resample_pool", C.c_uint32),
                ("read_ahead", C.c_uint32), ("sample_pool_budget", C.c_uint64)]


class KhSynthBankSpec(C.Structure):
    _fields_ = [("presets", C.c_uint32), ("sample_frames", C.c_uint32), ("sample_rate", C.c_uint32),
                ("loop_frames", C.c_uint32), ("amplitude", C.c_float), ("noise", C.c_float),
                ("attack_tc", C.c_int16), ("decay_tc", C.c_int16), ("sustain_cb", C.c_int16),
                ("release_tc", C.c_int16), ("filter_fc_cents", C.c_int16), ("filter_q_cb", C.c_int16),
                ("random_generators", C.c_uint32), ("seed", C.c_uint64)]


class KhMidiSpec(C.Structure):
    _fields_ = [("notes", C.c_uint64), ("seconds", C.c_double), ("channels", C.c_uint32),
                ("key_lo", C.c_uint32), ("key_hi", C.c_uint32), ("vel_lo", C.c_uint32), ("vel_hi", C.c_uint32),
                ("dur_median_s", C.c_double), ("dur_sigma", C.c_double), ("cluster_share", C.c_double),
                ("cluster_lo", C.c_uint32), ("cluster_hi", C.c_uint32), ("cc_period_ms", C.c_double),
                ("program_period_s", C.c_double), ("programs", C.c_uint32), ("ppq", C.c_uint32),
                ("seed", C.c_uint64)]


class KhBlock(C.Structure):
    _fields_ = [("gates", C.POINTER(C.c_uint32)), ("n_gates", C.c_size_t), ("chan", C.POINTER(C.c_uint32)),
                ("n_chan", C.c_size_t), ("bend", C.c_int), ("gain", C.c_int), ("variant", C.c_int),
                ("cmds", C.c_void_p), ("n_cmds", C.c_size_t), ("n_variants", C.c_uint32), ("live", C.c_uint32),
                ("want", C.c_uint32), ("take", C.c_uint32), ("block_index", C.c_uint64), ("notes", C.c_uint64),
                ("want_energy", C.c_uint64), ("take_energy", C.c_uint64)]


class KhRegionInfo(C.Structure):
    _fields_ = [("sample", C.c_uint32), ("key_lo", C.c_uint8), ("key_hi", C.c_uint8), ("vel_lo", C.c_uint8),
                ("vel_hi", C.c_uint8), ("root_key_override", C.c_int16), ("fixed_key", C.c_int16),
                ("fixed_vel", C.c_int16), ("coarse_tune", C.c_int16), ("fine_tune", C.c_int16),
                ("scale_tuning", C.c_int16), ("keynum_to_hold", C.c_int16), ("keynum_to_decay", C.c_int16),
                ("loop_mode", C.c_uint8), ("exclusive_class", C.c_uint8), ("attenuation_cb", C.c_float),
                ("pan", C.c_float), ("addr_start", C.c_int32), ("addr_end", C.c_int32),
                ("addr_loop_start", C.c_int32), ("addr_loop_end", C.c_int32), ("delay", C.c_float),
                ("attack", C.c_float), ("hold", C.c_float), ("decay", C.c_float), ("sustain", C.c_float),
                ("release", C.c_float), ("filter_fc_cents", C.c_float), ("filter_q_cb", C.c_float)]


class KhSampleInfo(C.Structure):
    _fields_ = [("start", C.c_uint32), ("len", C.c_uint32), ("loop_start", C.c_uint32), ("loop_end", C.c_uint32),
                ("rate", C.c_uint32), ("root_key", C.c_uint32), ("correction_cents", C.c_float),
                ("resample_ratio", C.c_float)]


def _as_dict(s: C.Structure) -> dict:
    return {name: getattr(s, name) for name, _ in s._fields_}


_P = C.c_void_p
HOST_SYMBOLS = {
    "kh_options_default": (None, [C.POINTER(KhOptions)]),
    "kh_synth_bank_spec_default": (None, [C.POINTER(KhSynthBankSpec)]),
    "kh_bank_synthetic": (_P, [C.POINTER(KhSynthBankSpec), C.POINTER(N.KcConfig), C.POINTER(KhOptions)]),
    "kh_bank_destroy": (None, [_P]),
    "kh_bank_open_sf2": (_P, [C.c_char_p, C.POINTER(N.KcConfig), C.POINTER(KhOptions)]),
    "kh_bank_open_sfz": (_P, [C.c_char_p, C.POINTER(N.KcConfig), C.POINTER(KhOptions)]),
    "kh_bank_open": (_P, [C.c_char_p, C.POINTER(N.KcConfig), C.POINTER(KhOptions)]),
    "kh_bank_report": (C.c_char_p, [_P]),
    "kh_sfz_note_name": (C.c_int, [C.c_char_p, C.POINTER(C.c_int32)]),
    "kh_sfz_value_end": (C.c_size_t, [C.c_char_p]),
    "kh_sf2_write_synthetic": (C.c_int, [C.POINTER(KhSynthBankSpec), C.c_char_p]),
    "kh_bank_samples": (C.c_uint32, [_P]),
    "kh_bank_region_info": (C.c_int, [_P, C.c_uint32, C.POINTER(KhRegionInfo)]),
    "kh_bank_sample_info": (C.c_int, [_P, C.c_uint32, C.POINTER(KhSampleInfo)]),
    "kh_bank_preset_info": (C.c_int, [_P, C.c_uint32, C.POINTER(C.c_uint16), C.POINTER(C.c_uint16),
                                      C.POINTER(C.c_uint32), _P, C.c_uint32]),
    "kh_bank_pool": (C.c_int, [_P, C.POINTER(C.POINTER(C.c_int16)), C.POINTER(C.c_uint64)]),
    "kh_bank_params": (C.c_int, [_P, C.POINTER(_P), C.POINTER(C.c_uint32)]),
    "kh_bank_regions": (C.c_uint32, [_P]),
    "kh_bank_presets": (C.c_uint32, [_P]),
    "kh_bank_max_sample_len": (C.c_uint32, [_P]),
    "kh_bank_pool_rate": (C.c_uint32, [_P]),
    "kh_bank_filter_inputs": (C.c_int, [_P, _P, _P, _P, C.c_uint32]),
    "kh_midi_spec_default": (None, [C.POINTER(KhMidiSpec)]),
    "kh_driver_open": (_P, [C.POINTER(N.KcConfig), C.POINTER(KhOptions), _P, C.POINTER(KhMidiSpec)]),
    "kh_driver_destroy": (None, [_P]),
    "kh_driver_open_smf": (_P, [C.POINTER(N.KcConfig), C.POINTER(KhOptions), _P, C.c_char_p]),
    "kh_smf_open": (_P, [C.c_char_p]),
    "kh_smf_close": (None, [_P]),
    "kh_smf_info": (C.c_int, [_P, C.POINTER(C.c_uint16), C.POINTER(C.c_uint16), C.POINTER(C.c_uint32),
                              C.POINTER(C.c_uint8), C.POINTER(C.c_uint8)]),
    "kh_smf_next": (C.c_int, [_P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint32), C.POINTER(C.c_uint8),
                              C.POINTER(C.c_uint8), C.POINTER(C.c_uint8), C.POINTER(C.c_int16),
                              C.POINTER(C.c_uint32)]),
    "kh_midi_write_synthetic": (C.c_int, [C.POINTER(KhMidiSpec), C.c_char_p, C.c_uint64]),
    "kh_driver_prepare": (C.c_int, [_P, C.c_uint32, C.POINTER(KhBlock)]),
    "kh_driver_variant": (C.c_int, [_P, C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(_P), C.POINTER(C.c_size_t)]),
    "kh_driver_finish": (C.c_int, [_P, C.c_uint64, C.POINTER(C.c_int)]),
    "kh_driver_collect": (C.c_int, [_P]),
    "kh_driver_admit": (C.c_int, [_P, C.c_uint32, C.POINTER(KhBlock)]),
    "kh_driver_advance": (C.c_int, [_P]),
    "kh_driver_admit_ready": (C.c_int, [_P]),
    "kh_driver_more": (C.c_int, [_P, C.c_uint64, C.POINTER(C.c_int)]),
    "kh_last_error": (C.c_char_p, []),
    "kh_gates_new": (_P, [C.c_uint32, C.c_uint32]),
    "kh_gates_destroy": (None, [_P]),
    "kh_gates_begin_block": (None, [_P]),
    "kh_gates_end_block": (None, [_P]),
    "kh_gates_note_on": (C.c_uint32, [_P, C.c_uint8, C.c_uint8, C.c_uint32]),
    "kh_gates_note_off": (None, [_P, C.c_uint8, C.c_uint8, C.c_uint32]),
    "kh_gates_set_sustain": (None, [_P, C.c_uint8, C.c_int, C.c_uint32]),
    "kh_gates_set_sostenuto": (None, [_P, C.c_uint8, C.c_int, C.c_uint32]),
    "kh_gates_row": (C.c_uint32, [_P, C.c_uint32, C.c_uint32]),
    "kh_gates_tiles": (C.c_uint32, [_P]),
    "kh_gates_sounding": (C.c_uint64, [_P]),
    "kh_velocity_atten_cb": (C.c_float, [C.c_uint8, C.c_float]),
    "kh_biquad_lowpass": (None, [C.c_float, C.c_float, C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                 C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "kh_timecents_to_secs": (C.c_float, [C.c_float]),
    "kh_resample_i16": (C.c_size_t, [_P, C.c_size_t, C.c_double, _P, C.c_size_t]),
    "kh_set_resampler": (None, [_P, _P]),
    "kh_limiter_create": (_P, [C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int]),
    "kh_limiter_destroy": (None, [_P]),
    "kh_limiter_latency": (C.c_uint32, [_P]),
    "kh_limiter_process": (C.c_uint64, [_P, _P, C.c_size_t]),
    "kh_limiter_report": (C.c_int, [_P, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "kh_clamp_block": (C.c_uint64, [_P, C.c_size_t]),
    "kh_wav_create": (_P, [C.c_char_p, C.c_uint32, C.c_uint16, C.c_uint32]),
    "kh_wav_write": (C.c_int, [_P, _P, C.c_size_t]),
    "kh_wav_finish": (C.c_int, [_P, C.POINTER(C.c_uint64)]),
    "kh_sinc_table": (C.c_int, [C.c_double, _P, C.c_size_t]),
    "kh_mix48": (C.c_uint64, [C.c_uint64]),
    "kh_rank_gain_q": (C.c_uint64, [C.c_float, C.c_float]),
}

_lib: C.CDLL | None = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not HOST_LIB_PATH.exists():
            raise RuntimeError(f"{HOST_LIB_PATH} is not built; run `python -m kestrel_b200.build`")
        _lib = N.bind(C.CDLL(str(HOST_LIB_PATH)), HOST_SYMBOLS)
    return _lib


class GateTable:
    """voice::GateTable (src/voice.rs:212-452) from the host library."""

    def __init__(self, block_frames: int, gate_frames: int):
        self._lib = lib()
        self._h = self._lib.kh_gates_new(block_frames, gate_frames)
        if not self._h:
            raise ValueError("gate_frames must divide block_frames")
        self.tiles = self._lib.kh_gates_tiles(self._h)

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.kh_gates_destroy(self._h)
            self._h = None

    @staticmethod
    def slot(ch: int, key: int) -> int:
        return (ch & 15) * 128 + (key & 127)

    def begin_block(self):
        self._lib.kh_gates_begin_block(self._h)

    def end_block(self):
        self._lib.kh_gates_end_block(self._h)

    def note_on(self, ch, key, frame) -> int:
        return self._lib.kh_gates_note_on(self._h, ch, key, frame)

    def note_off(self, ch, key, frame):
        self._lib.kh_gates_note_off(self._h, ch, key, frame)

    def set_sustain(self, ch, down, frame):
        self._lib.kh_gates_set_sustain(self._h, ch, int(down), frame)

    def set_sostenuto(self, ch, down, frame):
        self._lib.kh_gates_set_sostenuto(self._h, ch, int(down), frame)

    def row(self, tile: int) -> np.ndarray:
        return np.array([self._lib.kh_gates_row(self._h, tile, s) for s in range(2048)], np.uint32)

    def sounding(self) -> int:
        return self._lib.kh_gates_sounding(self._h)


def velocity_atten_cb(vel: int, veltrack: float) -> float:
    return lib().kh_velocity_atten_cb(vel, veltrack)


def biquad_lowpass(fc: float, q_cb: float, sr: float):
    o = [C.c_float() for _ in range(4)]
    lib().kh_biquad_lowpass(fc, q_cb, sr, *[C.byref(x) for x in o])
    return tuple(np.float32(x.value) for x in o)


def timecents_to_secs(tc: float) -> float:
    return lib().kh_timecents_to_secs(tc)


def resample_i16(src: np.ndarray, ratio: float) -> np.ndarray:
    src = np.ascontiguousarray(src, np.int16)
    cap = int(round(src.size * ratio)) + 2
    out = np.empty(cap, np.int16)
    n = lib().kh_resample_i16(N.ptr(src), src.size, ratio, N.ptr(out), cap)
    return out[:n].copy()


EV_NAMES = ["note_on", "note_off", "cc", "program", "pitch_bend", "tempo", "other"]


def read_smf(path):
    """(info, events) of a standard MIDI file: info = (format, tracks, ppq,
    fps, ticks_per_frame), events = [(tick, kind, ch, a, b, bend, tempo)] in
    merged tick order (MidiStream, src/midi.rs:239-374)."""
    L = lib()
    h = L.kh_smf_open(str(path).encode())
    if not h:
        raise RuntimeError(L.kh_last_error().decode())
    try:
        f, t, q = C.c_uint16(), C.c_uint16(), C.c_uint32()
        fps, tpf = C.c_uint8(), C.c_uint8()
        L.kh_smf_info(h, C.byref(f), C.byref(t), C.byref(q), C.byref(fps), C.byref(tpf))
        info = (f.value, t.value, q.value, fps.value, tpf.value)
        ev = []
        tick, typ = C.c_uint64(), C.c_uint32()
        ch, a, b = C.c_uint8(), C.c_uint8(), C.c_uint8()
        bend, tempo = C.c_int16(), C.c_uint32()
        while L.kh_smf_next(h, C.byref(tick), C.byref(typ), C.byref(ch), C.byref(a), C.byref(b), C.byref(bend),
                            C.byref(tempo)):
            ev.append((tick.value, EV_NAMES[typ.value], ch.value, a.value, b.value, bend.value, tempo.value))
        return info, ev
    finally:
        L.kh_smf_close(h)


def write_synthetic_midi(spec: KhMidiSpec, path, max_events: int = 0) -> None:
    """The synthetic stream of `spec` as a format-1, one-track SMF."""
    if lib().kh_midi_write_synthetic(C.byref(spec), str(path).encode(), max_events) != 0:
        raise OSError(lib().kh_last_error().decode())


LIMITER_OFF, LIMITER_OMNI, LIMITER_BRICKWALL = 0, 1, 2
WAV_PCM16, WAV_FLOAT32 = 0, 1


class Limiter:
    """The output stage after each render (src/driver.rs:596-606): the
    limiter, then clamp_block. Defaults are the reference's config."""

    def __init__(self, mode: int = LIMITER_BRICKWALL, sample_rate: int = 48000, ceiling_db: float = 0.0,
                 lookahead_ms: float = 2.0, release_ms: float = 60.0, sustain_ms: float = 0.0,
                 true_peak: bool = True):
        self._lib = lib()
        h = self._lib.kh_limiter_create(mode, sample_rate, ceiling_db, lookahead_ms, release_ms, sustain_ms,
                                        1 if true_peak else 0)
        if not h:
            raise ValueError(self._lib.kh_last_error().decode())
        self._h = h
        self.clipped = 0

    @property
    def latency(self) -> int:
        return self._lib.kh_limiter_latency(self._h)

    def process(self, buf: np.ndarray) -> np.ndarray:
        """In place on an interleaved f32 block; returns it."""
        assert buf.dtype == np.float32 and buf.flags["C_CONTIGUOUS"]
        self.clipped += self._lib.kh_limiter_process(self._h, N.ptr(buf), buf.size)
        return buf

    def report(self):
        p, g = C.c_double(), C.c_double()
        self._lib.kh_limiter_report(self._h, C.byref(p), C.byref(g))
        return p.value, g.value

    def close(self):
        if getattr(self, "_h", None):
            self._lib.kh_limiter_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


class WavWriter:
    """WavWriter (src/wav.rs:50-159): pcm16 or float32, sizes patched at finish."""

    def __init__(self, path, sample_rate: int = 48000, channels: int = 2, fmt: int = WAV_FLOAT32):
        self._lib = lib()
        h = self._lib.kh_wav_create(str(path).encode(), sample_rate, channels, fmt)
        if not h:
            raise OSError(self._lib.kh_last_error().decode())
        self._h = h

    def write(self, block: np.ndarray) -> None:
        block = np.ascontiguousarray(block, dtype=np.float32)
        if self._lib.kh_wav_write(self._h, N.ptr(block), block.size) != 0:
            raise OSError("wav write failed")

    def finish(self) -> int:
        n = C.c_uint64()
        rc = self._lib.kh_wav_finish(self._h, C.byref(n))
        self._h = None
        if rc != 0:
            raise OSError("wav finish failed")
        return n.value


def write_synthetic_sf2(spec: KhSynthBankSpec, path) -> None:
    """The synthetic bank of `spec` as a SoundFont 2 file."""
    if lib().kh_sf2_write_synthetic(C.byref(spec), str(path).encode()) != 0:
        raise OSError(lib().kh_last_error().decode())


def sinc_table(ratio: float) -> np.ndarray:
    """SincBank::new's 512 x 32 f32 table for a ratio (phase-major)."""
    t = np.empty(512 * 32, np.float32)
    if lib().kh_sinc_table(ratio, N.ptr(t), t.size) != 0:
        raise RuntimeError(lib().kh_last_error().decode())
    return t.reshape(512, 32)


_device_ordinals: dict = {}


def use_device_resampler(device: int | None = 0) -> None:
    """Route every bank's load-time resampling through kc_resample_i16_batch
    on `device` (None: back to the host loop). Process-wide."""
    if device is None:
        lib().kh_set_resampler(None, None)
        return
    cuda = N.cuda_lib()
    ordinal = _device_ordinals.setdefault(device, C.c_int(device))  # kept alive for the hook
    lib().kh_set_resampler(C.cast(cuda.kc_resample_i16_batch, C.c_void_p), C.cast(C.byref(ordinal), C.c_void_p))


def mix48(i: int) -> int:
    return lib().kh_mix48(i)


def rank_gain_q(gl: float, gr: float) -> int:
    return lib().kh_rank_gain_q(gl, gr)


def options(**kw) -> KhOptions:
    o = KhOptions()
    lib().kh_options_default(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def bank_spec(**kw) -> KhSynthBankSpec:
    s = KhSynthBankSpec()
    lib().kh_synth_bank_spec_default(C.byref(s))
    for k, v in kw.items():
        setattr(s, k, v)
    return s


def midi_spec(**kw) -> KhMidiSpec:
    s = KhMidiSpec()
    lib().kh_midi_spec_default(C.byref(s))
    for k, v in kw.items():
        setattr(s, k, v)
    return s


class Bank:
    """A loaded bank: the i16 sample pool and the variant-0 params table.
    `spec` is a synthetic bank spec or the path of a soundfont (.sf2 or .sfz)."""

    def __init__(self, spec, cfg: N.KcConfig, opt: KhOptions | None = None):
        self._lib = lib()
        self.opt = opt or options()
        if isinstance(spec, KhSynthBankSpec):
            h = self._lib.kh_bank_synthetic(C.byref(spec), C.byref(cfg), C.byref(self.opt))
        else:
            h = self._lib.kh_bank_open(str(spec).encode(), C.byref(cfg), C.byref(self.opt))
        if not h:
            raise RuntimeError(self._lib.kh_last_error().decode())
        self._h = h
        p = C.POINTER(C.c_int16)()
        n = C.c_uint64()
        self._lib.kh_bank_pool(h, C.byref(p), C.byref(n))
        self.pool = np.ctypeslib.as_array(p, shape=(n.value,)).copy() if n.value else np.zeros(0, np.int16)
        pp = C.c_void_p()
        m = C.c_uint32()
        self._lib.kh_bank_params(h, C.byref(pp), C.byref(m))
        self.params = np.frombuffer((C.c_char * (m.value * 48)).from_address(pp.value),
                                    dtype=N.PARAMS_DTYPE).copy()
        self.regions = self._lib.kh_bank_regions(h)
        self.presets = self._lib.kh_bank_presets(h)
        self.max_sample_len = self._lib.kh_bank_max_sample_len(h)
        self.pool_rate = self._lib.kh_bank_pool_rate(h)

    @property
    def report(self) -> list[str]:
        """The loader's warnings (unreadable samples, unsupported opcodes)."""
        return [x for x in self._lib.kh_bank_report(self._h).decode().split("\n") if x]

    @property
    def n_samples(self) -> int:
        return self._lib.kh_bank_samples(self._h)

    def region_info(self, i: int) -> dict:
        r = KhRegionInfo()
        if self._lib.kh_bank_region_info(self._h, i, C.byref(r)) != 0:
            raise IndexError(self._lib.kh_last_error().decode())
        return _as_dict(r)

    def sample_info(self, i: int) -> dict:
        s = KhSampleInfo()
        if self._lib.kh_bank_sample_info(self._h, i, C.byref(s)) != 0:
            raise IndexError(self._lib.kh_last_error().decode())
        return _as_dict(s)

    def preset_info(self, i: int) -> tuple[int, int, list[int]]:
        """(bank, program, region indexes) of preset i."""
        bank, prog, n = C.c_uint16(), C.c_uint16(), C.c_uint32()
        if self._lib.kh_bank_preset_info(self._h, i, C.byref(bank), C.byref(prog), C.byref(n), None, 0) != 0:
            raise IndexError(self._lib.kh_last_error().decode())
        regs = (C.c_uint32 * max(n.value, 1))()
        self._lib.kh_bank_preset_info(self._h, i, None, None, None, regs, n.value)
        return bank.value, prog.value, list(regs[:n.value])

    def filter_inputs(self):
        """(cutoff Hz, Q cB, on) per variant-0 params entry."""
        n = self.params.size
        fc = np.empty(n, np.float32)
        q = np.empty(n, np.float32)
        on = np.empty(n, np.uint8)
        if self._lib.kh_bank_filter_inputs(self._h, N.ptr(fc), N.ptr(q), N.ptr(on), n) != 0:
            raise RuntimeError(self._lib.kh_last_error().decode())
        return fc, q, on.astype(bool)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.kh_bank_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


@dataclass
class BlockInputs:
    """One block's backend arguments, owned (copied out of the driver)."""
    gates: np.ndarray
    chan: np.ndarray
    bend: bool
    gain: bool
    variant: bool
    cmds: np.ndarray
    variants: list = field(default_factory=list)
    live: int = 0
    want: int = 0
    take: int = 0
    want_energy: int = 0
    take_energy: int = 0


class Driver:
    """Driver::next_block's host side over a synthetic MIDI spec, or over a
    standard MIDI file when `midi` is a path."""

    def __init__(self, cfg: N.KcConfig, bank: Bank, midi):
        self._lib = lib()
        self.bank = bank
        if isinstance(midi, KhMidiSpec):
            h = self._lib.kh_driver_open(C.byref(cfg), C.byref(bank.opt), bank._h, C.byref(midi))
        else:
            h = self._lib.kh_driver_open_smf(C.byref(cfg), C.byref(bank.opt), bank._h, str(midi).encode())
        if not h:
            raise RuntimeError(self._lib.kh_last_error().decode())
        self._h = h
        self.more = True

    def close(self):
        if getattr(self, "_h", None):
            self._lib.kh_driver_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def prepare(self, live: int) -> BlockInputs:
        b = KhBlock()
        self._lib.kh_driver_prepare(self._h, live, C.byref(b))
        return self._inputs(b)

    # next_block in the halves a pipelined loop calls: collect() reads the
    # block's events and needs nothing from the backend, so it may run while
    # the backend renders the previous block; admit(live) then needs that
    # block's active_voices. advance() and more_after() are finish() split at
    # the same place.
    def collect(self) -> None:
        self._lib.kh_driver_collect(self._h)

    def admit(self, live: int) -> BlockInputs:
        return self._inputs(self.admit_raw(live))

    def admit_raw(self, live: int) -> KhBlock:
        """admit() without copying: the block's pointers reach into the
        driver's buffers and stay valid until the next collect()."""
        b = KhBlock()
        self._lib.kh_driver_admit(self._h, live, C.byref(b))
        return b

    def variant_ptrs(self, b: KhBlock) -> list[tuple[int, int, int]]:
        """The block's params variants as (index, address, entries)."""
        out = []
        for i in range(b.n_variants):
            idx, data, n = C.c_uint32(), C.c_void_p(), C.c_size_t()
            self._lib.kh_driver_variant(self._h, i, C.byref(idx), C.byref(data), C.byref(n))
            out.append((idx.value, data.value, n.value))
        return out

    def admit_ready(self) -> bool:
        """Whether the collected block's admission is the same for every
        live count, so it may run before the previous block has rendered."""
        return bool(self._lib.kh_driver_admit_ready(self._h))

    def advance(self) -> None:
        self._lib.kh_driver_advance(self._h)

    def more_after(self, active_voices: int) -> bool:
        more = C.c_int()
        self._lib.kh_driver_more(self._h, active_voices, C.byref(more))
        self.more = bool(more.value)
        return self.more

    def _inputs(self, b: KhBlock) -> BlockInputs:
        gates = np.ctypeslib.as_array(b.gates, shape=(b.n_gates,)).copy()
        chan = np.ctypeslib.as_array(b.chan, shape=(b.n_chan,)).copy()
        if b.n_cmds:
            cmds = np.frombuffer((C.c_char * (b.n_cmds * 76)).from_address(b.cmds), dtype=N.SPAWN_DTYPE).copy()
        else:
            cmds = np.zeros(0, N.SPAWN_DTYPE)
        variants = []
        for i in range(b.n_variants):
            idx = C.c_uint32()
            data = C.c_void_p()
            n = C.c_size_t()
            self._lib.kh_driver_variant(self._h, i, C.byref(idx), C.byref(data), C.byref(n))
            arr = np.frombuffer((C.c_char * (n.value * 48)).from_address(data.value), dtype=N.PARAMS_DTYPE).copy()
            variants.append((idx.value, arr))
        return BlockInputs(gates, chan, bool(b.bend), bool(b.gain), bool(b.variant), cmds, variants, b.live, b.want,
                           b.take, b.want_energy, b.take_energy)

    def finish(self, active_voices: int) -> bool:
        more = C.c_int()
        self._lib.kh_driver_finish(self._h, active_voices, C.byref(more))
        self.more = bool(more.value)
        return self.more


def feed(backend, blk: BlockInputs) -> None:
    """Hand one block to a backend in Driver::next_block's order
    (src/driver.rs:531-588): variants, gates, channels, spawn."""
    for idx, data in blk.variants:
        backend.set_params_variant(idx, data)
    backend.set_gates(blk.gates)
    backend.set_channels(blk.chan, blk.bend, blk.gain, blk.variant)
    backend.spawn(blk.cmds)


def run_blocks(backend, driver: Driver, n_blocks: int, record: bool = False, on_block=None):
    """Drive `backend` for up to n_blocks blocks. Returns (outputs, inputs)."""
    outs, inputs = [], []
    for _ in range(n_blocks):
        live = backend.stats().active_voices
        blk = driver.prepare(live)
        feed(backend, blk)
        out = backend.render()
        outs.append(out.copy())
        if record:
            inputs.append(blk)
        if on_block:
            on_block(blk, out)
        if not driver.finish(backend.stats().active_voices):
            break
    return outs, inputs


# ---- the benchmark configurations --------------------------------------------

def config_workload(name: str, seed: int = 1):
    """(kc_config, bank spec, midi spec) of a named workload: 'plain' (100k
    notes, 30 s, 1 preset, 65,536 voices), 'black' (20M notes, 180 s, 128
    presets, clusters, bend/CC7/CC11 every 10 ms, 1,048,576 voices), 'steal'
    (200M notes, 120 s, sustained concurrency over an 8,388,608-voice pool,
    steal-percent 10). Seeded synthetic stand-ins with the shapes the
    benchmark configurations describe."""
    if name == "plain":
        cfg = N.default_config(max_voices=65536)
        bs = bank_spec(presets=1, seed=seed)
        ms = midi_spec(notes=100_000, seconds=30.0, dur_median_s=0.150, dur_sigma=1.0, seed=seed)
    elif name == "black":
        cfg = N.default_config(max_voices=1_048_576)
        bs = bank_spec(presets=128, random_generators=1, seed=seed)
        ms = midi_spec(notes=20_000_000, seconds=180.0, dur_median_s=0.080, dur_sigma=1.0, cluster_share=0.6,
                       cluster_lo=1000, cluster_hi=50000, cc_period_ms=10.0, program_period_s=2.0, programs=128,
                       seed=seed)
    elif name in ("steal", "steal-bent"):
        cfg = N.default_config(max_voices=8_388_608, max_steal_percent=10)
        bs = bank_spec(presets=1, seed=seed)
        # steal-bent: the same notes with a pitch-bend, CC7 and CC11 curve per
        # channel every 10 ms, so every voice steps by a fractional ratio that
        # changes each gate tile (the interpolating path real soundfonts take).
        ms = midi_spec(notes=200_000_000, seconds=120.0, dur_median_s=6.0, dur_sigma=0.5, seed=seed,
                       cc_period_ms=10.0 if name == "steal-bent" else 0.0)
    else:
        raise ValueError(f"unknown workload {name!r}")
    return cfg, bs, ms
