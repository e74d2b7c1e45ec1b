"""ctypes declarations of the C ABI in include/kestrel_cuda.h.

The struct layouts are the reference's repr(C) records byte for byte:
``SpawnCmd`` (src/voice.rs:22-57, 76 bytes) and ``RegionParams``
(src/bank.rs:166-188, 48 bytes). NumPy structured dtypes with the same layout
are provided so per-block arrays can be handed to the library without copies.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
CUDA_LIB_PATH = PKG / "libkestrel_cuda.so"

# ---- enums (src/config.rs:11-109) -------------------------------------------
INTERP_NEAREST, INTERP_LINEAR, INTERP_CUBIC = 0, 1, 2
CURVE_EXPONENTIAL, CURVE_LINEAR = 0, 1
STEAL_OLDEST, STEAL_DROP_NEW, STEAL_QUIETEST = 0, 1, 2
ADMIT_LOUDEST, ADMIT_EVEN = 0, 1
MIX_F32_TREE, MIX_TWO_SUM, MIX_F64 = 0, 1, 2

ENV_ATTACK, ENV_DECAY, ENV_SUSTAIN, ENV_RELEASE, ENV_DEAD = 0, 1, 2, 3, 4
GATE_SLOTS = 2048
BEND_CHANNELS, CHAN_FIELDS = 16, 4
VF_LOOP, VF_LOOP_UNTIL_RELEASE = 1, 2
RP_FILTER = 1

# Pool field order of kc_read_pool (shaders/common.wgsl:15-43).
FIELDS = ["phase_lo", "phase_hi", "step_lo", "step_hi", "smp_base", "smp_len", "loop_start",
          "loop_end", "flags", "env_stage", "env_level", "gain_l", "gain_r", "filt_z1", "filt_z2",
          "params", "region", "gate_slot", "ordinal", "start_rel", "note_lo", "note_hi",
          "born_variant", "stop_rel"]
FIELD = {n: i for i, n in enumerate(FIELDS)}

SPAWN_DTYPE = np.dtype([
    ("phase_lo", "<u4"), ("phase_hi", "<u4"), ("step_lo", "<u4"), ("step_hi", "<u4"),
    ("smp_base", "<u4"), ("smp_len", "<u4"), ("loop_start", "<u4"), ("loop_end", "<u4"),
    ("flags", "<u4"), ("params", "<u4"), ("variant", "<u4"), ("region", "<u4"),
    ("gate_slot", "<u4"), ("ordinal", "<u4"), ("start_rel", "<u4"), ("note_id_lo", "<u4"),
    ("note_id_hi", "<u4"), ("gain_l", "<f4"), ("gain_r", "<f4")])
assert SPAWN_DTYPE.itemsize == 76

PARAMS_DTYPE = np.dtype([
    ("attack_rate", "<f4"), ("attack_end", "<f4"), ("decay_coef", "<f4"), ("decay_target", "<f4"),
    ("sustain", "<f4"), ("release_coef", "<f4"), ("b0", "<f4"), ("b1", "<f4"), ("a1", "<f4"),
    ("a2", "<f4"), ("flags", "<u4"), ("pad", "<u4")])
assert PARAMS_DTYPE.itemsize == 48


class KcConfig(C.Structure):
    _fields_ = [
        ("sample_rate", C.c_uint32), ("block_frames", C.c_uint32), ("gate_frames", C.c_uint32),
        ("max_voices", C.c_uint32), ("max_steal_percent", C.c_uint32),
        ("steal_fade_frames", C.c_uint32), ("steal_rule", C.c_uint32), ("admit_rule", C.c_uint32),
        ("interpolation", C.c_uint32), ("decay_curve", C.c_uint32), ("release_curve", C.c_uint32),
        ("env_floor", C.c_float), ("sort_voices", C.c_uint32), ("max_param_variants", C.c_uint32),
        ("mix_mode", C.c_uint32), ("strict_fp", C.c_uint32), ("device", C.c_uint32),
        ("voices_per_lane", C.c_uint32), ("sort_radix_bits", C.c_uint32), ("unit_tile_frames", C.c_uint32),
        ("reserved", C.c_uint32 * 4)]


class KcBlockStats(C.Structure):
    _fields_ = [("active_voices", C.c_uint64), ("stolen", C.c_uint64), ("dropped", C.c_uint64),
                ("peak", C.c_float), ("pad", C.c_uint32)]


def default_config(**overrides) -> KcConfig:
    """config.rs:345-409 defaults (the same values kc_config_default writes)."""
    c = KcConfig()
    c.sample_rate = 48000
    c.block_frames = 4096
    c.gate_frames = 32
    c.max_voices = 1 << 20
    c.max_steal_percent = 25
    c.steal_fade_frames = 96
    c.steal_rule = STEAL_QUIETEST
    c.admit_rule = ADMIT_LOUDEST
    c.interpolation = INTERP_LINEAR
    c.decay_curve = CURVE_EXPONENTIAL
    c.release_curve = CURVE_EXPONENTIAL
    c.env_floor = 1.0e-5
    c.sort_voices = 1
    c.max_param_variants = 32
    c.mix_mode = MIX_F32_TREE
    c.strict_fp = 1
    c.device = 0
    c.voices_per_lane = 0
    c.sort_radix_bits = 0
    c.unit_tile_frames = 0
    for k, v in overrides.items():
        if not hasattr(c, k):
            raise AttributeError(f"kc_config has no field {k!r}")
        setattr(c, k, v)
    return c


class KcBatchConfig(C.Structure):
    _fields_ = [
        ("device", C.c_uint32), ("max_jobs", C.c_uint32), ("block_frames", C.c_uint32),
        ("interpolation", C.c_uint32), ("strict_fp", C.c_uint32), ("mix_mode", C.c_uint32),
        ("voices_per_lane", C.c_uint32), ("use_graph", C.c_uint32), ("sort_radix_bits", C.c_uint32),
        ("reserved", C.c_uint32 * 7)]


def batch_config_for(cfg: KcConfig, max_jobs: int = 256, use_graph: bool = True) -> KcBatchConfig:
    """The batch variant that accepts contexts created with `cfg`."""
    b = KcBatchConfig()
    b.device = cfg.device
    b.max_jobs = max_jobs
    b.block_frames = cfg.block_frames
    b.interpolation = cfg.interpolation
    b.strict_fp = cfg.strict_fp
    b.mix_mode = cfg.mix_mode
    b.voices_per_lane = 2 if cfg.voices_per_lane == 2 else 1
    b.use_graph = 1 if use_graph else 0
    b.sort_radix_bits = cfg.sort_radix_bits
    return b


# Every symbol include/kestrel_cuda.h declares, with its ctypes signature.
_P = C.c_void_p
CUDA_SYMBOLS = {
    "kc_config_default": (C.c_int, [C.POINTER(KcConfig)]),
    "kc_pool_slots": (C.c_uint32, [C.POINTER(KcConfig)]),
    "kc_synth_create": (C.c_int, [C.POINTER(KcConfig), _P, C.c_uint64, _P, C.c_uint32, C.c_uint32,
                                  C.c_uint32, C.POINTER(_P)]),
    "kc_synth_destroy": (None, [_P]),
    "kc_synth_clone": (C.c_int, [_P, C.POINTER(_P)]),
    "kc_synth_clone_config": (C.c_int, [_P, C.POINTER(KcConfig), C.POINTER(_P)]),
    "kc_set_gates": (C.c_int, [_P, _P, C.c_size_t]),
    "kc_set_channels": (C.c_int, [_P, _P, C.c_size_t, C.c_int, C.c_int, C.c_int]),
    "kc_set_params_variant": (C.c_int, [_P, C.c_uint32, _P, C.c_size_t]),
    "kc_spawn": (C.c_int, [_P, _P, C.c_size_t]),
    "kc_render": (C.c_int, [_P, _P, C.c_size_t]),
    "kc_render_begin": (C.c_int, [_P]),
    "kc_render_end": (C.c_int, [_P, _P, C.c_size_t]),
    "kc_render_pending": (C.c_int, [_P]),
    "kc_stats": (C.c_int, [_P, C.POINTER(KcBlockStats)]),
    "kc_name": (C.c_char_p, [_P]),
    "kc_set_profile": (C.c_int, [_P, C.c_int]),
    "kc_timings": (C.c_int, [_P, C.POINTER(C.c_char_p), C.POINTER(C.c_double), C.c_size_t,
                             C.POINTER(C.c_size_t)]),
    "kc_timings_total": (C.c_int, [_P, C.POINTER(C.c_double), C.c_size_t, C.POINTER(C.c_uint64)]),
    "kc_last_error": (C.c_char_p, []),
    "kc_enqueue_block_device": (C.c_int, [_P, _P, _P, C.c_int, C.c_int, C.c_int, _P, C.c_uint32, _P]),
    "kc_synchronize": (C.c_int, [_P]),
    "kc_stream": (_P, [_P]),
    "kc_block_launches": (C.c_int, [_P, C.POINTER(C.c_uint32)]),
    "kc_read_pool": (C.c_int, [_P, _P, C.c_size_t, C.POINTER(C.c_uint32)]),
    "kc_design_lowpass_f64": (C.c_int, [_P, _P, C.c_uint32, C.c_float, _P, C.c_int]),
    "kc_resample_i16_batch": (C.c_int, [_P, C.c_uint32, _P, _P, _P, _P, _P, _P]),
    "kc_batch_config_default": (C.c_int, [C.POINTER(KcBatchConfig)]),
    "kc_batch_create": (C.c_int, [C.POINTER(KcBatchConfig), C.POINTER(_P)]),
    "kc_batch_destroy": (None, [_P]),
    "kc_batch_render": (C.c_int, [_P, C.POINTER(_P), C.c_uint32, C.POINTER(_P)]),
    "kc_batch_last_ms": (C.c_int, [_P, C.POINTER(C.c_float)]),
    "kc_synth_device_bytes": (C.c_uint64, [_P]),
    "kc_estimate_device_bytes": (C.c_int, [C.POINTER(KcConfig), C.c_uint64, C.c_uint32, C.POINTER(C.c_uint64)]),
    "kc_last_block_voices": (C.c_int, [_P, C.POINTER(C.c_uint32)]),
    "kc_last_block_tiles": (C.c_int, [_P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "kc_launches_total": (C.c_int, [_P, C.POINTER(C.c_uint64)]),
    "kc_device_memory": (C.c_int, [C.c_int, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "kc_render_block_noalloc": (C.c_int, [C.POINTER(KcConfig), _P, C.c_uint32, C.c_uint32, _P, C.c_uint64, _P,
                                          C.c_uint32, C.c_uint32, _P, _P, C.c_int, C.c_int, C.c_int, _P, _P]),
}


def bind(lib: C.CDLL, table: dict) -> C.CDLL:
    for name, (res, args) in table.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_cuda_lib: C.CDLL | None = None


def cuda_lib() -> C.CDLL:
    """Load libkestrel_cuda.so. There is no fallback: if the CUDA library is
    missing or cannot load, this raises."""
    global _cuda_lib
    if _cuda_lib is None:
        if not CUDA_LIB_PATH.exists():
            raise RuntimeError(
                f"{CUDA_LIB_PATH} is not built; run `python -m kestrel_b200.build` "
                "(the CUDA backend has no CPU fallback)")
        _cuda_lib = bind(C.CDLL(str(CUDA_LIB_PATH)), CUDA_SYMBOLS)
    return _cuda_lib


class KestrelError(RuntimeError):
    pass


def check(rc: int, lib: C.CDLL | None = None) -> None:
    if rc != 0:
        lib = lib or cuda_lib()
        msg = lib.kc_last_error().decode(errors="replace")
        raise KestrelError(f"status {rc}: {msg}")


def ptr(a: np.ndarray) -> int:
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return a.ctypes.data
