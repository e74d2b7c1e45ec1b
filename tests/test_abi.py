"""The C-ABI libraries load and export every symbol their headers declare.

No compute calls: this runs without a GPU (loading libkestrel_cuda.so needs
only the CUDA runtime library, not a device).
"""
import ctypes as C
import re
from pathlib import Path

import pytest

from kestrel_b200 import host as H
from kestrel_b200 import native as N

ROOT = Path(__file__).resolve().parent.parent


def declared(header: str, prefix: str) -> set[str]:
    text = (ROOT / "include" / header).read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(rf"\b({prefix}[a-z0-9_]+)\s*\(", text))


def test_cuda_header_symbols_exported():
    names = declared("kestrel_cuda.h", "kc_")
    assert len(names) >= 20
    lib = C.CDLL(str(N.CUDA_LIB_PATH))
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    # the ctypes table covers the whole header
    assert names == set(N.CUDA_SYMBOLS), names ^ set(N.CUDA_SYMBOLS)


def test_host_header_symbols_exported():
    names = declared("kestrel_host.h", "kh_")
    lib = C.CDLL(str(H.HOST_LIB_PATH))
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    assert names == set(H.HOST_SYMBOLS), names ^ set(H.HOST_SYMBOLS)


def test_struct_layouts_match_reference():
    # voice::SpawnCmd is 19 x u32 (src/voice.rs:22-57); RegionParams 48 B (src/bank.rs:166-188)
    assert N.SPAWN_DTYPE.itemsize == 76
    assert N.PARAMS_DTYPE.itemsize == 48
    assert C.sizeof(N.KcConfig) == 24 * 4
    assert C.sizeof(N.KcBlockStats) == 32


def test_config_default_matches_reference_defaults():
    lib = N.cuda_lib()
    c = N.KcConfig()
    assert lib.kc_config_default(C.byref(c)) == 0
    d = N.default_config()
    for f, _ in N.KcConfig._fields_:
        if f == "reserved":
            continue
        assert getattr(c, f) == pytest.approx(getattr(d, f)), f
    # src/config.rs:345-409
    assert (c.block_frames, c.gate_frames, c.max_voices, c.max_steal_percent, c.steal_fade_frames) == \
        (4096, 32, 1 << 20, 25, 96)
    assert lib.kc_pool_slots(C.byref(c)) == (1 << 20) + (1 << 20) * 25 // 100


def test_create_without_device_fails_loudly():
    """No CPU fallback: without a usable GPU, creating a context is an error,
    not a silent host render."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    from kestrel_b200.backend import CudaSynth
    import numpy as np
    with pytest.raises(N.KestrelError):
        CudaSynth(N.default_config(max_voices=16), np.zeros(16, np.int16), np.zeros(1, N.PARAMS_DTYPE), 1, 16)


def test_config_validation_needs_no_device():
    """Invalid configs are refused before any device call (validation of the
    tunables the autotuner sets included)."""
    import numpy as np
    lib = N.cuda_lib()
    out = C.c_void_p()
    pool = np.zeros(16, np.int16)
    params = np.zeros(1, N.PARAMS_DTYPE)
    for bad in (dict(sort_radix_bits=3), dict(sort_radix_bits=11), dict(voices_per_lane=3),
                dict(block_frames=1000), dict(mix_mode=7), dict(unit_tile_frames=24), dict(unit_tile_frames=64)):
        cfg = N.default_config(max_voices=16, **bad)
        rc = lib.kc_synth_create(C.byref(cfg), N.ptr(pool), pool.size, N.ptr(params), 1, 1, 16, C.byref(out))
        assert rc == 1, bad  # KC_ERR_INVALID
        assert lib.kc_last_error()
    b = N.KcBatchConfig()
    lib.kc_batch_config_default(C.byref(b))
    b.sort_radix_bits = 12
    assert lib.kc_batch_create(C.byref(b), C.byref(out)) == 1
