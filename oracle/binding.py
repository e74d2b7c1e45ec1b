"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA backend. Imported by
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs, never by the
product package. ``OracleSynth`` has the same methods as
``kestrel_b200.backend.CudaSynth`` so a parity test drives both identically.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from kestrel_b200 import native as N

ORACLE_LIB_PATH = Path(__file__).resolve().parent / "liboracle.so"

_P = C.c_void_p
ORACLE_SYMBOLS = {
    "ko_create": (_P, [C.POINTER(N.KcConfig), _P, C.c_uint64, _P, C.c_uint32]),
    "ko_destroy": (None, [_P]),
    "ko_set_gates": (C.c_int, [_P, _P, C.c_size_t]),
    "ko_set_channels": (C.c_int, [_P, _P, C.c_size_t, C.c_int, C.c_int, C.c_int]),
    "ko_set_params_variant": (C.c_int, [_P, C.c_uint32, _P, C.c_size_t]),
    "ko_spawn": (C.c_int, [_P, _P, C.c_size_t]),
    "ko_render": (C.c_int, [_P, _P, C.c_size_t, _P, C.c_int]),
    "ko_stats": (C.c_int, [_P, C.POINTER(N.KcBlockStats)]),
    "ko_read_pool": (C.c_int, [_P, _P, C.c_size_t, C.POINTER(C.c_uint32)]),
    "ko_load_pool": (C.c_int, [_P, _P, C.c_uint32, C.c_uint64, C.c_uint64]),
    "ko_max_steal": (C.c_uint32, [C.POINTER(N.KcConfig)]),
    "ko_steal_span": (C.c_uint32, [C.POINTER(N.KcConfig)]),
    "ko_pool_slots": (C.c_uint32, [C.POINTER(N.KcConfig)]),
    "ko_admit_take": (C.c_uint32, [C.POINTER(N.KcConfig), C.c_uint32, C.c_uint32]),
    "ko_fixed_from_f64": (C.c_uint64, [C.c_double]),
    "ko_fixed_scale": (C.c_uint64, [C.c_uint64, C.c_uint32]),
    "ko_bend_factor": (C.c_uint32, [C.c_double]),
    "ko_catmull_rom": (C.c_float, [C.c_float, C.c_float, C.c_float, C.c_float, C.c_float]),
}

_lib: C.CDLL | None = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not ORACLE_LIB_PATH.exists():
            from kestrel_b200 import build
            build.build_oracle()
        _lib = N.bind(C.CDLL(str(ORACLE_LIB_PATH)), ORACLE_SYMBOLS)
    return _lib


class OracleSynth:
    """CpuSynth (src/cpu.rs) behind the same method names as CudaSynth."""

    def __init__(self, cfg: N.KcConfig, pool: np.ndarray, params: np.ndarray, n_regions: int = 0,
                 max_sample_len: int = 0, threads: int = 1):
        self._lib = lib()
        self.cfg = cfg
        self._pool = np.ascontiguousarray(pool, dtype=np.int16)
        params = np.ascontiguousarray(params, dtype=N.PARAMS_DTYPE)
        h = self._lib.ko_create(C.byref(cfg), N.ptr(self._pool) if self._pool.size else None,
                                self._pool.size, N.ptr(params), params.size)
        if not h:
            raise ValueError("oracle rejected the config")
        self._h = h
        self.block_frames = cfg.block_frames
        self.threads = threads
        self.last_mix64: np.ndarray | None = None

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.ko_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def set_gates(self, rows):
        rows = np.ascontiguousarray(rows, dtype=np.uint32)
        assert self._lib.ko_set_gates(self._h, N.ptr(rows), rows.size) == 0

    def set_channels(self, rows, bend, gain, variant):
        rows = np.ascontiguousarray(rows, dtype=np.uint32)
        assert self._lib.ko_set_channels(self._h, N.ptr(rows), rows.size, int(bend), int(gain),
                                         int(variant)) == 0

    def set_params_variant(self, index, data):
        data = np.ascontiguousarray(data, dtype=N.PARAMS_DTYPE)
        assert self._lib.ko_set_params_variant(self._h, index, N.ptr(data), data.size) == 0

    def spawn(self, cmds):
        cmds = np.ascontiguousarray(cmds, dtype=N.SPAWN_DTYPE)
        assert self._lib.ko_spawn(self._h, N.ptr(cmds) if cmds.size else None, cmds.size) == 0

    def render(self, out=None, keep_mix64: bool = True):
        if out is None:
            out = np.empty(self.block_frames * 2, dtype=np.float32)
        mix = np.empty(self.block_frames * 2, dtype=np.float64) if keep_mix64 else None
        assert self._lib.ko_render(self._h, N.ptr(out), out.size,
                                   N.ptr(mix) if mix is not None else None, self.threads) == 0
        self.last_mix64 = mix
        return out

    def stats(self):
        from kestrel_b200.backend import BlockStats
        s = N.KcBlockStats()
        self._lib.ko_stats(self._h, C.byref(s))
        return BlockStats(s.active_voices, s.stolen, s.dropped, s.peak)

    def name(self):
        return "cpu-reference"

    def read_pool(self):
        st = self.stats()
        n = int(st.active_voices)
        buf = np.empty(max(n, 1) * 24, dtype=np.uint32)
        live = C.c_uint32()
        assert self._lib.ko_read_pool(self._h, N.ptr(buf), buf.size, C.byref(live)) == 0
        n = live.value
        return buf[: 24 * n].reshape(24, n).copy()

    def load_pool(self, fields: np.ndarray, stolen: int, dropped: int) -> None:
        """Take over a pool read from another backend ([24, live] u32, the
        kc_read_pool layout) with its cumulative counters."""
        f = np.ascontiguousarray(fields, dtype=np.uint32)
        assert f.ndim == 2 and f.shape[0] == 24
        assert self._lib.ko_load_pool(self._h, N.ptr(f) if f.size else None, f.shape[1], stolen, dropped) == 0
