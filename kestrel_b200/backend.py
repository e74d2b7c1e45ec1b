"""CudaSynth: the Backend trait (src/backend.rs:22-58) over the CUDA library.

Method names, argument meaning and error behaviour mirror the reference trait
so a test reads like the reference's own: ``set_gates``, ``set_channels``,
``set_params_variant``, ``spawn``, ``render``, ``stats``, ``name``,
``timings``. Failures raise ``KestrelError`` carrying the library's message
(the reference returns ``anyhow::Result``).

This class only marshals arguments; every pass of the block runs in
libkestrel_cuda.so on the GPU. Constructing it without the built library, or
without a CUDA device, raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import native as N


@dataclass
class BlockStats:
    """backend::BlockStats (src/backend.rs:11-20)."""
    active_voices: int
    stolen: int
    dropped: int
    peak: float


class CudaSynth:
    # kc_spawn only stages the commands: the steal, drop and admission happen
    # on the device in the next render, so a block's inputs may be staged
    # while the previous block renders without touching its voices or stats.
    spawn_deferred = True

    def __init__(self, cfg: N.KcConfig, pool: np.ndarray, params: np.ndarray, n_regions: int,
                 max_sample_len: int):
        self._lib = N.cuda_lib()
        self.cfg = cfg
        pool = np.ascontiguousarray(pool, dtype=np.int16)
        params = np.ascontiguousarray(params, dtype=N.PARAMS_DTYPE)
        h = C.c_void_p()
        N.check(self._lib.kc_synth_create(C.byref(cfg), N.ptr(pool) if pool.size else None, pool.size,
                                          N.ptr(params), params.size, n_regions, max_sample_len,
                                          C.byref(h)), self._lib)
        self._h = h
        self.block_frames = cfg.block_frames
        self.tiles = cfg.block_frames // cfg.gate_frames
        self.params_per = params.size

    def clone(self, cfg: N.KcConfig | None = None) -> "CudaSynth":
        """A second context in this one's exact state (kc_synth_clone), or
        with other tunables -- voices_per_lane, sort_radix_bits -- when `cfg`
        is given (kc_synth_clone_config)."""
        h = C.c_void_p()
        if cfg is None:
            N.check(self._lib.kc_synth_clone(self._h, C.byref(h)), self._lib)
        else:
            N.check(self._lib.kc_synth_clone_config(self._h, C.byref(cfg), C.byref(h)), self._lib)
        other = object.__new__(CudaSynth)
        other._lib = self._lib
        other.cfg = cfg if cfg is not None else self.cfg
        other._h = h
        other.block_frames = self.block_frames
        other.tiles = self.tiles
        other.params_per = self.params_per
        return other

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.kc_synth_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- Backend trait -------------------------------------------------------
    def set_gates(self, rows: np.ndarray) -> None:
        rows = np.ascontiguousarray(rows, dtype=np.uint32)
        N.check(self._lib.kc_set_gates(self._h, N.ptr(rows), rows.size), self._lib)

    def set_channels(self, rows: np.ndarray, bend: bool, gain: bool, variant: bool) -> None:
        rows = np.ascontiguousarray(rows, dtype=np.uint32)
        N.check(self._lib.kc_set_channels(self._h, N.ptr(rows), rows.size, int(bend), int(gain),
                                          int(variant)), self._lib)

    def set_params_variant(self, index: int, data: np.ndarray) -> None:
        data = np.ascontiguousarray(data, dtype=N.PARAMS_DTYPE)
        N.check(self._lib.kc_set_params_variant(self._h, index, N.ptr(data), data.size), self._lib)

    def spawn(self, cmds: np.ndarray) -> None:
        cmds = np.ascontiguousarray(cmds, dtype=N.SPAWN_DTYPE)
        N.check(self._lib.kc_spawn(self._h, N.ptr(cmds) if cmds.size else None, cmds.size), self._lib)

    def render(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty(self.block_frames * 2, dtype=np.float32)
        N.check(self._lib.kc_render(self._h, N.ptr(out), out.size), self._lib)
        return out

    def feed_raw(self, blk, variants) -> None:
        """feed() from a driver block's own buffers (a KhBlock and its
        (index, address, entries) variants), with no copies on this side."""
        lib, h = self._lib, self._h
        for idx, addr, n in variants:
            N.check(lib.kc_set_params_variant(h, idx, addr, n), lib)
        N.check(lib.kc_set_gates(h, C.cast(blk.gates, C.c_void_p), blk.n_gates), lib)
        N.check(lib.kc_set_channels(h, C.cast(blk.chan, C.c_void_p), blk.n_chan, blk.bend, blk.gain, blk.variant),
                lib)
        N.check(lib.kc_spawn(h, blk.cmds if blk.n_cmds else None, blk.n_cmds), lib)

    def render_begin(self) -> None:
        """Enqueue the staged block and return; render_end collects it."""
        N.check(self._lib.kc_render_begin(self._h), self._lib)

    def render_end(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty(self.block_frames * 2, dtype=np.float32)
        N.check(self._lib.kc_render_end(self._h, N.ptr(out), out.size), self._lib)
        return out

    @property
    def pending(self) -> bool:
        return bool(self._lib.kc_render_pending(self._h))

    def stats(self) -> BlockStats:
        s = N.KcBlockStats()
        N.check(self._lib.kc_stats(self._h, C.byref(s)), self._lib)
        return BlockStats(s.active_voices, s.stolen, s.dropped, s.peak)

    def name(self) -> str:
        return self._lib.kc_name(self._h).decode()

    def set_profile(self, on: bool) -> None:
        N.check(self._lib.kc_set_profile(self._h, int(on)), self._lib)

    def timings(self) -> list[tuple[str, float]]:
        names = (C.c_char_p * 8)()
        ms = (C.c_double * 8)()
        n = C.c_size_t()
        N.check(self._lib.kc_timings(self._h, names, ms, 8, C.byref(n)), self._lib)
        return [(names[i].decode(), ms[i]) for i in range(n.value)]

    def timings_total(self) -> tuple[dict, int]:
        """Per-pass milliseconds summed over all profiled blocks, and their count."""
        ms = (C.c_double * 8)()
        nb = C.c_uint64()
        N.check(self._lib.kc_timings_total(self._h, ms, 8, C.byref(nb)), self._lib)
        names = ["steal", "spawn", "render", "reduce", "compact"]
        return {k: ms[i] for i, k in enumerate(names)}, nb.value

    # ---- device-resident form and inspection --------------------------------
    def enqueue_block_device(self, d_gates: int, d_chan: int, bend: bool, gain: bool, variant: bool,
                             d_cmds: int, n_cmds: int, d_out: int) -> None:
        N.check(self._lib.kc_enqueue_block_device(self._h, d_gates, d_chan, int(bend), int(gain),
                                                  int(variant), d_cmds or None, n_cmds, d_out),
                self._lib)

    def synchronize(self) -> None:
        N.check(self._lib.kc_synchronize(self._h), self._lib)

    def stream(self) -> int:
        return self._lib.kc_stream(self._h)

    def block_launches(self) -> int:
        n = C.c_uint32()
        N.check(self._lib.kc_block_launches(self._h, C.byref(n)), self._lib)
        return n.value

    def read_pool(self) -> np.ndarray:
        """The live voice pool as a (24, live) u32 array, field-major."""
        st = self.stats()
        cap = max(int(st.active_voices), 1) * 24 + 24 * 1024
        buf = np.empty(cap, dtype=np.uint32)
        live = C.c_uint32()
        N.check(self._lib.kc_read_pool(self._h, N.ptr(buf), buf.size, C.byref(live)), self._lib)
        n = live.value
        return buf[: 24 * n].reshape(24, n).copy()

    def device_bytes(self) -> int:
        """Device memory this context holds (kc_synth_device_bytes)."""
        return int(self._lib.kc_synth_device_bytes(self._h))

    def last_block_voices(self) -> int:
        """Voices the last block rendered (live before spawn + admitted)."""
        n = C.c_uint32()
        N.check(self._lib.kc_last_block_voices(self._h, C.byref(n)), self._lib)
        return n.value

    def launches_total(self) -> int:
        """Kernel launches this context's blocks have enqueued so far."""
        n = C.c_uint64()
        N.check(self._lib.kc_launches_total(self._h, C.byref(n)), self._lib)
        return n.value

    def last_block_tiles(self) -> tuple[int, int]:
        """(hot-path warp-tiles -- unit, integral or fractional step -- and all
        warp-tiles) of the last block."""
        u, a = C.c_uint32(), C.c_uint32()
        N.check(self._lib.kc_last_block_tiles(self._h, C.byref(u), C.byref(a)), self._lib)
        return u.value, a.value


class CudaBatch:
    """One block of many contexts per call (kc_batch_render).

    Each job is a CudaSynth whose inputs were set with set_gates /
    set_channels / spawn, exactly as before CudaSynth.render; after
    render(jobs) every job's output, state and stats are those of rendering it
    alone.
    """

    def __init__(self, cfg: N.KcBatchConfig):
        self._lib = N.cuda_lib()
        self.cfg = cfg
        h = C.c_void_p()
        N.check(self._lib.kc_batch_create(C.byref(cfg), C.byref(h)), self._lib)
        self._h = h
        self.block_frames = cfg.block_frames

    @classmethod
    def for_config(cls, cfg: N.KcConfig, max_jobs: int = 256, use_graph: bool = True) -> "CudaBatch":
        return cls(N.batch_config_for(cfg, max_jobs, use_graph))

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.kc_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def render(self, jobs: list[CudaSynth], outs: list[np.ndarray] | None = None) -> list[np.ndarray]:
        n = len(jobs)
        if outs is None:
            outs = [np.empty(self.block_frames * 2, dtype=np.float32) for _ in range(n)]
        hs = (C.c_void_p * max(n, 1))(*[j._h.value for j in jobs])
        ps = (C.c_void_p * max(n, 1))(*[N.ptr(o) for o in outs])
        N.check(self._lib.kc_batch_render(self._h, hs, n, ps), self._lib)
        return outs

    def last_ms(self) -> float:
        ms = C.c_float()
        N.check(self._lib.kc_batch_last_ms(self._h, C.byref(ms)), self._lib)
        return ms.value
