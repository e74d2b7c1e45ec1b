"""The render server (include/kestrel_serve.h) from Python.

``serve`` runs a list of render jobs on one GPU, either by continuous
batching (jobs admitted by device memory while others render, one
kc_batch_render per step for every resident job) or on the plain path one job
at a time. Each job is its own seeded synthetic soundfont, MIDI stream and
backend config. ``served_jobs`` builds the batched-and-served benchmark
configuration's job mix: Poisson arrivals, log-uniform note counts, uniform
durations, voice pools of 16k-2M, 1-128 presets per soundfont.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import host as H
from . import native as N

SERVE_LIB_PATH = Path(__file__).resolve().parent / "libkestrel_serve.so"

MODE_BATCHED, MODE_SEQUENTIAL, MODE_PARALLEL = 0, 1, 2


class KsJobSpec(C.Structure):
    _fields_ = [("arrival_s", C.c_double), ("cfg", N.KcConfig), ("opt", H.KhOptions),
                ("bank", H.KhSynthBankSpec), ("midi", H.KhMidiSpec), ("max_blocks", C.c_uint64)]


BLOCK_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_uint32, C.c_uint64, C.POINTER(C.c_float), C.c_size_t)


class KsServerConfig(C.Structure):
    _fields_ = [("mode", C.c_uint32), ("device", C.c_uint32), ("max_jobs", C.c_uint32),
                ("host_threads", C.c_uint32), ("vram_budget", C.c_uint64), ("use_graph", C.c_uint32),
                ("realtime_arrivals", C.c_uint32), ("on_block", BLOCK_FN), ("user", C.c_void_p),
                ("autotune", C.c_uint32), ("device_resample", C.c_uint32), ("reserved", C.c_uint32 * 6)]


class KsJobResult(C.Structure):
    _fields_ = [("arrival_s", C.c_double), ("admit_s", C.c_double), ("first_block_s", C.c_double),
                ("done_s", C.c_double), ("setup_s", C.c_double), ("blocks", C.c_uint64),
                ("voice_samples", C.c_uint64), ("out_hash", C.c_uint64), ("device_bytes", C.c_uint64),
                ("max_live", C.c_uint32), ("peak", C.c_float), ("status", C.c_int), ("pad", C.c_uint32)]


class KsRunStats(C.Structure):
    _fields_ = [("wall_s", C.c_double), ("gpu_ms", C.c_double), ("setup_s", C.c_double),
                ("voice_samples", C.c_uint64), ("job_blocks", C.c_uint64), ("steps", C.c_uint64),
                ("peak_device_bytes", C.c_uint64), ("max_resident", C.c_uint32), ("host_threads", C.c_uint32),
                ("tuned_voices_per_lane", C.c_uint32), ("tuned_sort_radix_bits", C.c_uint32), ("tune_s", C.c_double)]


class KsTuneSpace(C.Structure):
    _fields_ = [("voices_per_lane_mask", C.c_uint32), ("radix_mask", C.c_uint32), ("block_frames", C.c_uint32 * 4),
                ("preroll_blocks", C.c_uint32), ("timed_blocks", C.c_uint32), ("reserved", C.c_uint32 * 6)]


class KsTuneResult(C.Structure):
    _fields_ = [("voices_per_lane", C.c_uint32), ("sort_radix_bits", C.c_uint32), ("block_frames", C.c_uint32),
                ("blocks", C.c_uint32), ("device_ms", C.c_double), ("voice_samples", C.c_uint64),
                ("voice_samples_per_s", C.c_double)]


SERVE_SYMBOLS = {
    "ks_server_config_default": (None, [C.POINTER(KsServerConfig)]),
    "ks_serve": (C.c_int, [C.POINTER(KsServerConfig), C.POINTER(KsJobSpec), C.c_uint32, C.POINTER(KsJobResult),
                           C.POINTER(KsRunStats)]),
    "ks_hash_block": (C.c_uint64, [C.c_uint64, C.c_void_p, C.c_size_t]),
    "ks_autotune": (C.c_int, [C.POINTER(KsJobSpec), C.POINTER(KsTuneSpace), C.POINTER(N.KcConfig),
                              C.POINTER(KsTuneResult), C.c_uint32, C.POINTER(C.c_uint32)]),
    "ks_last_error": (C.c_char_p, []),
}

_lib: C.CDLL | None = None


def lib() -> C.CDLL:
    """Load libkestrel_serve.so (which links the CUDA backend; no fallback)."""
    global _lib
    if _lib is None:
        if not SERVE_LIB_PATH.exists():
            raise RuntimeError(f"{SERVE_LIB_PATH} is not built; run `python -m kestrel_b200.build`")
        N.cuda_lib()  # the same in-tree backend the server links against
        H.lib()
        _lib = N.bind(C.CDLL(str(SERVE_LIB_PATH)), SERVE_SYMBOLS)
    return _lib


@dataclass
class JobSpec:
    cfg: N.KcConfig
    bank: H.KhSynthBankSpec
    midi: H.KhMidiSpec
    arrival_s: float = 0.0
    max_blocks: int = 0
    opt: H.KhOptions | None = None


@dataclass
class RunResult:
    jobs: list          # KsJobResult per job, in the order given
    stats: KsRunStats

    def latencies(self) -> np.ndarray:
        """Completion minus arrival per job, seconds (server clock)."""
        return np.array([r.done_s - r.arrival_s for r in self.jobs])

    def hashes(self) -> list[int]:
        return [r.out_hash for r in self.jobs]


def hash_block(h: int, out: np.ndarray) -> int:
    """The server's running output hash, one block at a time (starts at 0)."""
    out = np.ascontiguousarray(out, dtype=np.float32)
    return lib().ks_hash_block(h, out.ctypes.data, out.size)


def _spec(j: JobSpec) -> KsJobSpec:
    s = KsJobSpec()
    s.arrival_s = j.arrival_s
    s.cfg = j.cfg
    s.opt = j.opt if j.opt is not None else H.options()
    s.bank = j.bank
    s.midi = j.midi
    s.max_blocks = j.max_blocks
    return s


def autotune(job: JobSpec, voices_per_lane=(1, 2), radix_bits=(6, 8, 10), block_frames=(), preroll: int = 16,
             timed: int = 4):
    """ks_autotune: (best kc_config, [KsTuneResult per candidate]).
    block_frames lists block lengths to try; empty keeps the job's own."""
    L = lib()
    sp = KsTuneSpace()
    sp.voices_per_lane_mask = sum(1 << (v - 1) for v in voices_per_lane)
    sp.radix_mask = sum(1 << r for r in radix_bits)
    for i, bf in enumerate(block_frames):
        sp.block_frames[i] = bf
    sp.preroll_blocks = preroll
    sp.timed_blocks = timed
    best = N.KcConfig()
    cap = len(voices_per_lane) * len(radix_bits) * max(len(block_frames), 1)
    res = (KsTuneResult * cap)()
    n = C.c_uint32()
    rc = L.ks_autotune(C.byref(_spec(job)), C.byref(sp), C.byref(best), res, cap, C.byref(n))
    if rc != 0:
        raise N.KestrelError(f"status {rc}: {L.ks_last_error().decode(errors='replace')}")
    return best, [res[i] for i in range(n.value)]


def serve(jobs: list[JobSpec], mode: int = MODE_BATCHED, device: int = 0, max_jobs: int = 256,
          host_threads: int = 0, vram_budget: int = 0, use_graph: bool = True, realtime_arrivals: bool = True,
          on_block=None, autotune: bool = False, device_resample: bool = True) -> RunResult:
    """Run every job to completion; raises on a failure that stopped the
    server (a job's own failure is its result's `status`).

    on_block(job, block, out) is called from server threads for every rendered
    block (calls for one job are in order and never concurrent)."""
    L = lib()
    sc = KsServerConfig()
    L.ks_server_config_default(C.byref(sc))
    sc.mode = mode
    sc.device = device
    sc.max_jobs = max_jobs
    sc.host_threads = host_threads
    sc.vram_budget = vram_budget
    sc.use_graph = 1 if use_graph else 0
    sc.realtime_arrivals = 1 if realtime_arrivals else 0
    sc.autotune = 1 if autotune else 0
    sc.device_resample = 1 if device_resample else 0
    cb = None
    if on_block is not None:
        def _cb(_user, job, block, out, n):
            on_block(int(job), int(block), np.ctypeslib.as_array(out, shape=(n,)).copy())
        cb = BLOCK_FN(_cb)
        sc.on_block = cb
    n = len(jobs)
    specs = (KsJobSpec * max(n, 1))()
    for i, j in enumerate(jobs):
        specs[i] = _spec(j)
    results = (KsJobResult * max(n, 1))()
    stats = KsRunStats()
    rc = L.ks_serve(C.byref(sc), specs, n, results, C.byref(stats))
    del cb
    if rc != 0:
        raise N.KestrelError(f"status {rc}: {L.ks_last_error().decode(errors='replace')}")
    return RunResult([results[i] for i in range(n)], stats)


def served_jobs(n_jobs: int = 256, seed: int = 1, rate_per_s: float = 20.0, notes=(10_000, 20_000_000),
                seconds=(5.0, 300.0), pools=(16_384, 2_097_152), presets=(1, 128), max_seconds: float = 0.0,
                block_frames: int = 4096, **cfg_overrides) -> list[JobSpec]:
    """The batched-and-served configuration's job mix, seeded: Poisson
    arrivals at `rate_per_s`, per-job note counts log-uniform in `notes`,
    durations uniform in `seconds`, voice pools log-uniform in `pools`, each
    job its own synthetic soundfont of log-uniform 1-128 presets (presets
    beyond one draw their own envelope and filter generators).

    max_seconds > 0 bounds every job to that much rendered audio (its MIDI
    keeps its full length and note density; rendering stops early)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n_jobs):
        t += rng.exponential(1.0 / rate_per_s)
        n_notes = int(round(math.exp(rng.uniform(math.log(notes[0]), math.log(notes[1])))))
        dur = float(rng.uniform(*seconds))
        pool = int(round(math.exp(rng.uniform(math.log(pools[0]), math.log(pools[1])))))
        n_pre = int(round(math.exp(rng.uniform(math.log(presets[0]), math.log(presets[1])))))
        cfg = N.default_config(max_voices=pool, block_frames=block_frames, **cfg_overrides)
        bs = H.bank_spec(presets=n_pre, random_generators=1 if n_pre > 1 else 0, seed=seed * 1_000_003 + i)
        ms = H.midi_spec(notes=n_notes, seconds=dur, dur_median_s=0.150, dur_sigma=1.0,
                         program_period_s=2.0 if n_pre > 1 else 0.0, programs=n_pre,
                         seed=seed * 7_000_003 + i)
        max_blocks = 0
        if max_seconds > 0:
            max_blocks = max(1, int(math.ceil(max_seconds * cfg.sample_rate / block_frames)))
        out.append(JobSpec(cfg, bs, ms, arrival_s=t, max_blocks=max_blocks))
    return out
