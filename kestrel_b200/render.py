"""Render a workload to a WAV file: the reference's render loop end to end.

    python -m kestrel_b200.render --workload plain --out plain.wav [--midi FILE.mid] [--sf2 FILE.sf2]
        [--limiter brickwall|omni|off] [--format float32|pcm16] [--seconds S]
    python -m kestrel_b200.render --workload black --write-sf2 black.sf2 [--write-midi black.mid]

The loop of src/bin/kestrel.rs:311-365 around Driver::next_block
(src/driver.rs:434-642): the driver prepares the block's inputs and hands
them to the backend in the reference's call order, the backend renders, the
output stage runs (the limiter, then clamp_block, src/driver.rs:596-606) and
the block is appended to the WAV file. The backend is the CUDA one unless
the caller hands in another object with the Backend methods.

With a backend that renders asynchronously (render_begin / render_end, as
the CUDA one does) the loop is pipelined: while the device renders block n,
the host collects block n + 1's events and then runs block n's limiter and
WAV write after block n + 1 is on its way. Only admission waits for block
n, since it needs block n's active voice count. The driver and the backend
see the same calls with the same arguments as in the serial loop, so the
file is byte-identical.
"""
from __future__ import annotations

import argparse
import sys
import time
from dataclasses import dataclass

import numpy as np

from . import host as H


@dataclass
class RenderStats:
    blocks: int
    seconds: float        # audio rendered
    wall_s: float
    peak_voices: int
    clipped: int          # samples clamp_block moved
    data_bytes: int
    latency_frames: int   # the brickwall's delay
    pipelined: bool = False
    # host seconds by phase: collecting events, admission + feeding the
    # backend, waiting on the backend, limiter + WAV write
    phases: dict | None = None

    @property
    def x_realtime(self) -> float:
        return self.seconds / self.wall_s if self.wall_s > 0 else 0.0


def cuda_backend(cfg, bank: H.Bank):
    from .backend import CudaSynth
    return CudaSynth(cfg, bank.pool, bank.params, bank.regions, bank.max_sample_len)


def render_file(path, cfg, bank_spec, midi_spec, backend=cuda_backend, limiter: int = H.LIMITER_BRICKWALL,
                fmt: int = H.WAV_FLOAT32, max_seconds: float = 0.0, limiter_opts: dict | None = None,
                on_block=None, pipelined: bool | None = None, options=None) -> RenderStats:
    """Render (cfg, soundfont spec, MIDI spec or MIDI file path) into `path`
    until the stream ends or `max_seconds` of audio (0: no bound).
    `backend(cfg, bank)` makes the Backend (the CUDA one by default).
    `pipelined` (default: whenever the backend can) overlaps the host's work
    with the backend's render. `options` are the driver's kh_options."""
    bank = H.Bank(bank_spec, cfg, options)
    drv = H.Driver(cfg, bank, midi_spec)
    synth = backend(cfg, bank)
    lim = H.Limiter(limiter, cfg.sample_rate, **(limiter_opts or {}))
    wav = H.WavWriter(path, cfg.sample_rate, 2, fmt)
    max_frames = int(max_seconds * cfg.sample_rate) if max_seconds > 0 else 0
    if pipelined is None:
        pipelined = hasattr(synth, "render_begin")
    t0 = time.perf_counter()
    try:
        if pipelined:
            blocks, frames, peak_voices, phases = _pipelined(drv, synth, lim, wav, cfg, max_frames, on_block)
        else:
            blocks, frames, peak_voices, phases = _serial(drv, synth, lim, wav, cfg, max_frames, on_block)
    finally:
        data_bytes = wav.finish()
        wall = time.perf_counter() - t0
        synth.close()
        drv.close()
    return RenderStats(blocks, frames / cfg.sample_rate, wall, peak_voices, lim.clipped, data_bytes, lim.latency,
                       pipelined, phases)


def _serial(drv, synth, lim, wav, cfg, max_frames, on_block):
    """The reference's loop as written: prepare, feed, render, output, finish."""
    frames = blocks = peak_voices = 0
    while True:
        blk = drv.prepare(synth.stats().active_voices)
        H.feed(synth, blk)
        out = synth.render()
        lim.process(out)
        wav.write(out)
        if on_block:
            on_block(blocks, out)
        st = synth.stats()
        peak_voices = max(peak_voices, st.active_voices)
        frames += cfg.block_frames
        blocks += 1
        more = drv.finish(st.active_voices)
        if not more or (max_frames and frames >= max_frames):
            break
    return blocks, frames, peak_voices, None


def _pipelined(drv, synth, lim, wav, cfg, max_frames, on_block):
    """The same calls as _serial, reordered so the host overlaps the device:
    collect(n + 1) runs while block n renders, and block n's limiter and WAV
    write run while block n + 1 renders."""
    clock = time.perf_counter
    ph = {"collect": 0.0, "admit_feed": 0.0, "wait": 0.0, "output": 0.0}
    frames = blocks = peak_voices = 0
    bufs = [np.empty(cfg.block_frames * 2, np.float32) for _ in range(2)]

    def launch(live):
        t = clock()
        kb = drv.admit_raw(live)
        synth.feed_raw(kb, drv.variant_ptrs(kb))
        synth.render_begin()
        drv.advance()
        ph["admit_feed"] += clock() - t

    t = clock()
    drv.collect()
    ph["collect"] += clock() - t
    launch(synth.stats().active_voices)
    while True:
        t = clock()
        drv.collect()
        t1 = clock()
        out = synth.render_end(bufs[blocks & 1])
        t2 = clock()
        ph["collect"] += t1 - t
        ph["wait"] += t2 - t1
        st = synth.stats()
        peak_voices = max(peak_voices, st.active_voices)
        frames += cfg.block_frames
        n = blocks
        blocks += 1
        more = drv.more_after(st.active_voices)
        stop = not more or (max_frames and frames >= max_frames)
        if not stop:
            launch(st.active_voices)
        t = clock()
        lim.process(out)
        wav.write(out)
        ph["output"] += clock() - t
        if on_block:
            on_block(n, out)
        if stop:
            return blocks, frames, peak_voices, ph


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", choices=["plain", "black", "steal"], default="plain")
    ap.add_argument("--midi", default=None, help="a standard MIDI file to render instead of the workload's stream")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--sf2", default=None, help="a SoundFont 2 file to render with instead of the workload's bank")
    ap.add_argument("--out", default=None)
    ap.add_argument("--write-sf2", default=None, help="write the workload's synthetic bank as a .sf2 file and exit")
    ap.add_argument("--write-midi", default=None, help="write the workload's synthetic stream as a .mid file and exit")
    ap.add_argument("--limiter", choices=["brickwall", "omni", "off"], default="brickwall")
    ap.add_argument("--format", choices=["float32", "pcm16"], default="float32")
    ap.add_argument("--seconds", type=float, default=0.0, help="stop after this much audio (0: the whole file)")
    ap.add_argument("--serial", action="store_true", help="the reference's serial loop instead of the pipelined one")
    ap.add_argument("--no-read-ahead", action="store_true", help="read MIDI events on the driver's thread")
    args = ap.parse_args(argv)
    cfg, bs, ms = H.config_workload(args.workload, seed=args.seed)
    if args.write_sf2 or args.write_midi:
        if args.write_sf2:
            H.write_synthetic_sf2(bs, args.write_sf2)
        if args.write_midi:
            H.write_synthetic_midi(ms, args.write_midi)
        return 0
    if not args.out:
        ap.error("--out is required to render")
    if args.midi:
        ms = args.midi
    if args.sf2:
        bs = args.sf2
    mode = {"brickwall": H.LIMITER_BRICKWALL, "omni": H.LIMITER_OMNI, "off": H.LIMITER_OFF}[args.limiter]
    fmt = H.WAV_FLOAT32 if args.format == "float32" else H.WAV_PCM16
    opt = H.options(read_ahead=0 if args.no_read_ahead else 1)
    st = render_file(args.out, cfg, bs, ms, limiter=mode, fmt=fmt, max_seconds=args.seconds,
                     pipelined=False if args.serial else None, options=opt)
    print(f"{st.seconds:.2f} s rendered in {st.wall_s:.2f} s ({st.x_realtime:.2f}x realtime), {st.blocks} blocks, "
          f"peak {st.peak_voices} voices, {st.clipped} samples clipped, {st.data_bytes} bytes"
          + (", host s: " + ", ".join(f"{k} {v:.2f}" for k, v in st.phases.items()) if st.phases else ""),
          flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
