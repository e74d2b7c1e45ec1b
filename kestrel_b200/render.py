"""Render a workload to a WAV file: the reference's render loop end to end.

    python -m kestrel_b200.render --workload plain --out plain.wav [--midi FILE.mid]
        [--limiter brickwall|omni|off] [--format float32|pcm16] [--seconds S]

The loop of src/bin/kestrel.rs:311-365 around Driver::next_block
(src/driver.rs:434-642): the driver prepares the block's inputs and hands
them to the backend in the reference's call order, the backend renders, the
output stage runs (the limiter, then clamp_block, src/driver.rs:596-606) and
the block is appended to the WAV file. The backend is the CUDA one unless
the caller hands in another object with the Backend methods.
"""
from __future__ import annotations

import argparse
import sys
import time
from dataclasses import dataclass


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

    @property
    def x_realtime(self) -> float:
        return self.seconds / self.wall_s if self.wall_s > 0 else 0.0


def cuda_backend(cfg, bank: H.Bank):
    from .backend import CudaSynth
    return CudaSynth(cfg, bank.pool, bank.params, bank.regions, bank.max_sample_len)


def render_file(path, cfg, bank_spec, midi_spec, backend=cuda_backend, limiter: int = H.LIMITER_BRICKWALL,
                fmt: int = H.WAV_FLOAT32, max_seconds: float = 0.0, limiter_opts: dict | None = None,
                on_block=None) -> RenderStats:
    """Render (cfg, soundfont spec, MIDI spec or MIDI file path) into `path`
    until the stream ends or `max_seconds` of audio (0: no bound).
    `backend(cfg, bank)` makes the Backend (the CUDA one by default)."""
    bank = H.Bank(bank_spec, cfg)
    drv = H.Driver(cfg, bank, midi_spec)
    synth = backend(cfg, bank)
    lim = H.Limiter(limiter, cfg.sample_rate, **(limiter_opts or {}))
    wav = H.WavWriter(path, cfg.sample_rate, 2, fmt)
    max_frames = int(max_seconds * cfg.sample_rate) if max_seconds > 0 else 0
    frames = blocks = peak_voices = 0
    t0 = time.perf_counter()
    try:
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
    finally:
        data_bytes = wav.finish()
        wall = time.perf_counter() - t0
        synth.close()
        drv.close()
    return RenderStats(blocks, frames / cfg.sample_rate, wall, peak_voices, lim.clipped, data_bytes, lim.latency)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", choices=["plain", "black", "steal"], default="plain")
    ap.add_argument("--midi", default=None, help="a standard MIDI file to render instead of the workload's stream")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--out", required=True)
    ap.add_argument("--limiter", choices=["brickwall", "omni", "off"], default="brickwall")
    ap.add_argument("--format", choices=["float32", "pcm16"], default="float32")
    ap.add_argument("--seconds", type=float, default=0.0, help="stop after this much audio (0: the whole file)")
    args = ap.parse_args(argv)
    cfg, bs, ms = H.config_workload(args.workload, seed=args.seed)
    if args.midi:
        ms = args.midi
    mode = {"brickwall": H.LIMITER_BRICKWALL, "omni": H.LIMITER_OMNI, "off": H.LIMITER_OFF}[args.limiter]
    fmt = H.WAV_FLOAT32 if args.format == "float32" else H.WAV_PCM16
    st = render_file(args.out, cfg, bs, ms, limiter=mode, fmt=fmt, max_seconds=args.seconds)
    print(f"{st.seconds:.2f} s rendered in {st.wall_s:.2f} s ({st.x_realtime:.2f}x realtime), {st.blocks} blocks, "
          f"peak {st.peak_voices} voices, {st.clipped} samples clipped, {st.data_bytes} bytes", flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
