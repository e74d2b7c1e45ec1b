"""Render a workload to a WAV file: the reference's render loop end to end.

    python -m kestrel_b200.render song.mid -s bank.sf2 -o out.wav [--max-voices N] [--limiter ...] ...
    python -m kestrel_b200.render --workload plain -o plain.wav     (a seeded synthetic workload)
    python -m kestrel_b200.render --workload black --write-sf2 black.sf2 --write-midi black.mid

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
    # backend, waiting on the backend, limiter + WAV write; and how many
    # blocks were admitted and staged while the block before them rendered
    phases: dict | None = None

    @property
    def x_realtime(self) -> float:
        return self.seconds / self.wall_s if self.wall_s > 0 else 0.0


def cuda_backend(cfg, bank: H.Bank):
    from .backend import CudaSynth
    return CudaSynth(cfg, bank.pool, bank.params, bank.regions, bank.max_sample_len)


class BlockCsv:
    """`--block-csv` (src/bin/kestrel.rs:301-340): one row per block with the
    admission decision and the level it produced."""

    HEADER = "block,t,live,want,take,stolen,dropped,rms,peak,want_e,take_e\n"

    def __init__(self, path, sample_rate: int):
        self.f = open(path, "w")
        self.f.write(self.HEADER)
        self.rate = sample_rate
        self.dropped = 0

    def row(self, block: int, frames: int, adm, stolen: int, out: np.ndarray) -> None:
        """adm: (live, want, take, want_energy, take_energy) of the block."""
        live, want, take, we, te = adm
        self.dropped += want - take
        x = out.astype(np.float64)
        rms = float(np.sqrt(np.dot(x, x) / max(out.size, 1)))
        peak = float(np.max(np.abs(out))) if out.size else 0.0
        self.f.write(f"{block},{frames / self.rate:.6f},{live},{want},{take},{stolen},{self.dropped},"
                     f"{rms:.9f},{peak:.9f},{we},{te}\n")

    def close(self) -> None:
        self.f.close()


def render_file(path, cfg, bank_spec, midi_spec, backend=cuda_backend, limiter: int = H.LIMITER_BRICKWALL,
                fmt: int = H.WAV_FLOAT32, max_seconds: float = 0.0, limiter_opts: dict | None = None,
                on_block=None, pipelined: bool | None = None, options=None, block_csv=None,
                nan_guard: bool = False, progress=None) -> RenderStats:
    """Render (cfg, soundfont spec, MIDI spec or MIDI file path) into `path`
    until the stream ends or `max_seconds` of audio (0: no bound).
    `backend(cfg, bank)` makes the Backend (the CUDA one by default).
    `pipelined` (default: whenever the backend can) overlaps the host's work
    with the backend's render. `options` are the driver's kh_options;
    `block_csv` a path for the per-block diagnostic rows; `nan_guard` stops
    at the first block holding a NaN or an infinity; `progress(seconds,
    voices, x_realtime, timings)` is called about once a second."""
    bank = H.Bank(bank_spec, cfg, options)
    drv = H.Driver(cfg, bank, midi_spec)
    synth = backend(cfg, bank)
    lim = H.Limiter(limiter, cfg.sample_rate, **(limiter_opts or {}))
    wav = H.WavWriter(path, cfg.sample_rate, 2, fmt)
    max_frames = int(max_seconds * cfg.sample_rate) if max_seconds > 0 else 0
    if pipelined is None:
        pipelined = hasattr(synth, "render_begin")
    csv = BlockCsv(block_csv, cfg.sample_rate) if block_csv else None
    t0 = time.perf_counter()
    if nan_guard or progress:
        user_cb, last = on_block, [t0]

        def on_block(n, out):
            if nan_guard and not np.isfinite(out).all():
                raise FloatingPointError(f"block {n}: non-finite samples in the output")
            if progress and time.perf_counter() - last[0] > 1.0:
                last[0] = time.perf_counter()
                secs = (n + 1) * cfg.block_frames / cfg.sample_rate
                t = synth.timings() if hasattr(synth, "timings") else []
                progress(secs, synth.stats().active_voices, secs / max(last[0] - t0, 1e-9), t)
            if user_cb:
                user_cb(n, out)
    try:
        if pipelined:
            blocks, frames, peak_voices, phases = _pipelined(drv, synth, lim, wav, cfg, max_frames, on_block, csv)
        else:
            blocks, frames, peak_voices, phases = _serial(drv, synth, lim, wav, cfg, max_frames, on_block, csv)
    finally:
        if csv:
            csv.close()
        data_bytes = wav.finish()
        wall = time.perf_counter() - t0
        synth.close()
        drv.close()
    return RenderStats(blocks, frames / cfg.sample_rate, wall, peak_voices, lim.clipped, data_bytes, lim.latency,
                       pipelined, phases)


def _serial(drv, synth, lim, wav, cfg, max_frames, on_block, csv=None):
    """The reference's loop as written: prepare, feed, render, output, finish."""
    frames = blocks = peak_voices = 0
    while True:
        st0 = synth.stats()
        blk = drv.prepare(st0.active_voices)
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
        if csv:
            csv.row(blocks, frames, (blk.live, blk.want, blk.take, blk.want_energy, blk.take_energy),
                    st.stolen - st0.stolen, out)
        more = drv.finish(st.active_voices)
        if not more or (max_frames and frames >= max_frames):
            break
    return blocks, frames, peak_voices, None


def _pipelined(drv, synth, lim, wav, cfg, max_frames, on_block, csv=None):
    """The same calls as _serial, reordered so the host overlaps the device:
    collect(n + 1) runs while block n renders, and block n's limiter and WAV
    write run while block n + 1 renders. When block n + 1's admission cannot
    depend on how many voices block n leaves (every queued layer fits in what
    one block may steal), it is admitted and staged while block n renders
    too, and block n + 1 starts as soon as block n ends."""
    clock = time.perf_counter
    ph = {"collect": 0.0, "admit_feed": 0.0, "wait": 0.0, "output": 0.0, "early_blocks": 0}
    frames = blocks = peak_voices = 0
    bufs = [np.empty(cfg.block_frames * 2, np.float32) for _ in range(2)]

    adm = []   # admission of the blocks in flight, for the diagnostic rows

    def stage(live):
        t = clock()
        kb = drv.admit_raw(live)
        adm.append([kb.live, kb.want, kb.take, kb.want_energy, kb.take_energy])
        synth.feed_raw(kb, drv.variant_ptrs(kb))
        ph["admit_feed"] += clock() - t

    def launch(live):
        stage(live)
        synth.render_begin()
        drv.advance()

    t = clock()
    drv.collect()
    ph["collect"] += clock() - t
    stolen = synth.stats().stolen
    launch(synth.stats().active_voices)
    while True:
        t = clock()
        drv.collect()
        t1 = clock()
        ph["collect"] += t1 - t
        # (only for a backend whose spawn is staged until its render, so
        # that staging block n + 1 cannot touch block n's voices or stats)
        early = getattr(synth, "spawn_deferred", False) and drv.admit_ready()
        if early:
            stage(0)    # the live count is filled in below, for the diagnostic row
            ph["early_blocks"] += 1
        t1 = clock()
        out = synth.render_end(bufs[blocks & 1])
        t2 = clock()
        ph["wait"] += t2 - t1
        st = synth.stats()
        peak_voices = max(peak_voices, st.active_voices)
        frames += cfg.block_frames
        n = blocks
        blocks += 1
        more = drv.more_after(st.active_voices)
        stop = not more or (max_frames and frames >= max_frames)
        if early:
            adm[-1][0] = st.active_voices
            if not stop:
                synth.render_begin()
                drv.advance()
        elif not stop:
            launch(st.active_voices)
        t = clock()
        lim.process(out)
        wav.write(out)
        ph["output"] += clock() - t
        if on_block:
            on_block(n, out)
        if csv:
            csv.row(blocks, frames, adm.pop(0), st.stolen - stolen, out)
        stolen = st.stolen
        if stop:
            return blocks, frames, peak_voices, ph


# The spellings each option accepts (src/config.rs:20-150).
_INTERP = {"nearest": 0, "none": 0, "0": 0, "linear": 1, "1": 1, "cubic": 2, "hermite": 2, "2": 2}
_CURVE = {"exp": 0, "exponential": 0, "db": 0, "lin": 1, "linear": 1}
_STEAL = {"oldest": 0, "drop": 1, "dropnew": 1, "drop-new": 1, "quietest": 2, "quiet": 2, "level": 2}
_ADMIT = {"loudest": 0, "loud": 0, "rank": 0, "ranked": 0, "even": 1, "spread": 1, "flat": 1}


def _choice(table, name):
    def parse(v):
        key = v.lower()
        if key not in table:
            raise argparse.ArgumentTypeError(f"unknown {name} {v!r}")
        return table[key]
    return parse


def main(argv=None) -> int:
    """`kestrel render` (src/bin/kestrel.rs:72-187) with the CUDA backend:
    MIDI file, -s soundfont.sf2, -o out.wav and the options that reach the
    driver, the backend and the output stage. Without a MIDI file, a seeded
    synthetic workload stands in (--workload)."""
    ap = argparse.ArgumentParser(prog="python -m kestrel_b200.render")
    ap.add_argument("midi", nargs="?", default=None, help="input MIDI file (default: the workload's synthetic stream)")
    ap.add_argument("-s", "--soundfont", "--sf2", dest="soundfont", default=None,
                    help="SoundFont 2 file (default: the workload's synthetic bank)")
    ap.add_argument("-o", "--out", default=None, help="output WAV")
    ap.add_argument("--midi", dest="midi_opt", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--workload", choices=["plain", "black", "steal", "steal-bent"], default="plain")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--write-sf2", default=None, help="write the workload's synthetic bank as a .sf2 file and exit")
    ap.add_argument("--write-midi", default=None, help="write the workload's synthetic stream as a .mid file and exit")
    ap.add_argument("--rate", type=int, default=None, help="output sample rate (48000)")
    ap.add_argument("--block", type=int, default=None, help="frames per block (4096)")
    ap.add_argument("--gate-frames", type=int, default=None, help="frames between note-off gate checks (32)")
    ap.add_argument("--max-voices", type=int, default=None)
    ap.add_argument("--layers", type=int, default=None, help="regions a note may sound (16)")
    ap.add_argument("--interp", type=_choice(_INTERP, "interpolation"), default=None)
    ap.add_argument("--decay-curve", type=_choice(_CURVE, "curve"), default=None)
    ap.add_argument("--release-curve", type=_choice(_CURVE, "curve"), default=None)
    ap.add_argument("--steal", type=_choice(_STEAL, "steal rule"), default=None)
    ap.add_argument("--admit", type=_choice(_ADMIT, "admit rule"), default=None)
    ap.add_argument("--steal-percent", type=int, default=None)
    ap.add_argument("--format", choices=["float32", "pcm16"], default="float32")
    ap.add_argument("--volume", type=float, default=None, help="master volume (1.0)")
    ap.add_argument("--no-limiter", action="store_true")
    ap.add_argument("--limiter", choices=["brickwall", "omni", "off"], default="brickwall")
    ap.add_argument("--ceiling-db", type=float, default=0.0)
    ap.add_argument("--lookahead-ms", type=float, default=2.0)
    ap.add_argument("--limiter-release-ms", type=float, default=60.0)
    ap.add_argument("--limiter-sustain-ms", type=float, default=0.0)
    ap.add_argument("--no-true-peak", action="store_true")
    ap.add_argument("--no-filter", action="store_true")
    ap.add_argument("--no-sort", action="store_true")
    ap.add_argument("--no-resample-pool", action="store_true")
    ap.add_argument("--pool-budget", type=int, default=2048, help="sample pool budget in MiB")
    ap.add_argument("--seconds", type=float, default=0.0, help="stop after this much audio (0: the whole file)")
    ap.add_argument("--profile", action="store_true", help="log per-pass device timings with the progress line")
    ap.add_argument("--nan-guard", action="store_true", help="stop at the first block with a NaN or an infinity")
    ap.add_argument("--quiet", action="store_true", help="no progress lines")
    ap.add_argument("--block-csv", default=None, metavar="PATH",
                    help="one row per block: the admission decision and the level it produced")
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
        ap.error("-o/--out is required to render")
    midi = args.midi or args.midi_opt
    if midi:
        ms = midi
    if args.soundfont:
        bs = args.soundfont
    for field, val in (("sample_rate", args.rate), ("block_frames", args.block), ("gate_frames", args.gate_frames),
                       ("max_voices", args.max_voices), ("interpolation", args.interp),
                       ("decay_curve", args.decay_curve), ("release_curve", args.release_curve),
                       ("steal_rule", args.steal), ("admit_rule", args.admit),
                       ("max_steal_percent", args.steal_percent)):
        if val is not None:
            setattr(cfg, field, val)
    if args.no_sort:
        cfg.sort_voices = 0
    opt = H.options(read_ahead=0 if args.no_read_ahead else 1, filter_enabled=0 if args.no_filter else 1,
                    resample_pool=0 if args.no_resample_pool else 1, sample_pool_budget=args.pool_budget << 20)
    if args.layers is not None:
        opt.max_layers = args.layers
    if args.volume is not None:
        opt.master_volume = args.volume
    mode = H.LIMITER_OFF if args.no_limiter else \
        {"brickwall": H.LIMITER_BRICKWALL, "omni": H.LIMITER_OMNI, "off": H.LIMITER_OFF}[args.limiter]
    fmt = H.WAV_FLOAT32 if args.format == "float32" else H.WAV_PCM16
    lim_opts = dict(ceiling_db=args.ceiling_db, lookahead_ms=args.lookahead_ms, release_ms=args.limiter_release_ms,
                    sustain_ms=args.limiter_sustain_ms, true_peak=not args.no_true_peak)
    def progress(secs, voices, xrt, timings):
        print(f"{secs:8.2f}s rendered | {voices:10d} voices | {xrt:.2f}x realtime", file=sys.stderr, flush=True)
        if args.profile and timings:
            print("  passes: " + "  ".join(f"{n} {ms:.3f}ms" for n, ms in timings), file=sys.stderr, flush=True)

    def backend(cfg, bank):
        s = cuda_backend(cfg, bank)
        if args.profile:
            s.set_profile(True)
        return s

    st = render_file(args.out, cfg, bs, ms, backend=backend, limiter=mode, fmt=fmt, max_seconds=args.seconds,
                     pipelined=False if args.serial else None, options=opt, limiter_opts=lim_opts,
                     block_csv=args.block_csv, nan_guard=args.nan_guard, progress=None if args.quiet else progress)
    print(f"{st.seconds:.2f} s rendered in {st.wall_s:.2f} s ({st.x_realtime:.2f}x realtime), {st.blocks} blocks, "
          f"peak {st.peak_voices} voices, {st.clipped} samples clipped, {st.data_bytes} bytes"
          + (", host s: " + ", ".join(f"{k} {v:.2f}" for k, v in st.phases.items() if k != "early_blocks")
             + f", {st.phases['early_blocks']} blocks staged early" if st.phases else ""),
          flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
