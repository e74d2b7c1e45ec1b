"""A fixed synthetic pool for profiling the render pass.

    python -m kestrel_b200.profile_case --voices 262144 --blocks 3 [--sort 1] [--strict 1] [--chan 0]

Builds the plain workload's bank (128 looped 35,666-frame samples at 48 kHz),
spawns `voices` sustained looping voices in the first block (random region,
phase and a pitch within +-10% of unity, so the interpolation is exercised),
then renders `blocks` blocks with per-pass CUDA-event timing and prints the
render rate. Used as the small case for ncu captures (one render launch per
block; capture with -k regex:k_render -s 1 -c 1) and for quick rate probes.
"""
from __future__ import annotations

import argparse
import sys

import numpy as np

from . import host as H
from . import native as N
from .backend import CudaSynth


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--voices", type=int, default=262144)
    ap.add_argument("--blocks", type=int, default=3)
    ap.add_argument("--sort", type=int, default=1)
    ap.add_argument("--strict", type=int, default=1)
    ap.add_argument("--chan", type=int, default=0)
    ap.add_argument("--unity", type=int, default=0, help="1: every voice at exactly unity step")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--vpl", type=int, default=0, help="voices per lane (0 = default)")
    ap.add_argument("--tile", type=int, default=0, help="longest hot tile in frames: 16, 32 or 0 = per block")
    args = ap.parse_args(argv)

    nv = args.voices
    cfg = N.default_config(max_voices=nv, sort_voices=args.sort, strict_fp=args.strict, voices_per_lane=args.vpl,
                           unit_tile_frames=args.tile)
    bank = H.Bank(H.bank_spec(presets=1), cfg)
    rng = np.random.default_rng(args.seed)
    params = bank.params.copy()
    s = CudaSynth(cfg, bank.pool, params, bank.regions, bank.max_sample_len)
    s.set_profile(True)
    tiles = cfg.block_frames // cfg.gate_frames
    s.set_gates(np.zeros(tiles * N.GATE_SLOTS, np.uint32))
    ch = np.zeros((tiles, 16, 4), np.uint32)
    ch[:, :, 0] = 1 << 24
    ch[:, :, 1:3] = np.float32(1.0).view(np.uint32)
    if args.chan:
        ch[:, :, 0] = np.round(2.0 ** (rng.uniform(-1, 1, (tiles, 16)) / 12.0) * (1 << 24)).astype(np.uint32)
    s.set_channels(ch.reshape(-1), bool(args.chan), bool(args.chan), False)
    # Sustained voices: the driver never releases them (gate rows stay 0).
    starts = np.array([0] + [int(x) for x in np.cumsum([bank.max_sample_len + 8] * 127)], np.uint64)
    cmds = np.zeros(nv, N.SPAWN_DTYPE)
    r = rng.integers(0, 128, nv)
    L = bank.max_sample_len
    cmds["smp_base"] = starts[r]
    cmds["smp_len"] = L
    cmds["loop_start"] = L - int(round(8192 * 48000 / 44100))
    cmds["loop_end"] = L
    cmds["flags"] = N.VF_LOOP
    cmds["params"] = 0
    cmds["region"] = r
    cmds["phase_hi"] = rng.integers(0, L - 9000, nv)
    if args.unity:
        cmds["step_hi"] = 1
    else:
        st = (2.0 ** rng.uniform(-0.14, 0.14, nv) * 2**32).astype(np.uint64)
        cmds["step_hi"] = (st >> np.uint64(32)).astype(np.uint32)
        cmds["step_lo"] = (st & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    cmds["gate_slot"] = rng.integers(0, N.GATE_SLOTS, nv)
    cmds["ordinal"] = 1
    ids = np.arange(1, nv + 1, dtype=np.uint64)
    cmds["note_id_lo"] = (ids & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    cmds["gain_l"] = 0.01
    cmds["gain_r"] = 0.01
    out = np.empty(cfg.block_frames * 2, np.float32)
    for b in range(args.blocks):
        s.spawn(cmds if b == 0 else cmds[:0])
        s.render(out)
        t = dict(s.timings())
        live = s.stats().active_voices
        rate = live * cfg.block_frames / (t["render"] * 1e-3) if t.get("render") else 0.0
        print(f"vpl={args.vpl} tile={args.tile} strict={args.strict} chan={args.chan} unity={args.unity} block {b}: live {live} render {t.get('render', 0):.3f} ms "
              f"({rate:.3e} voice-frames/s) " + " ".join(f"{k}={v:.3f}" for k, v in t.items()), flush=True)
    s.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
