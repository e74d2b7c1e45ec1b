"""Seeded synthetic inputs at the Backend boundary, for parity tests.

A scenario is a sample pool, a params table, and a sequence of blocks, each a
(spawn commands, gate rows, channel rows, flags) tuple -- exactly what
Driver::next_block hands a backend (src/driver.rs:531-594). The generator is
free to produce any *valid* input (indices in range, ordinals counting from 1
per gate slot, note ids unique and increasing), which exercises paths the
driver reaches only rarely: steals every block, loop-until-release, sample
ends, born-in-block variants, bends far from unity.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from kestrel_b200 import native as N


@dataclass
class Block:
    cmds: np.ndarray
    gates: np.ndarray
    chan: np.ndarray
    bend: bool
    gain: bool
    variant: bool
    variants: list = field(default_factory=list)  # (index, params) installed before this block


@dataclass
class Scenario:
    cfg: N.KcConfig
    pool: np.ndarray
    params: np.ndarray
    n_regions: int
    max_len: int
    blocks: list


def make_bank(rng: np.random.Generator, n_samples: int, frames: int, n_params: int, filt_frac=0.8):
    """i16 pool of sines + noise with an 8-frame guard after each sample
    (sf2.rs:583 POOL_GUARD), plus a params table with envelope rates in the
    ranges make_params produces (bank.rs:876-954)."""
    chunks, starts = [], []
    pos = 0
    for s in range(n_samples):
        t = np.arange(frames)
        f = 110.0 * 2 ** (s / 12.0) / 48000.0
        x = 0.5 * np.sin(2 * np.pi * f * t) + 0.01 * rng.standard_normal(frames)
        x = np.clip(np.round(x * 32767.0), -32768, 32767).astype(np.int16)
        starts.append(pos)
        chunks.append(x)
        chunks.append(np.zeros(8, np.int16))
        pos += frames + 8
    pool = np.concatenate(chunks)
    p = np.zeros(n_params, dtype=N.PARAMS_DTYPE)
    attack_frames = rng.uniform(0.5, 800.0, n_params).astype(np.float32)
    ar = np.where(attack_frames < 1.0, 1.0, 1.0 / attack_frames).astype(np.float32)
    hold = rng.uniform(0, 200, n_params).astype(np.float32)
    p["attack_rate"] = ar
    p["attack_end"] = (np.float32(1.0) + hold * ar).astype(np.float32)
    decay_frames = rng.uniform(50, 20000, n_params).astype(np.float32)
    p["decay_coef"] = np.power(np.float32(10.0), np.float32(-100.0) / (np.float32(20.0) * decay_frames)).astype(np.float32)
    sus = rng.choice(np.array([0.0, 0.05, 0.3, 0.5, 1.0], np.float32), n_params)
    p["sustain"] = sus
    p["decay_target"] = np.maximum(sus, np.float32(1e-5))
    rel_frames = rng.uniform(50, 20000, n_params).astype(np.float32)
    p["release_coef"] = np.power(np.float32(10.0), np.float32(-100.0) / (np.float32(20.0) * rel_frames)).astype(np.float32)
    # RBJ lowpass coefficients (bank.rs:963-979) in f32 for random cutoffs.
    fc = rng.uniform(200.0, 12000.0, n_params)
    q = rng.uniform(0.5, 4.0, n_params)
    w0 = 2 * np.pi * fc / 48000.0
    alpha = np.sin(w0) / (2 * q)
    a0 = 1 + alpha
    p["b0"] = ((1 - np.cos(w0)) * 0.5 / a0).astype(np.float32)
    p["b1"] = ((1 - np.cos(w0)) / a0).astype(np.float32)
    p["a1"] = (-2 * np.cos(w0) / a0).astype(np.float32)
    p["a2"] = ((1 - alpha) / a0).astype(np.float32)
    p["flags"] = (rng.random(n_params) < filt_frac).astype(np.uint32)
    return pool, np.array(starts, np.uint32), p


def make_scenario(seed: int = 1, *, max_voices: int = 4096, n_blocks: int = 6, spawn_per_block=(0, 3000),
                  block_frames: int = 1024, gate_frames: int = 32, n_samples: int = 12, frames: int = 6000,
                  n_params: int = 24, chan: bool = True, variants: int = 3, steal_rule=N.STEAL_QUIETEST,
                  admit_rule=N.ADMIT_LOUDEST, interpolation=N.INTERP_LINEAR, sort_voices: int = 0,
                  mix_mode=N.MIX_F32_TREE, strict_fp: int = 1, steal_percent: int = 25,
                  release_rate: float = 0.3, steps: str = "ratio", decay_curve=N.CURVE_EXPONENTIAL,
                  release_curve=N.CURVE_EXPONENTIAL, voices_per_lane: int = 0, sort_radix_bits: int = 0,
                  bend_prob: float = 1.0, unit_tile_frames: int = 0) -> Scenario:
    """steps: "ratio" (pitch ratios 2^U(-1.5, 1.5), random phase fractions),
    "unit" (every step exactly 1.0 and every phase fraction zero: the root key
    at the pool rate) or "integral" (steps of exactly 1, 2 or 3 with zero
    phase fractions). bend_prob < 1 leaves a channel's bend at exactly unity
    on the other tiles (steps keep their whole-number ratio there)."""
    rng = np.random.default_rng(seed)
    cfg = N.default_config(max_voices=max_voices, block_frames=block_frames, gate_frames=gate_frames,
                           steal_rule=steal_rule, admit_rule=admit_rule, interpolation=interpolation,
                           sort_voices=sort_voices, mix_mode=mix_mode, strict_fp=strict_fp,
                           max_steal_percent=steal_percent, max_param_variants=max(variants + 1, 1),
                           decay_curve=decay_curve, release_curve=release_curve,
                           voices_per_lane=voices_per_lane, sort_radix_bits=sort_radix_bits,
                           unit_tile_frames=unit_tile_frames)
    pool, starts, params = make_bank(rng, n_samples, frames, n_params)
    tiles = block_frames // gate_frames
    on_count = np.zeros(N.GATE_SLOTS, np.uint32)
    off_count = np.zeros(N.GATE_SLOTS, np.uint32)
    next_id = 1
    blocks = []
    for b in range(n_blocks):
        lo, hi = spawn_per_block
        n = int(rng.integers(lo, hi + 1))
        cmds = np.zeros(n, dtype=N.SPAWN_DTYPE)
        s = rng.integers(0, n_samples, n)
        cmds["smp_base"] = starts[s]
        length = rng.integers(frames // 2, frames + 1, n).astype(np.uint32)
        cmds["smp_len"] = length
        ls = (rng.random(n) * length * 0.5).astype(np.uint32)
        le = np.minimum(length, ls + 2 + (rng.random(n) * length * 0.5).astype(np.uint32))
        cmds["loop_start"] = ls
        cmds["loop_end"] = le
        mode = rng.choice(np.array([0, 1, 3], np.uint32), n, p=[0.3, 0.5, 0.2])
        cmds["flags"] = np.where(le <= ls + 1, 0, mode)
        start = (rng.random(n) ** 3 * length * 0.9).astype(np.uint32)
        edge = rng.random(n) < 0.03
        start[edge] = length[edge] - 1
        cmds["phase_hi"] = start
        cmds["phase_lo"] = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
        if steps in ("unit", "integral"):
            cmds["phase_lo"] = 0
            cmds["step_hi"] = 1 if steps == "unit" else rng.integers(1, 4, n)
            cmds["step_lo"] = 0
        else:
            ratio = 2.0 ** rng.uniform(-1.5, 1.5, n)
            st = (ratio * 2**32).astype(np.uint64)
            cmds["step_hi"] = (st >> 32).astype(np.uint32)
            cmds["step_lo"] = (st & 0xFFFFFFFF).astype(np.uint32)
        cmds["params"] = rng.integers(0, n_params, n)
        cmds["variant"] = rng.integers(0, variants + 1, n) if variants else 0
        cmds["region"] = rng.integers(0, max(n_params // 2, 1), n)
        ch = rng.integers(0, 16, n)
        key = rng.integers(0, 128, n)
        slot = (ch * 128 + key).astype(np.uint32)
        cmds["gate_slot"] = slot
        ords = np.zeros(n, np.uint32)
        for i in range(n):  # ordinals count from 1 per slot, in command order
            on_count[slot[i]] += 1
            ords[i] = on_count[slot[i]]
        cmds["ordinal"] = ords
        cmds["start_rel"] = rng.integers(0, block_frames, n)
        ids = np.arange(next_id, next_id + n, dtype=np.uint64)
        next_id += n
        cmds["note_id_lo"] = (ids & 0xFFFFFFFF).astype(np.uint32)
        cmds["note_id_hi"] = (ids >> 32).astype(np.uint32)
        g = rng.uniform(0.0, 0.2, (n, 2)).astype(np.float32)
        cmds["gain_l"] = g[:, 0]
        cmds["gain_r"] = g[:, 1]
        # Gate rows: off counts published tile by tile, each tile releasing a
        # random share of what is sounding.
        gates = np.zeros((tiles, N.GATE_SLOTS), np.uint32)
        for t in range(tiles):
            gates[t] = off_count
            sounding = on_count - off_count
            rel = (rng.random(N.GATE_SLOTS) < release_rate / tiles * 4) & (sounding > 0)
            off_count[rel] += 1
        chan_rows = np.zeros((tiles, 16, 4), np.uint32)
        bend_f = 2.0 ** (rng.uniform(-2, 2, (tiles, 16)) / 12.0)
        bend_f = np.where(rng.random((tiles, 16)) < bend_prob, bend_f, 1.0)
        chan_rows[:, :, 0] = np.round(bend_f * (1 << 24)).astype(np.uint32)
        chan_rows[:, :, 1] = rng.uniform(0.2, 1.4, (tiles, 16)).astype(np.float32).view(np.uint32)
        chan_rows[:, :, 2] = rng.uniform(0.2, 1.4, (tiles, 16)).astype(np.float32).view(np.uint32)
        chan_rows[:, :, 3] = rng.integers(0, variants + 1, (tiles, 16)) if variants else 0
        blk_variants = []
        if variants and b == 0:
            for vi in range(1, variants + 1):
                _, _, pv = make_bank(rng, 1, 16, n_params)
                blk_variants.append((vi, pv))
        on = bool(chan) and (b % 3 != 2)
        blocks.append(Block(cmds, gates.reshape(-1), chan_rows.reshape(-1), bend=on, gain=on,
                            variant=on and bool(variants), variants=blk_variants))
    return Scenario(cfg, pool, params, n_params // 2, frames, blocks)


def run(synth, sc: Scenario, collect_pool=False):
    """Drive one backend through a scenario in Driver::next_block's call
    order (src/driver.rs:531-594); return per-block outputs and stats."""
    outs, stats, pools, mixes = [], [], [], []
    for blk in sc.blocks:
        for vi, pv in blk.variants:
            synth.set_params_variant(vi, pv)
        synth.set_gates(blk.gates)
        synth.set_channels(blk.chan, blk.bend, blk.gain, blk.variant)
        synth.spawn(blk.cmds)
        outs.append(synth.render().copy())
        stats.append(synth.stats())
        mixes.append(getattr(synth, "last_mix64", None))
        if collect_pool:
            pools.append(synth.read_pool())
    return outs, stats, pools, mixes


def null_db(a: np.ndarray, ref: np.ndarray) -> float:
    """Peak absolute difference in dBFS (kestrel null, src/bin/kestrel.rs:596-646)."""
    d = float(np.max(np.abs(a.astype(np.float64) - ref.astype(np.float64)))) if a.size else 0.0
    return -np.inf if d == 0 else 20 * np.log10(d)


def pool_by_note(pool: np.ndarray) -> dict:
    ids = (pool[N.FIELD["note_hi"]].astype(np.uint64) << 32) | pool[N.FIELD["note_lo"]]
    return {int(i): pool[:, k] for k, i in enumerate(ids)}
