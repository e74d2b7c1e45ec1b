"""The pool sort's order: region, envelope stage, predicted coarse phase.

The reference packs region, stage and a coarsened phase into 32 bits
(SortKeyLayout::plan, src/gpu/mod.rs:77-105). The CUDA backend keeps that
layout and fills the phase field with the phase each voice is predicted to
reach halfway through the next block: phase + base step x the channel's bend
at the block's last gate tile x half a block, wrapped into a looping voice's
loop and clamped to the field. After a sorted block the live pool read back
must be in that order, restated here; the order is what the render's locality
depends on (the live set and every voice's state are checked against the
oracle elsewhere, as a multiset when the sort is on).
"""
import numpy as np
import pytest

from kestrel_b200 import native as N

from scenarios import make_scenario, run

gpu = pytest.mark.gpu
F = N.FIELD


def layout(n_regions: int, max_len: int, block_frames: int) -> dict:
    dead = max(n_regions, 1)
    region_bits = dead.bit_length()
    len_bits = max(max_len, 1).bit_length()
    phase_bits = min(32 - (region_bits + 3), len_bits)
    return dict(dead=dead, phase_shift=max(len_bits - phase_bits, 0), phase_bits=phase_bits,
                stage_shift=phase_bits, region_shift=phase_bits + 3, half=block_frames // 2)


def predicted_phase(pool: np.ndarray, L: dict, chan_rows: np.ndarray | None) -> np.ndarray:
    u64 = np.uint64
    ph = pool[F["phase_hi"]].astype(u64)
    step = (pool[F["step_hi"]].astype(u64) << u64(32)) | pool[F["step_lo"]].astype(u64)
    adv = np.minimum((step >> u64(16)) * u64(L["half"]), u64(1 << 36))
    if chan_rows is not None:
        ch = (pool[F["gate_slot"]] >> 7) & 15
        bend = chan_rows[-1, ch, 0].astype(u64)
        adv = ((adv >> u64(8)) * bend) >> u64(16)
    p = ph + (adv >> u64(16))
    ls, le = pool[F["loop_start"]].astype(u64), pool[F["loop_end"]].astype(u64)
    wrap = ((pool[F["flags"]] & N.VF_LOOP) != 0) & (le > ls + u64(1)) & (p >= le)
    p[wrap] = ls[wrap] + (p[wrap] - ls[wrap]) % (le[wrap] - ls[wrap])
    top = (((1 << L["phase_bits"]) - 1) << L["phase_shift"]) | ((1 << L["phase_shift"]) - 1)
    return np.minimum(p, u64(top))


def keys(pool: np.ndarray, L: dict, chan_rows: np.ndarray | None) -> np.ndarray:
    stage = pool[F["env_stage"]]
    region = np.where(stage == N.ENV_DEAD, L["dead"], np.minimum(pool[F["region"]], L["dead"] - 1)).astype(np.uint64)
    ph = (predicted_phase(pool, L, chan_rows) >> np.uint64(L["phase_shift"])) & np.uint64((1 << L["phase_bits"]) - 1)
    return ((region << np.uint64(L["region_shift"])) | (np.minimum(stage, 7).astype(np.uint64) << np.uint64(L["stage_shift"]))
            | ph)


def test_prediction_wraps_into_the_loop_and_clamps():
    L = layout(4, 1000, 512)           # 3 + 3 + 10 bits, half a block = 256 frames
    pool = np.zeros((24, 4), np.uint32)
    pool[F["step_hi"]] = [1, 1, 2, 1]
    pool[F["step_lo"]] = [0, 0, 0, 1 << 31]
    pool[F["phase_hi"]] = [100, 900, 900, 900]
    pool[F["loop_start"]] = [0, 500, 500, 0]
    pool[F["loop_end"]] = [1000, 1000, 1000, 1000]
    pool[F["flags"]] = [N.VF_LOOP, N.VF_LOOP, N.VF_LOOP, 0]
    p = predicted_phase(pool, L, None)
    # 100 + 256; 900 + 256 wraps to 500 + 156; 900 + 512 to 500 + 412; 900 + 384 clamps at 1023
    assert list(p) == [356, 656, 912, 1023]
    rows = np.zeros((8, 16, 4), np.uint32)
    rows[-1, :, 0] = 1 << 25            # bend x2 on the last tile
    assert predicted_phase(pool[:, :1], L, rows)[0] == 100 + 512


@gpu
@pytest.mark.parametrize("seed", [31, 32])
def test_sorted_pool_is_in_key_order(seed):
    from kestrel_b200.backend import CudaSynth

    sc = make_scenario(seed=seed, sort_voices=1, n_blocks=4, spawn_per_block=(2000, 3000))
    L = layout(sc.n_regions, sc.max_len, sc.cfg.block_frames)
    tiles = sc.cfg.block_frames // sc.cfg.gate_frames
    with CudaSynth(sc.cfg, sc.pool, sc.params, sc.n_regions, sc.max_len) as s:
        _, _, pools, _ = run(s, sc, collect_pool=True)
    for blk, pool in zip(sc.blocks, pools):
        assert pool.shape[1] > 1000
        rows = blk.chan.reshape(tiles, 16, 4) if blk.bend else None
        k = keys(pool, L, rows)
        assert np.all(np.diff(k.astype(np.int64)) >= 0), "pool not in (region, stage, predicted phase) order"
        # the prediction moved voices: the current phase alone is not this order
        cur = keys(pool, dict(L, half=0), None)
        assert np.any(np.diff(cur.astype(np.int64)) < 0)
