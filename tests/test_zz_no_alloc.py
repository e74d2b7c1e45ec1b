"""kc_render_block_noalloc: the render entry point for callers that cannot allocate.

Some hosts cannot call cudaMalloc while they run -- an allocation can stall
the whole device for milliseconds, which a real-time audio callback cannot
afford, and hosts with their own device-memory arenas pass every buffer in.
This entry point renders a block of a voice pool the caller owns, keeping its
scratch in a fixed file-scope device array instead of allocating.

Each case hands it a copy of a context's pool and checks two calls in a row
against the context's own kc_render of the same block: the audio nulls below
-100 dBFS (the tolerance every parity test here uses; the two differ only in
how many warps the mix is folded over) and the surviving voices' state is
bit-identical (the context compacts dead voices away; the caller's pool keeps
them in place, marked dead). The cases cover ragged voice counts (not a
multiple of 32), voices released and dying inside the block, both mixes it
supports and every interpolation. A pool with an out-of-range gate slot and
params index must render in bounds, as slot 0 and entry 0.
This file is named so pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from kestrel_b200 import host as H
from kestrel_b200 import native as N

gpu = pytest.mark.gpu
STAGE = N.FIELD["env_stage"]


def _null_db(a, b):
    d = float(np.max(np.abs(a.astype(np.float64) - b.astype(np.float64))))
    return -np.inf if d == 0 else 20 * np.log10(d)


def _sustained_cmds(bank, n, rng, fast_release):
    L = bank.max_sample_len
    starts = np.arange(128, dtype=np.uint64) * np.uint64(L + 8)
    r = rng.integers(0, 128, n)
    cmds = np.zeros(n, N.SPAWN_DTYPE)
    cmds["smp_base"] = starts[r]
    cmds["smp_len"] = L
    cmds["loop_start"] = L - 8916
    cmds["loop_end"] = L
    cmds["flags"] = N.VF_LOOP
    cmds["region"] = r
    # params entry 0 is the bank's; entry `fast_release` (when given) is a
    # copy whose release dies within a few dozen frames.
    if fast_release is not None:
        cmds["params"] = np.where(rng.random(n) < 0.5, fast_release, 0)
    cmds["phase_hi"] = rng.integers(0, L - 9000, n)
    st = (2.0 ** rng.uniform(-0.14, 0.14, n) * 2**32).astype(np.uint64)
    cmds["step_hi"] = (st >> np.uint64(32)).astype(np.uint32)
    cmds["step_lo"] = (st & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    cmds["gate_slot"] = rng.integers(0, N.GATE_SLOTS, n)
    cmds["ordinal"] = 1
    ids = np.arange(1, n + 1, dtype=np.uint64)
    cmds["note_id_lo"] = (ids & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    cmds["gain_l"] = rng.uniform(0.001, 0.02, n).astype(np.float32)
    cmds["gain_r"] = rng.uniform(0.001, 0.02, n).astype(np.float32)
    return cmds


def _call(lib, cfg, d_pool, cap, n, d_pcm, pcm_len, d_params, params_len, d_gates, d_chan, ctrl, d_out, stream):
    return lib.kc_render_block_noalloc(C.byref(cfg), d_pool.data_ptr(), cap, n, d_pcm.data_ptr(), pcm_len,
                                       d_params.data_ptr(), params_len, 1, d_gates.data_ptr(), d_chan.data_ptr(),
                                       int(ctrl), int(ctrl), 0, d_out.data_ptr(), stream)


CASES = {
    # name: (interpolation, mix_mode, controllers, voices spawned, release some voices mid-block)
    "linear-f32": (N.INTERP_LINEAR, 0, False, 12000, False),
    "linear-f32-controllers": (N.INTERP_LINEAR, 0, True, 12000, False),
    "linear-twosum-ragged-release": (N.INTERP_LINEAR, 1, False, 12013, True),
    "nearest-f32-controllers-ragged-release": (N.INTERP_NEAREST, 0, True, 9007, True),
    "cubic-twosum-controllers-ragged-release": (N.INTERP_CUBIC, 1, True, 5001, True),
    "cubic-f32-ragged": (N.INTERP_CUBIC, 0, False, 3333, False),
}


@gpu
@pytest.mark.parametrize("name", list(CASES))
def test_noalloc_render_matches_the_context_two_calls_in_a_row(name):
    import torch

    from kestrel_b200.backend import CudaSynth

    interp, mix, controllers, n_spawn, release = CASES[name]
    lib = N.cuda_lib()
    cfg = N.default_config(max_voices=20000, sort_voices=0, interpolation=interp, mix_mode=mix)
    bank = H.Bank(H.bank_spec(presets=1), cfg)
    params = bank.params.copy()
    fast = None
    if release:
        # A second params entry whose release halves the level every frame.
        params = np.concatenate([params, params[:1]])
        fast = params.size - 1
        params[fast]["release_coef"] = 0.5
    ctx = CudaSynth(cfg, bank.pool, params, bank.regions, bank.max_sample_len)
    rng = np.random.default_rng(5 + len(name))
    tiles = cfg.block_frames // cfg.gate_frames
    chan = np.zeros((tiles, 16, 4), np.uint32)
    chan[:, :, 0] = 1 << 24
    chan[:, :, 1:3] = np.float32(1.0).view(np.uint32)
    if controllers:
        chan[:, :, 0] = np.round(2.0 ** (rng.uniform(-1, 1, (tiles, 16)) / 12.0) * (1 << 24)).astype(np.uint32)
        chan[:, :, 1] = rng.uniform(0.5, 1.2, (tiles, 16)).astype(np.float32).view(np.uint32)
        chan[:, :, 2] = rng.uniform(0.5, 1.2, (tiles, 16)).astype(np.float32).view(np.uint32)
    chan = chan.reshape(-1)
    gates0 = np.zeros(tiles * N.GATE_SLOTS, np.uint32)

    # Block 0 through the context: spawn, render, compact.
    ctx.set_gates(gates0)
    ctx.set_channels(chan, controllers, controllers, False)
    ctx.spawn(_sustained_cmds(bank, n_spawn, rng, fast))
    ctx.render()
    pool = ctx.read_pool()
    n = pool.shape[1]
    assert n == n_spawn
    cap = (n + 31) // 32 * 32

    # The caller's own device buffers (allocated by the caller, not the entry point).
    d_pool = torch.zeros((24, cap), dtype=torch.int32, device="cuda")
    d_pool[:, :n] = torch.from_numpy(pool.view(np.int32))
    d_pcm = torch.from_numpy(bank.pool).cuda()
    d_params = torch.from_numpy(params.view(np.uint8).copy()).cuda()
    d_chan = torch.from_numpy(chan.view(np.int32)).cuda()
    d_out = torch.empty(cfg.block_frames * 2, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()

    for call in range(2):
        gates = gates0.copy()
        if release and call == 0:
            # A quarter of the gate slots release from tile 40 on: their
            # fast-release voices die within the block, the others fade.
            g = gates.reshape(tiles, N.GATE_SLOTS)
            g[40:, rng.random(N.GATE_SLOTS) < 0.25] = 1
        d_gates = torch.from_numpy(gates.view(np.int32)).cuda()
        rc = _call(lib, cfg, d_pool, cap, n, d_pcm, bank.pool.size, d_params, params.size, d_gates, d_chan,
                   controllers, d_out, stream)
        assert rc == 0, lib.kc_last_error().decode()
        torch.cuda.synchronize()
        got = d_out.cpu().numpy()

        ctx.set_gates(gates)
        ctx.set_channels(chan, controllers, controllers, False)
        ctx.spawn(np.zeros(0, N.SPAWN_DTYPE))
        want = ctx.render()
        assert np.abs(want).max() > 0.1
        db = _null_db(got, want)
        assert db <= -100.0, f"{name} call {call}: null {db:.1f} dBFS"
        after = ctx.read_pool()
        mine = d_pool[:, :n].cpu().numpy().view(np.uint32)
        alive = mine[STAGE] != N.ENV_DEAD
        if release and call == 0:
            assert (~alive).sum() > 100  # voices did die inside the block
        np.testing.assert_array_equal(mine[:, alive], after, err_msg=f"{name} call {call}: voice state")
    ctx.close()


@gpu
def test_noalloc_clamps_out_of_range_indexes():
    """A caller-owned pool is not validated on the host the way kc_spawn's
    commands are: a voice with a gate slot past KC_GATE_SLOTS or a params
    index past the table must read slot 0 / entry 0, in bounds, not past the
    caller's buffers. Checked against the same pool with those indexes
    already 0: the same output bits and the same state."""
    import torch

    from kestrel_b200.backend import CudaSynth

    lib = N.cuda_lib()
    cfg = N.default_config(max_voices=4096, sort_voices=0)
    bank = H.Bank(H.bank_spec(presets=1), cfg)
    ctx = CudaSynth(cfg, bank.pool, bank.params, bank.regions, bank.max_sample_len)
    rng = np.random.default_rng(9)
    tiles = cfg.block_frames // cfg.gate_frames
    chan = np.zeros(tiles * 64, np.uint32)
    gates = np.zeros(tiles * N.GATE_SLOTS, np.uint32)
    ctx.set_gates(gates)
    ctx.set_channels(chan, False, False, False)
    cmds = _sustained_cmds(bank, 1000, rng, None)
    cmds["gate_slot"][:3] = 0
    cmds["params"][:3] = 0
    ctx.spawn(cmds)
    ctx.render()
    pool = ctx.read_pool()
    ctx.close()
    n = pool.shape[1]
    bad = pool.copy()
    bad[N.FIELD["gate_slot"], 0] = 5000          # past the 2048-word gate row
    bad[N.FIELD["gate_slot"], 1] = 0xFFFFFFFF
    bad[N.FIELD["params"], 2] = bank.params.size + 7  # past the params table
    cap = (n + 31) // 32 * 32
    d_pcm = torch.from_numpy(bank.pool).cuda()
    d_params = torch.from_numpy(bank.params.view(np.uint8).copy()).cuda()
    d_gates = torch.from_numpy(gates.view(np.int32)).cuda()
    d_chan = torch.from_numpy(chan.view(np.int32)).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    res = []
    for p in (pool, bad):
        d_pool = torch.zeros((24, cap), dtype=torch.int32, device="cuda")
        d_pool[:, :n] = torch.from_numpy(p.view(np.int32))
        d_out = torch.empty(cfg.block_frames * 2, dtype=torch.float32, device="cuda")
        rc = _call(lib, cfg, d_pool, cap, n, d_pcm, bank.pool.size, d_params, bank.params.size, d_gates, d_chan,
                   False, d_out, stream)
        assert rc == 0, lib.kc_last_error().decode()
        torch.cuda.synchronize()
        res.append((d_out.cpu().numpy(), d_pool[:, :n].cpu().numpy().view(np.uint32)))
    np.testing.assert_array_equal(res[0][0], res[1][0])
    keep = [f for f in range(24) if f not in (N.FIELD["gate_slot"], N.FIELD["params"])]
    np.testing.assert_array_equal(res[0][1][keep], res[1][1][keep])


@gpu
def test_noalloc_rejects_calls_beyond_its_scratch_and_bad_arguments():
    import torch

    lib = N.cuda_lib()
    cfg = N.default_config(max_voices=1 << 20)
    n = 40000  # over the 32,736 voices the scratch holds at block_frames 4096
    # Real buffers of the requested size: the host checks must refuse each
    # call, and nothing here would read past a buffer even if they did not.
    d_pool = torch.zeros((24, n), dtype=torch.int32, device="cuda")
    d_pcm = torch.zeros(64, dtype=torch.int16, device="cuda")
    d_params = torch.zeros(96, dtype=torch.uint8, device="cuda")
    d_gates = torch.zeros(128 * 2048, dtype=torch.int32, device="cuda")
    d_chan = torch.zeros(128 * 64 + 4, dtype=torch.int32, device="cuda")
    d_out = torch.zeros(8192, dtype=torch.float32, device="cuda")

    def call(cfg, n, params_ptr=None, chan_ptr=None):
        return lib.kc_render_block_noalloc(C.byref(cfg), d_pool.data_ptr(), n, n, d_pcm.data_ptr(), 64,
                                           params_ptr or d_params.data_ptr(), 1, 1, d_gates.data_ptr(),
                                           chan_ptr or d_chan.data_ptr(), 0, 0, 0, d_out.data_ptr(), None)

    assert call(cfg, n) == 1  # KC_ERR_INVALID
    msg = lib.kc_last_error().decode()
    assert "exceeds the no-alloc scratch" in msg and "32736" in msg
    assert call(N.default_config(mix_mode=N.MIX_F64), 64) == 1
    assert "KC_MIX_F64" in lib.kc_last_error().decode()
    assert call(N.default_config(), 64, params_ptr=d_params.data_ptr() + 4) == 1
    assert "16-byte aligned" in lib.kc_last_error().decode()
    assert call(N.default_config(), 64, chan_ptr=d_chan.data_ptr() + 8) == 1
    assert "16-byte aligned" in lib.kc_last_error().decode()
    assert call(N.default_config(steal_fade_frames=4096), 64) == 1
    assert "1..block_frames-1" in lib.kc_last_error().decode()
