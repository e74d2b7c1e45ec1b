"""kc_render_block_noalloc: the render entry point for callers that cannot allocate.

Some hosts cannot call cudaMalloc while they run -- an allocation can stall
the whole device for milliseconds, which a real-time audio callback cannot
afford, and hosts with their own device-memory arenas pass every buffer in.
This entry point renders a block of a voice pool the caller owns, keeping its
scratch in a fixed file-scope device array instead of allocating.

The test hands it a copy of a context's pool and checks two calls in a row
against the context's own kc_render of the same block: the audio nulls below
-100 dBFS (the tolerance every parity test here uses; the two differ only in
how many warps the mix is folded over) and the voices' state is bit-identical.
This file is named so pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from kestrel_b200 import host as H
from kestrel_b200 import native as N

gpu = pytest.mark.gpu


def _null_db(a, b):
    d = float(np.max(np.abs(a.astype(np.float64) - b.astype(np.float64))))
    return -np.inf if d == 0 else 20 * np.log10(d)


def _sustained_cmds(bank, n, rng):
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


@gpu
@pytest.mark.parametrize("controllers", [False, True])
def test_noalloc_render_matches_the_context_two_calls_in_a_row(controllers):
    import torch

    from kestrel_b200.backend import CudaSynth

    lib = N.cuda_lib()
    cfg = N.default_config(max_voices=20000, sort_voices=0)
    bank = H.Bank(H.bank_spec(presets=1), cfg)
    ctx = CudaSynth(cfg, bank.pool, bank.params, bank.regions, bank.max_sample_len)
    rng = np.random.default_rng(5)
    tiles = cfg.block_frames // cfg.gate_frames
    gates = np.zeros(tiles * N.GATE_SLOTS, np.uint32)
    chan = np.zeros((tiles, 16, 4), np.uint32)
    chan[:, :, 0] = 1 << 24
    chan[:, :, 1:3] = np.float32(1.0).view(np.uint32)
    if controllers:
        chan[:, :, 0] = np.round(2.0 ** (rng.uniform(-1, 1, (tiles, 16)) / 12.0) * (1 << 24)).astype(np.uint32)
        chan[:, :, 1] = rng.uniform(0.5, 1.2, (tiles, 16)).astype(np.float32).view(np.uint32)
        chan[:, :, 2] = rng.uniform(0.5, 1.2, (tiles, 16)).astype(np.float32).view(np.uint32)
    chan = chan.reshape(-1)

    # Block 0 through the context: spawn, render, compact.
    ctx.set_gates(gates)
    ctx.set_channels(chan, controllers, controllers, False)
    ctx.spawn(_sustained_cmds(bank, 12000, rng))
    ctx.render()
    pool = ctx.read_pool()
    n = pool.shape[1]
    cap = (n + 31) // 32 * 32

    # The caller's own device buffers (allocated by the caller, not the entry point).
    d_pool = torch.zeros((24, cap), dtype=torch.int32, device="cuda")
    d_pool[:, :n] = torch.from_numpy(pool.view(np.int32))
    d_pcm = torch.from_numpy(bank.pool).cuda()
    d_params = torch.from_numpy(bank.params.view(np.uint8).copy()).cuda()
    d_gates = torch.from_numpy(gates.view(np.int32)).cuda()
    d_chan = torch.from_numpy(chan.view(np.int32)).cuda()
    d_out = torch.empty(cfg.block_frames * 2, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()

    for call in range(2):
        rc = lib.kc_render_block_noalloc(C.byref(cfg), d_pool.data_ptr(), cap, n, d_pcm.data_ptr(), bank.pool.size,
                                         d_params.data_ptr(), bank.params.size, 1, d_gates.data_ptr(),
                                         d_chan.data_ptr(), int(controllers), int(controllers), 0, d_out.data_ptr(),
                                         stream)
        assert rc == 0, lib.kc_last_error().decode()
        torch.cuda.synchronize()
        got = d_out.cpu().numpy()

        ctx.set_gates(gates)
        ctx.set_channels(chan, controllers, controllers, False)
        ctx.spawn(np.zeros(0, N.SPAWN_DTYPE))
        want = ctx.render()
        assert np.abs(want).max() > 0.1
        db = _null_db(got, want)
        assert db <= -100.0, f"call {call}: null {db:.1f} dBFS"
        after = ctx.read_pool()
        assert after.shape[1] == n  # sustained voices: nobody died, order kept
        np.testing.assert_array_equal(d_pool[:, :n].cpu().numpy().view(np.uint32), after,
                                      err_msg=f"call {call}: voice state")
    ctx.close()


@gpu
def test_noalloc_rejects_calls_beyond_its_scratch():
    import torch

    lib = N.cuda_lib()
    cfg = N.default_config(max_voices=1 << 20)
    n = 40000  # over the 32,736 voices the scratch holds at block_frames 4096
    # Real buffers of the requested size: the host check must refuse the call,
    # and nothing here would read past a buffer even if it did not.
    d_pool = torch.zeros((24, n), dtype=torch.int32, device="cuda")
    d_pcm = torch.zeros(64, dtype=torch.int16, device="cuda")
    d_params = torch.zeros(48, dtype=torch.uint8, device="cuda")
    d_gates = torch.zeros(128 * 2048, dtype=torch.int32, device="cuda")
    d_chan = torch.zeros(128 * 64, dtype=torch.int32, device="cuda")
    d_out = torch.zeros(8192, dtype=torch.float32, device="cuda")
    rc = lib.kc_render_block_noalloc(C.byref(cfg), d_pool.data_ptr(), n, n, d_pcm.data_ptr(), 64, d_params.data_ptr(),
                                     1, 1, d_gates.data_ptr(), d_chan.data_ptr(), 0, 0, 0, d_out.data_ptr(), None)
    assert rc == 1  # KC_ERR_INVALID
    msg = lib.kc_last_error().decode()
    assert "exceeds the no-alloc scratch" in msg and "32736" in msg
