"""The C++ oracle against an independent Python restatement of src/cpu.rs.

Two restatements of the same reference file, written separately, driven by
the same seeded Backend-boundary inputs, must agree bit for bit: the f64 mix
(same voice order, same f32 terms), the f32 block, every pool field, and the
steal/drop counters. Small sizes only -- the Python side is loops.
"""
import numpy as np
import pytest

from kestrel_b200 import native as N
from oracle.binding import OracleSynth
from pyref import PyCpuSynth
from scenarios import make_scenario

CASES = {
    "quietest-linear-chan": dict(seed=21),
    "oldest-even": dict(seed=22, steal_rule=N.STEAL_OLDEST, admit_rule=N.ADMIT_EVEN),
    "dropnew": dict(seed=23, steal_rule=N.STEAL_DROP_NEW),
    "nearest": dict(seed=24, interpolation=N.INTERP_NEAREST),
    "cubic": dict(seed=25, interpolation=N.INTERP_CUBIC),
    "linear-curves": dict(seed=26, decay_curve=N.CURVE_LINEAR, release_curve=N.CURVE_LINEAR),
}


@pytest.mark.parametrize("name", list(CASES))
def test_oracle_matches_python_restatement(name):
    sc = make_scenario(max_voices=48, n_blocks=4, spawn_per_block=(0, 40), block_frames=256, n_samples=4,
                       frames=1500, n_params=6, **CASES[name])
    orc = OracleSynth(sc.cfg, sc.pool, sc.params)
    py = PyCpuSynth(sc.cfg, sc.pool, sc.params)
    for b, blk in enumerate(sc.blocks):
        for vi, pv in blk.variants:
            orc.set_params_variant(vi, pv)
            py.set_params_variant(vi, pv)
        for s in (orc, py):
            s.set_gates(blk.gates)
            s.set_channels(blk.chan, blk.bend, blk.gain, blk.variant)
            s.spawn(blk.cmds)
        out_o = orc.render()
        out_p, mix_p = py.render()
        np.testing.assert_array_equal(orc.last_mix64, mix_p, err_msg=f"{name} block {b} mix")
        np.testing.assert_array_equal(out_o, out_p, err_msg=f"{name} block {b} out")
        po, pp = orc.read_pool(), py.read_pool()
        keep = [i for i in range(24) if i != N.FIELD["region"]]
        np.testing.assert_array_equal(po[keep], pp[keep], err_msg=f"{name} block {b} pool")
        st = orc.stats()
        assert (st.stolen, st.dropped) == (py.stolen, py.dropped)


def test_instant_envelope_renders_exactly_the_sample():
    """testkit::simple_sf2 (src/testkit.rs:318-348): a looped sine with an
    instant envelope renders to exactly the sample at unity step. Known answer:
    out[f] = sample[f] / 32767 * gain on both channels, bit for bit."""
    n = 2000
    t = np.arange(n)
    smp = np.round(np.sin(2 * np.pi * t / 100.0) * 0.5 * 32767).astype(np.int16)
    pool = np.concatenate([smp, np.zeros(8, np.int16)])
    p = np.zeros(1, N.PARAMS_DTYPE)
    # make_params for attack/decay -12000 tc, sustain 0 cB, release -12000 tc
    # (bank.rs:876-954): instant attack, one-frame decay to full sustain.
    p["attack_rate"], p["attack_end"] = 1.0, 1.0
    p["decay_coef"] = np.float32(10.0) ** np.float32(-100.0 / 20.0)
    p["decay_target"], p["sustain"] = 1.0, 1.0
    p["release_coef"] = np.float32(10.0) ** np.float32(-100.0 / 20.0)
    p["b0"] = 1.0
    cfg = N.default_config(max_voices=4, block_frames=512)
    cmd = np.zeros(1, N.SPAWN_DTYPE)
    cmd["step_hi"] = 1
    cmd["smp_len"] = n
    cmd["loop_start"], cmd["loop_end"], cmd["flags"] = 0, n, 1
    cmd["gate_slot"], cmd["ordinal"], cmd["note_id_lo"] = 60, 1, 1
    g = np.float32(np.cos(np.float32(np.pi / 4)))
    cmd["gain_l"], cmd["gain_r"] = g, g
    orc = OracleSynth(cfg, pool, p)
    orc.set_gates(np.zeros(16 * 2048, np.uint32))
    orc.set_channels(np.zeros(16 * 64, np.uint32), False, False, False)
    orc.spawn(cmd)
    got = []
    for _ in range(3):
        got.append(orc.render().copy())
        orc.spawn(cmd[:0])
    out = np.concatenate(got).reshape(-1, 2)
    frames = np.arange(out.shape[0]) % n
    want = np.maximum(smp[frames].astype(np.float32) * np.float32(1.0 / 32767.0), np.float32(-1.0)) * g
    np.testing.assert_array_equal(out[:, 0], want)
    np.testing.assert_array_equal(out[:, 1], want)
