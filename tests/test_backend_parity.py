"""Parity of the CUDA backend with the CPU oracle at the Backend boundary.

Both backends are driven through identical calls (set_params_variant,
set_gates, set_channels, spawn, render -- src/driver.rs:531-594 order) on
seeded scenarios, and compared:

* integer state bit-exact: phase, stage, envelope level bits, the steal set
  (stop_rel), spawn slots, compaction order (parity mode), counters;
* with strict rounding, every float field of the pool bit-exact too;
* audio: peak null against the oracle's f64 mix below -100 dBFS
  (the reference's null criterion, README.md:37-38) at these sizes.
"""
import numpy as np
import pytest

from kestrel_b200 import native as N
from scenarios import make_scenario, null_db, pool_by_note, run

gpu = pytest.mark.gpu


def _pair(sc):
    from kestrel_b200.backend import CudaSynth
    from oracle.binding import OracleSynth
    cu = CudaSynth(sc.cfg, sc.pool, sc.params, sc.n_regions, sc.max_len)
    orc = OracleSynth(sc.cfg, sc.pool, sc.params)
    return cu, orc


def _compare(sc, exact_pool=True, sorted_pool=False, null_limit=-100.0):
    cu, orc = _pair(sc)
    o_c, s_c, p_c, _ = run(cu, sc, collect_pool=True)
    o_o, s_o, p_o, m_o = run(orc, sc, collect_pool=True)
    for b in range(len(sc.blocks)):
        assert (s_c[b].active_voices, s_c[b].stolen, s_c[b].dropped) == \
               (s_o[b].active_voices, s_o[b].stolen, s_o[b].dropped), f"block {b} counters"
        if sorted_pool:
            a, r = pool_by_note(p_c[b]), pool_by_note(p_o[b])
            assert a.keys() == r.keys(), f"block {b}: live note sets differ"
            for k in r:
                np.testing.assert_array_equal(a[k], r[k], err_msg=f"block {b} note {k}")
        elif exact_pool:
            assert p_c[b].shape == p_o[b].shape
            np.testing.assert_array_equal(p_c[b], p_o[b], err_msg=f"block {b} pool")
        db = null_db(o_c[b], m_o[b])
        assert db <= null_limit, f"block {b}: null {db:.1f} dB"
    cu.close()
    orc.close()
    return o_c, o_o


@gpu
@pytest.mark.parametrize("vpl", [1, 2])
def test_parity_linear_quietest_chan(vpl):
    sc = make_scenario(seed=1, voices_per_lane=vpl)
    _compare(sc)


@gpu
@pytest.mark.parametrize("vpl", [1, 2])
def test_parity_large_pool_sustained(vpl):
    """Many long-lived voices so most tiles take the branch-free hot path."""
    sc = make_scenario(seed=12, max_voices=40000, n_blocks=4, spawn_per_block=(9000, 12000), release_rate=0.02,
                       voices_per_lane=vpl, sort_voices=1)
    _compare(sc, sorted_pool=True)


@gpu
@pytest.mark.parametrize("vpl", [1, 2])
def test_parity_unit_steps(vpl):
    """Every voice plays its sample at the root pitch (step exactly 1.0, zero
    phase fractions), so sustained tiles take the fixed-offset path."""
    sc = make_scenario(seed=14, max_voices=40000, n_blocks=4, spawn_per_block=(9000, 12000), release_rate=0.02,
                       voices_per_lane=vpl, sort_voices=1, steps="unit", chan=False)
    _compare(sc, sorted_pool=True)


@gpu
@pytest.mark.parametrize("vpl", [1, 2])
def test_parity_spans_broken_by_gate_rows(vpl):
    """Unit-step voices under controller rows that mostly leave the bend at
    unity: hot spans of up to 128 frames carry across gate tiles until a row
    bends a channel, switches its params variant or releases a voice."""
    sc = make_scenario(seed=17, max_voices=40000, n_blocks=4, spawn_per_block=(9000, 12000), release_rate=0.05,
                       voices_per_lane=vpl, sort_voices=1, steps="unit", chan=True, bend_prob=0.02,
                       block_frames=4096)
    _compare(sc, sorted_pool=True)


@gpu
@pytest.mark.parametrize("steps", ["ratio", "unit", "integral"])
def test_parity_loop_wraps_inside_hot_tiles(steps):
    """Sustained voices in short loops that end at the sample's end (the
    shape of a real bank's looped zones): most lanes pass their loop end every
    few tiles, read the seam tap (loop_end - 1, whose neighbour is
    loop_start) at fractional phases, and switch between the hot paths and
    the general one around each wrap; spans of 2 to 400 frames cover one wrap
    a tile and loops short enough to wrap twice in one. Every pool field, the
    filter state included, must equal the CPU reference's."""
    sc = make_scenario(seed=21, max_voices=40000, n_blocks=4, spawn_per_block=(9000, 12000), release_rate=0.02,
                       steps=steps, chan=steps == "ratio", bend_prob=0.5, block_frames=4096)
    rng = np.random.default_rng(22)
    for blk in sc.blocks:
        c = blk.cmds
        span = rng.integers(17, 401, c.size).astype(np.uint32)
        short = rng.random(c.size) < 0.05
        span[short] = rng.integers(2, 17, int(short.sum()))
        c["loop_end"] = c["smp_len"]
        c["loop_start"] = c["smp_len"] - np.minimum(span, c["smp_len"] - 1)
        c["flags"] = np.where(rng.random(c.size) < 0.85, N.VF_LOOP, N.VF_LOOP | N.VF_LOOP_UNTIL_RELEASE)
        c["phase_hi"] = c["loop_start"] + (rng.random(c.size) * (c["loop_end"] - c["loop_start"])).astype(np.uint32)
    _compare(sc)


@gpu
@pytest.mark.parametrize("interp", [N.INTERP_LINEAR, N.INTERP_NEAREST])
def test_parity_integral_steps(interp):
    """Whole-number steps (1, 2, 3) with zero phase fractions: the
    zero-fraction paths for linear and nearest interpolation."""
    sc = make_scenario(seed=15, max_voices=40000, n_blocks=4, spawn_per_block=(9000, 12000), release_rate=0.02,
                       sort_voices=1, steps="integral", chan=False, interpolation=interp)
    _compare(sc, sorted_pool=True)


@gpu
def test_sort_radix_widths_agree():
    """The pool sort at every digit width leaves the same pool, so blocks
    and pools are byte-identical to the default 8-bit width."""
    from kestrel_b200.backend import CudaSynth
    ref = None
    for rb in (8, 4, 5, 7, 10):
        sc = make_scenario(seed=16, max_voices=20000, n_blocks=4, spawn_per_block=(4000, 7000), sort_voices=1,
                           sort_radix_bits=rb)
        cu = CudaSynth(sc.cfg, sc.pool, sc.params, sc.n_regions, sc.max_len)
        o, s, p, _ = run(cu, sc, collect_pool=True)
        cu.close()
        got = (np.concatenate(o).tobytes(), [x.tobytes() for x in p])
        if ref is None:
            ref = got
        else:
            assert got == ref, f"radix {rb}"


@gpu
@pytest.mark.parametrize("steps,chan", [("unit", True), ("integral", False), (None, True)])
def test_unit_tile_lengths_agree(steps, chan):
    """16-frame and 32-frame hot tiles (unit, integral and, with the default
    steps, fractional), and the per-block choice between them, leave
    byte-identical blocks and pools; the 32-frame form against the CPU
    reference as well."""
    from kestrel_b200.backend import CudaSynth
    ref = None
    for utf in (16, 32, 0):
        kw = dict(steps=steps) if steps else {}
        sc = make_scenario(seed=19, max_voices=30000, n_blocks=5, spawn_per_block=(6000, 9000), release_rate=0.03,
                           sort_voices=1, chan=chan, bend_prob=0.02, block_frames=4096, unit_tile_frames=utf, **kw)
        cu = CudaSynth(sc.cfg, sc.pool, sc.params, sc.n_regions, sc.max_len)
        o, s, p, _ = run(cu, sc, collect_pool=True)
        cu.close()
        got = (np.concatenate(o).tobytes(), [x.tobytes() for x in p])
        if ref is None:
            ref = got
        else:
            assert got == ref, f"unit_tile_frames {utf}"
        if utf == 32:
            _compare(sc, sorted_pool=True)


@gpu
def test_parity_oldest_even_nochan():
    sc = make_scenario(seed=2, steal_rule=N.STEAL_OLDEST, admit_rule=N.ADMIT_EVEN, chan=False, variants=0)
    _compare(sc)


@gpu
def test_parity_dropnew():
    sc = make_scenario(seed=3, steal_rule=N.STEAL_DROP_NEW)
    _compare(sc)


@gpu
@pytest.mark.parametrize("interp", [N.INTERP_NEAREST, N.INTERP_CUBIC])
def test_parity_interpolation(interp):
    sc = make_scenario(seed=4 + interp, interpolation=interp)
    _compare(sc)


@gpu
def test_parity_linear_curves():
    sc = make_scenario(seed=7, decay_curve=N.CURVE_LINEAR, release_curve=N.CURVE_LINEAR)
    _compare(sc)


@gpu
@pytest.mark.parametrize("vpl", [1, 2])
def test_parity_sorted_pool(vpl):
    sc = make_scenario(seed=8, sort_voices=1, voices_per_lane=vpl)
    _compare(sc, sorted_pool=True)


@gpu
def test_parity_two_sum_mix():
    sc = make_scenario(seed=9, mix_mode=N.MIX_TWO_SUM)
    _compare(sc)


@gpu
def test_fast_fp_nulls_and_integer_state_exact():
    """Without strict rounding the biquad/interpolation may contract into FMA;
    the integer state and envelope stay bit-exact and the audio still nulls."""
    sc = make_scenario(seed=10, strict_fp=0)
    cu, orc = _pair(sc)
    o_c, s_c, p_c, _ = run(cu, sc, collect_pool=True)
    o_o, s_o, p_o, m_o = run(orc, sc, collect_pool=True)
    exact = [N.FIELD[f] for f in N.FIELDS if f not in ("filt_z1", "filt_z2")]
    for b in range(len(sc.blocks)):
        np.testing.assert_array_equal(p_c[b][exact], p_o[b][exact])
        assert null_db(o_c[b], m_o[b]) <= -100.0


@gpu
def test_rerun_byte_identical():
    sc = make_scenario(seed=11, sort_voices=1)
    from kestrel_b200.backend import CudaSynth
    outs = []
    for _ in range(2):
        cu = CudaSynth(sc.cfg, sc.pool, sc.params, sc.n_regions, sc.max_len)
        o, _, _, _ = run(cu, sc)
        outs.append(np.concatenate(o))
        cu.close()
    assert outs[0].tobytes() == outs[1].tobytes()


@gpu
def test_f64_mix_matches_the_oracle_f64_mix():
    """KC_MIX_F64 accumulates the same f32 voice terms in double, like the
    oracle's f64 mixdown (src/cpu.rs:589-590): the blocks agree to within one
    f32 ulp (only the f64 summation order differs)."""
    sc = make_scenario(seed=13, mix_mode=N.MIX_F64)
    cu, orc = _pair(sc)
    o_c, _, _, _ = run(cu, sc)
    o_o, _, _, _ = run(orc, sc)
    for b in range(len(sc.blocks)):
        ulp = np.spacing(np.abs(o_o[b]).astype(np.float32))
        assert np.all(np.abs(o_c[b].astype(np.float64) - o_o[b]) <= ulp), f"block {b}"


@gpu
def test_fp64_lowpass_design():
    """kc_design_lowpass_f64 designs the RBJ lowpass in double: the poles
    (a1, a2) are the exact design rounded once to f32, and the numerator is
    matched to those rounded poles, b0 = gain (1 + a1 + a2) / 4 and b1 = 2 b0,
    so the stored f32 filter's DC gain is the design's to within b0's own
    rounding (2^-24 relative). The reference's f32 design, rounded
    coefficient by coefficient, misses the DC gain by the cancellation in
    1 + a1 + a2 (hundreds of ulp at 20 Hz), which the check below shows
    against the same bound."""
    from kestrel_b200 import host as H
    from kestrel_b200.precision import _design_exact
    lib = N.cuda_lib()
    fc = np.array([20.0, 35.0, 80.0, 200.0, 1000.0, 8000.0], np.float32)
    q_cb = np.array([290.0, 150.0, 30.0, 0.0, 30.0, 30.0], np.float32)
    out = np.empty((fc.size, 4), np.float32)
    N.check(lib.kc_design_lowpass_f64(N.ptr(fc), N.ptr(q_cb), fc.size, 48000.0, N.ptr(out), 0), lib)
    exact = _design_exact(fc.astype(np.float64), q_cb.astype(np.float64), 48000.0)
    o = out.astype(np.float64)
    # poles: the exact design rounded once
    assert np.all(np.abs(o[:, 2:] - exact[:, 2:]) <= np.spacing(np.abs(out[:, 2:])) * 0.5), (o, exact)
    # numerator: b1 = 2 b0 exactly, matched to the rounded poles
    assert np.array_equal(out[:, 1], 2.0 * out[:, 0])
    q = np.maximum(10.0 ** ((q_cb.astype(np.float64) / 10.0 - 3.01) / 20.0), 0.001)
    gain = np.sqrt(np.sqrt(0.5) / q)
    dc = (2 * o[:, 0] + o[:, 1]) / ((1 + o[:, 2]) + o[:, 3])
    assert np.all(np.abs(dc / gain - 1) <= 2.0 ** -23), dc / gain - 1
    ref = np.array([H.biquad_lowpass(float(f), float(c), 48000.0) for f, c in zip(fc, q_cb)], np.float64)
    dc_ref = (2 * ref[:, 0] + ref[:, 1]) / ((1 + ref[:, 2]) + ref[:, 3])
    assert np.abs(dc_ref[0] / gain[0] - 1) > 100 * 2.0 ** -23   # 20 Hz: the f32 design's DC drift
