"""The batched form (kc_batch_render) against each job rendered alone.

A batch renders one block of many contexts with one launch sequence. The
claim under test is that every job's output block, stats and voice pool are
byte-identical to rendering the same context alone through kc_render, for
jobs that differ in pool size, steal and admit rules, sort setting, channel
path and lifetime (jobs joining and leaving between blocks), with and
without the captured graph. Solo parity with the oracle is covered in
test_backend_parity.py; one job here is also checked against the oracle
directly.
"""
import numpy as np
import pytest

from kestrel_b200 import native as N
from scenarios import make_scenario, null_db, run

gpu = pytest.mark.gpu


def _jobs(strict_fp=1, mix_mode=N.MIX_F32_TREE, vpl=0):
    kw = dict(strict_fp=strict_fp, mix_mode=mix_mode, voices_per_lane=vpl)
    return [
        make_scenario(seed=21, max_voices=4096, n_blocks=6, **kw),
        make_scenario(seed=22, max_voices=512, n_blocks=5, spawn_per_block=(0, 400), steal_rule=N.STEAL_OLDEST,
                      admit_rule=N.ADMIT_EVEN, **kw),
        # sorted every third block (compacted on the others)
        make_scenario(seed=23, max_voices=30000, n_blocks=4, spawn_per_block=(6000, 9000), release_rate=0.02,
                      sort_voices=3, **kw),
        make_scenario(seed=24, max_voices=2048, n_blocks=6, chan=False, variants=0, steal_rule=N.STEAL_DROP_NEW,
                      **kw),
        make_scenario(seed=25, max_voices=64, n_blocks=3, spawn_per_block=(0, 40), sort_voices=2, **kw),
        make_scenario(seed=26, max_voices=8192, n_blocks=5, spawn_per_block=(0, 0), **kw),  # silent job
    ]


def _solo(sc):
    from kestrel_b200.backend import CudaSynth
    s = CudaSynth(sc.cfg, sc.pool, sc.params, sc.n_regions, sc.max_len)
    outs, stats, pools, _ = run(s, sc, collect_pool=True)
    s.close()
    return outs, stats, pools


def _feed(s, blk):
    for vi, pv in blk.variants:
        s.set_params_variant(vi, pv)
    s.set_gates(blk.gates)
    s.set_channels(blk.chan, blk.bend, blk.gain, blk.variant)
    s.spawn(blk.cmds)


def _batched(scs, starts, use_graph=True):
    """Jobs join at block `starts[i]` of the batch and leave after their last
    block; every batch step renders the jobs alive at that step."""
    from kestrel_b200.backend import CudaBatch, CudaSynth
    jobs = [None] * len(scs)
    res = [([], [], []) for _ in scs]
    end = max(st + len(sc.blocks) for sc, st in zip(scs, starts))
    with CudaBatch.for_config(scs[0].cfg, max_jobs=8, use_graph=use_graph) as b:
        for step in range(end):
            alive = []
            for i, (sc, st) in enumerate(zip(scs, starts)):
                k = step - st
                if 0 <= k < len(sc.blocks):
                    if jobs[i] is None:
                        jobs[i] = CudaSynth(sc.cfg, sc.pool, sc.params, sc.n_regions, sc.max_len)
                    _feed(jobs[i], sc.blocks[k])
                    alive.append(i)
            outs = b.render([jobs[i] for i in alive])
            for i, o in zip(alive, outs):
                res[i][0].append(o.copy())
                res[i][1].append(jobs[i].stats())
                res[i][2].append(jobs[i].read_pool())
                if step - starts[i] == len(scs[i].blocks) - 1:
                    jobs[i].close()
                    jobs[i] = None
    return res


def _assert_same(solo, batched, tag):
    so, ss, sp = solo
    bo, bs, bp = batched
    assert len(so) == len(bo)
    for k in range(len(so)):
        assert so[k].tobytes() == bo[k].tobytes(), f"{tag} block {k}: output differs"
        assert (ss[k].active_voices, ss[k].stolen, ss[k].dropped, ss[k].peak) == \
               (bs[k].active_voices, bs[k].stolen, bs[k].dropped, bs[k].peak), f"{tag} block {k}: stats"
        np.testing.assert_array_equal(sp[k], bp[k], err_msg=f"{tag} block {k}: pool")


@gpu
@pytest.mark.parametrize("use_graph", [True, False])
def test_batch_matches_each_job_alone(use_graph):
    scs = _jobs()
    starts = [0, 1, 0, 2, 4, 0]
    res = _batched(scs, starts, use_graph=use_graph)
    for i, sc in enumerate(scs):
        _assert_same(_solo(sc), res[i], f"job {i}")


@gpu
@pytest.mark.parametrize("mix_mode", [N.MIX_TWO_SUM, N.MIX_F64])
def test_batch_matches_alone_other_mixes(mix_mode):
    scs = _jobs(mix_mode=mix_mode)[:4]
    res = _batched(scs, [0, 0, 1, 0])
    for i, sc in enumerate(scs):
        _assert_same(_solo(sc), res[i], f"mix {mix_mode} job {i}")


@gpu
@pytest.mark.parametrize("use_graph", [True, False])
def test_batch_matches_alone_on_unit_spans(use_graph):
    """Unit and integral-step jobs: from the second batch on the batch runs
    its 32-frame unit-tile graph, and every job still matches itself alone."""
    scs = [make_scenario(seed=31 + i, max_voices=20000, n_blocks=6, spawn_per_block=(3000, 6000), release_rate=0.03,
                         sort_voices=1, steps=st, chan=ch, bend_prob=0.02, block_frames=4096)
           for i, (st, ch) in enumerate([("unit", False), ("unit", True), ("integral", False)])]
    res = _batched(scs, [0, 0, 1], use_graph=use_graph)
    for i, sc in enumerate(scs):
        _assert_same(_solo(sc), res[i], f"unit job {i}")


@gpu
def test_batch_matches_alone_two_voices_per_lane_fast_fp():
    scs = _jobs(strict_fp=0, vpl=2)[:3]
    res = _batched(scs, [0, 0, 0])
    for i, sc in enumerate(scs):
        _assert_same(_solo(sc), res[i], f"vpl2 job {i}")


@gpu
def test_batch_job_against_oracle():
    from oracle.binding import OracleSynth
    scs = _jobs()[:3]
    res = _batched(scs, [0, 0, 0])
    sc = scs[2]
    orc = OracleSynth(sc.cfg, sc.pool, sc.params)
    o_o, s_o, _, m_o = run(orc, sc, collect_pool=True)
    orc.close()
    for k in range(len(sc.blocks)):
        assert res[2][1][k].active_voices == s_o[k].active_voices
        assert null_db(res[2][0][k], m_o[k]) <= -100.0


@gpu
def test_batch_rejects_bad_job_lists():
    from kestrel_b200.backend import CudaBatch, CudaSynth
    a, c = _jobs()[0], _jobs(mix_mode=N.MIX_TWO_SUM)[0]
    with CudaBatch.for_config(a.cfg, max_jobs=2) as b:
        s1 = CudaSynth(a.cfg, a.pool, a.params, a.n_regions, a.max_len)
        s2 = CudaSynth(c.cfg, c.pool, c.params, c.n_regions, c.max_len)
        with pytest.raises(N.KestrelError, match="listed twice"):
            b.render([s1, s1])
        with pytest.raises(N.KestrelError, match="differs from the batch"):
            b.render([s1, s2])
        with pytest.raises(N.KestrelError, match="exceeds"):
            b.render([s1, s1, s1])
        # an empty step is fine
        assert b.render([]) == []
        s1.close()
        s2.close()
