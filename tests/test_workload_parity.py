"""Block-level parity on the benchmark workloads, driver included.

The C++ driver feeds the CUDA backend and the CPU oracle the same blocks
(exactly as Kestrel's Driver feeds whichever backend it was given,
src/driver.rs:1-6); both must agree on every counter, on the live pool as a
note-id keyed multiset (the pool is re-sorted on the device, src/gpu/mod.rs:
59-106), and on the audio: the peak null against the oracle's f64 mix stays
below -100 dBFS (README.md:37-38). Sizes are reduced so the single-threaded
oracle finishes in seconds; the shapes are the configurations'.
"""
import numpy as np
import pytest

from kestrel_b200 import host as H
from kestrel_b200 import native as N
from scenarios import null_db, pool_by_note

gpu = pytest.mark.gpu


def _run_pair(cfg, bs, ms, blocks, check_every=1):
    from kestrel_b200.backend import CudaSynth
    from oracle.binding import OracleSynth
    bank = H.Bank(bs, cfg)
    d1, d2 = H.Driver(cfg, bank, ms), H.Driver(cfg, bank, ms)
    cu = CudaSynth(cfg, bank.pool, bank.params, bank.regions, bank.max_sample_len)
    orc = OracleSynth(cfg, bank.pool, bank.params)
    worst = -np.inf
    for b in range(blocks):
        x = d1.prepare(cu.stats().active_voices)
        y = d2.prepare(orc.stats().active_voices)
        assert np.array_equal(x.cmds, y.cmds), f"block {b}: drivers diverged"
        H.feed(cu, x)
        H.feed(orc, y)
        oc = cu.render().copy()
        oo = orc.render()
        sc, so = cu.stats(), orc.stats()
        assert (sc.active_voices, sc.stolen, sc.dropped) == (so.active_voices, so.stolen, so.dropped), b
        db = null_db(oc, orc.last_mix64)
        worst = max(worst, db)
        assert db <= -100.0, f"block {b}: null {db:.1f} dB"
        if b % check_every == 0:
            pc, po = pool_by_note(cu.read_pool()), pool_by_note(orc.read_pool())
            assert pc.keys() == po.keys(), f"block {b}: live sets differ"
            for k in po:
                np.testing.assert_array_equal(pc[k], po[k], err_msg=f"block {b} note {k}")
        d1.finish(sc.active_voices)
        d2.finish(so.active_voices)
    return worst, cu.stats()


@gpu
def test_plain_workload_parity():
    cfg, bs, ms = H.config_workload("plain", seed=5)
    worst, st = _run_pair(cfg, bs, ms, blocks=40, check_every=4)
    assert st.active_voices > 500


@gpu
def test_black_midi_workload_parity():
    cfg, bs, ms = H.config_workload("black", seed=6)
    ms.notes, ms.seconds = 400_000, 20.0  # same density shape, fewer blocks
    cfg.max_voices = 32768
    worst, st = _run_pair(cfg, bs, ms, blocks=24, check_every=3)
    assert st.active_voices > 1000


@gpu
def test_steal_saturation_parity():
    """Sustained concurrency over the pool: the steal order must be bit-exact
    (victim sets show up as stop frames and then as the surviving set)."""
    cfg, bs, ms = H.config_workload("steal", seed=7)
    cfg.max_voices = 20000
    ms.notes, ms.seconds = 1_000_000, 30.0  # ~33k notes/s, 6 s notes: saturates in < 1 s
    worst, st = _run_pair(cfg, bs, ms, blocks=24, check_every=2)
    assert st.stolen > 10000 and st.active_voices == cfg.max_voices
