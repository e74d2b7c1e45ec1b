"""The render server: continuous batching against the plain path.

A served job must come out the same whatever else is on the device with it.
kc_batch_render is byte-identical to kc_render per job, so the stated
tolerance here is zero: every job's output hash (FNV-1a over its output
blocks' bytes) from the batched server equals its hash from the sequential
server (one job at a time through kc_render) and from rendering it alone
through the Python driver loop. The GPU tests also check that jobs overlap on
the device (several resident at once), that admission keeps the resident
device bytes inside the budget, and that latency accounting is consistent.
"""
import numpy as np
import pytest

from kestrel_b200 import host as H
from kestrel_b200 import native as N
from kestrel_b200 import serve as S

gpu = pytest.mark.gpu


def _small_jobs(n=6, seed=5, spacing=0.05, blocks=(6, 13)):
    """Small, uneven jobs: pools 512-8192 voices, 2k-40k notes, 1-8 presets,
    arrivals `spacing` s apart, 6-12 blocks each by default."""
    rng = np.random.default_rng(seed)
    jobs = []
    for i in range(n):
        pool = int(rng.choice([512, 1024, 3000, 8192]))
        presets = int(rng.choice([1, 2, 8]))
        cfg = N.default_config(max_voices=pool, block_frames=4096)
        bs = H.bank_spec(presets=presets, random_generators=1 if presets > 1 else 0, sample_frames=8192,
                         loop_frames=2048, seed=100 + i)
        ms = H.midi_spec(notes=int(rng.integers(2_000, 40_000)), seconds=1.0, dur_median_s=0.1,
                         program_period_s=0.25 if presets > 1 else 0.0, programs=presets, seed=200 + i)
        jobs.append(S.JobSpec(cfg, bs, ms, arrival_s=i * spacing, max_blocks=int(rng.integers(*blocks))))
    return jobs


def test_served_jobs_is_seeded_and_shaped():
    a = S.served_jobs(64, seed=3)
    b = S.served_jobs(64, seed=3)
    assert [j.arrival_s for j in a] == [j.arrival_s for j in b]
    arr = np.array([j.arrival_s for j in a])
    assert np.all(np.diff(arr) > 0)
    # Poisson at 20 jobs/s: mean gap near 50 ms
    assert 0.025 < np.mean(np.diff(arr)) < 0.1
    pools = np.array([j.cfg.max_voices for j in a])
    notes = np.array([j.midi.notes for j in a])
    secs = np.array([j.midi.seconds for j in a])
    assert pools.min() >= 16_384 and pools.max() <= 2_097_152
    assert notes.min() >= 10_000 and notes.max() <= 20_000_000
    assert secs.min() >= 5.0 and secs.max() <= 300.0
    pres = np.array([j.bank.presets for j in a])
    assert pres.min() >= 1 and pres.max() <= 128
    c = S.served_jobs(4, seed=3, max_seconds=2.0)
    assert all(j.max_blocks == 24 for j in c)


def test_serve_rejects_bad_arguments():
    jobs = _small_jobs(2)
    with pytest.raises(N.KestrelError, match="max_jobs"):
        S.serve(jobs, max_jobs=0)
    with pytest.raises(N.KestrelError, match="mode"):
        S.serve(jobs, mode=7)
    jobs[1].cfg.interpolation = N.INTERP_CUBIC
    with pytest.raises(N.KestrelError, match="differs from job 0"):
        S.serve(jobs)
    assert S.serve([]).stats.voice_samples == 0


def test_hash_block_is_fnv1a_over_words():
    x = np.arange(6, dtype=np.float32)
    h = 0xcbf29ce484222325
    for w in x.view(np.uint64):
        h = ((h ^ int(w)) * 0x100000001b3) & 0xFFFFFFFFFFFFFFFF
    assert S.hash_block(0, x) == h


def _alone(job: S.JobSpec) -> int:
    """The job rendered by itself through the Python driver loop."""
    from kestrel_b200.backend import CudaSynth
    bank = H.Bank(job.bank, job.cfg)
    drv = H.Driver(job.cfg, bank, job.midi)
    s = CudaSynth(job.cfg, bank.pool, bank.params, bank.regions, bank.max_sample_len)
    h = 0
    for _ in range(job.max_blocks):
        blk = drv.prepare(s.stats().active_voices)
        H.feed(s, blk)
        h = S.hash_block(h, s.render())
        if not drv.finish(s.stats().active_voices):
            break
    s.close()
    drv.close()
    bank.close()
    return h


@gpu
def test_batched_equals_sequential_equals_alone():
    # 30-50 blocks a job, so a job is still rendering when the next one's
    # bank is built (four setup threads of sixteen)
    jobs = _small_jobs(blocks=(30, 51))
    seq = S.serve(jobs, mode=S.MODE_SEQUENTIAL, realtime_arrivals=False)
    # all queued at start: they share the device, at most three at a time
    bat = S.serve(jobs, mode=S.MODE_BATCHED, max_jobs=3, host_threads=16, realtime_arrivals=False)
    assert all(r.status == 0 for r in seq.jobs + bat.jobs)
    assert seq.hashes() == bat.hashes()
    assert [r.blocks for r in seq.jobs] == [r.blocks for r in bat.jobs]
    assert [r.voice_samples for r in seq.jobs] == [r.voice_samples for r in bat.jobs]
    assert 2 <= bat.stats.max_resident <= 3     # jobs overlapped on the device, never more than the slots
    assert seq.stats.max_resident == 1
    assert seq.stats.gpu_ms > 0 and bat.stats.gpu_ms > 0   # device time recorded in both modes
    # the plain path on four threads at once, one context per job
    par = S.serve(jobs, mode=S.MODE_PARALLEL, host_threads=4, realtime_arrivals=False)
    assert all(r.status == 0 for r in par.jobs)
    assert par.hashes() == seq.hashes()
    assert 2 <= par.stats.max_resident <= 4 and par.stats.host_threads == 4
    for k in (0, 3):
        assert _alone(jobs[k]) == seq.jobs[k].out_hash
    # arrivals on the wall clock: each job is admitted no earlier than it arrives
    rt = S.serve(jobs, mode=S.MODE_BATCHED, max_jobs=3, host_threads=16, realtime_arrivals=True)
    assert rt.hashes() == seq.hashes()
    for r in rt.jobs:
        assert r.arrival_s <= r.admit_s <= r.first_block_s <= r.done_s
    assert np.all(rt.latencies() > 0)


@gpu
def test_admission_by_device_memory():
    jobs = _small_jobs(5, seed=9, spacing=0.0)
    est = []
    for j in jobs:
        bank = H.Bank(j.bank, j.cfg)
        b = C_u64()
        N.check(N.cuda_lib().kc_estimate_device_bytes(j.cfg, bank.pool.size, bank.params.size, b))
        est.append(b.value)
        bank.close()
    est = np.array(est)
    # Room for the two largest jobs at once, never all five.
    budget = int(np.sort(est)[-2:].sum())
    assert budget < est.sum()
    ref = S.serve(jobs, mode=S.MODE_SEQUENTIAL)
    bat = S.serve(jobs, mode=S.MODE_BATCHED, max_jobs=8, vram_budget=budget, realtime_arrivals=False)
    assert bat.hashes() == ref.hashes()
    assert 0 < bat.stats.peak_device_bytes <= budget
    assert bat.stats.max_resident < len(jobs)
    # the estimate admission charges is what the context holds
    assert all(r.device_bytes == e for r, e in zip(bat.jobs, est))


@gpu
def test_on_block_sees_every_block_in_order():
    jobs = _small_jobs(3, seed=12, spacing=0.0)
    seen = {}

    def cb(job, block, out):
        seen.setdefault(job, []).append((block, S.hash_block(0, out)))

    bat = S.serve(jobs, mode=S.MODE_BATCHED, max_jobs=4, on_block=cb)
    for k, r in enumerate(bat.jobs):
        blocks = [b for b, _ in seen[k]]
        assert blocks == list(range(r.blocks))


def C_u64():
    import ctypes
    return ctypes.c_uint64()


@gpu
def test_autotune_times_every_candidate():
    job = _small_jobs(1, seed=31)[0]
    job.cfg.max_voices = 8192
    job.midi.notes = 60_000
    job.max_blocks = 0
    best, res = S.autotune(job, voices_per_lane=(1, 2), radix_bits=(6, 8), preroll=4, timed=3)
    assert len(res) == 4
    assert {(r.voices_per_lane, r.sort_radix_bits) for r in res} == {(1, 6), (1, 8), (2, 6), (2, 8)}
    assert all(r.blocks == 3 and r.device_ms > 0 and r.voice_samples > 0 for r in res)
    win = max(res, key=lambda r: r.voice_samples_per_s)
    assert (best.voices_per_lane, best.sort_radix_bits, best.block_frames) == \
        (win.voices_per_lane, win.sort_radix_bits, win.block_frames)
    # every other field is the job's own
    for f, _ in N.KcConfig._fields_:
        if f not in ("voices_per_lane", "sort_radix_bits", "block_frames", "reserved"):
            assert getattr(best, f) == getattr(job.cfg, f), f
    # block lengths are tried only when listed
    best2, res2 = S.autotune(job, voices_per_lane=(1,), radix_bits=(8,), block_frames=(2048, 4096), preroll=2,
                             timed=2)
    assert sorted(r.block_frames for r in res2) == [2048, 4096]


@gpu
def test_serve_with_autotune_matches_sequential():
    jobs = _small_jobs(4, seed=33, spacing=0.0)
    bat = S.serve(jobs, mode=S.MODE_BATCHED, max_jobs=4, autotune=True, realtime_arrivals=False)
    v, r = bat.stats.tuned_voices_per_lane, bat.stats.tuned_sort_radix_bits
    assert v in (1, 2) and r in (6, 8, 10)
    for j in jobs:
        j.cfg.voices_per_lane = v
        j.cfg.sort_radix_bits = r
    seq = S.serve(jobs, mode=S.MODE_SEQUENTIAL, realtime_arrivals=False)
    assert bat.hashes() == seq.hashes()
