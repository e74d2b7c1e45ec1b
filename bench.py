#!/usr/bin/env python
"""Benchmark of the B200 synthesis backend on Kestrel's per-block hot path.

One step is one audio block (4096 frames, 48 kHz stereo) of the Backend
contract: steal-select, spawn, per-voice render, mix, compact/sort.

Workloads (seeded synthetic stand-ins with the shapes the benchmark
configurations describe; no public dataset is involved):
  steal  (default) 200M notes over 120 s, log-normal durations (median 6 s,
         sigma 0.5) so concurrency exceeds the pool; --max-voices 8,388,608,
         steal-percent 10. The largest single-GPU configuration and the one
         that actually sustains 8.4M concurrent voices.
  black  20M notes over 180 s, 60% of onsets in 1 ms clusters of 1k-50k notes,
         128 presets, bend/CC7/CC11 every 10 ms; --max-voices 1,048,576.
  plain  100k notes over 30 s, 1 preset, --max-voices 65,536.

Measurement. A driver (the C++ restatement of src/driver.rs) renders a
pre-roll until the pool reaches its steady state. Then:
  serial W + K blocks through the C ABI with host buffers (kc_set_gates,
         kc_set_channels, kc_spawn, kc_render), one at a time; records the
         blocks' inputs (reported as measured.e2e_serial).
  e2e    a clone of the context at the same state replays the recorded host
         buffers through the pipelined form of the same calls: the next
         block's inputs are staged (kc_set_* / kc_spawn) while this one
         renders, between kc_render_begin and kc_render_end. The host->device
         copies of every block's inputs and the device->host read of its
         stereo block are inside the timed region; the driver's own
         preparation is not.
  value  another clone replays the same W + K recorded blocks from HBM
         (kc_enqueue_block_device), K timed back to back with CUDA events on
         the context's stream.
The three renders are checked to be byte-identical.

Metric: voice-samples/s = sum over blocks of (voices rendered x 4096) / time;
x-realtime = audio seconds / time.

`--impl reference` times the CPU restatement of the reference backend
(src/cpu.rs, the oracle) on the host's cores over the workload's first
W + K blocks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

PREROLL = {"steal": 64, "steal-bent": 64, "black": 48, "plain": 24}


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["cuda", "reference"], default="cuda")
    ap.add_argument("--workload", choices=["steal", "steal-bent", "black", "plain", "served"], default="steal")
    ap.add_argument("--served-jobs", type=int, default=32, help="jobs of the served workload")
    ap.add_argument("--served-seconds", type=float, default=2.0,
                    help="audio seconds rendered per served job (its MIDI keeps its full length)")
    ap.add_argument("--served-arrivals", choices=["poisson", "queued"], default="poisson")
    ap.add_argument("--preroll", type=int, default=None)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="bound of the cpu_baseline sample")
    ap.add_argument("--voices-per-lane", type=int, default=0)
    ap.add_argument("--strict-fp", type=int, default=1)
    ap.add_argument("--mix-mode", type=int, default=0, help="0 f32 tree, 1 compensated two-sum, 2 FP64")
    ap.add_argument("--sort-every", type=int, default=1,
                    help="re-sort the voice pool every N blocks (compact it on the others); 0 never")
    ap.add_argument("--tile-frames", type=int, default=0,
                    help="longest render tile on the hot paths: 16, 32 or 0 = chosen per block")
    return ap.parse_args(argv)


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# ---- clocks during the timed region ------------------------------------------------

class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in Path(self.path).read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---- roofline ------------------------------------------------------------------------

def render_algorithmic_bytes(n_render: int, block_frames: int, tiles: int) -> int:
    """Algorithmic bytes of one render launch: each voice's 96-byte slot read
    and its 36 bytes of state written back, one new i16 sample per voice-frame
    (2 B at step ~1; the sample bank is L2-resident), and the block's gate and
    channel rows."""
    return n_render * (96 + 36 + 2 * block_frames) + tiles * 2048 * 4 + tiles * 64 * 4


def measured_peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


# The render path a workload's blocks run on (at the f32 tree mix), and so
# the captured case whose per-voice-sample figures describe its launch.
PROFILE_PATH = {"steal": "unit", "steal-bent": "fractional"}


def render_profile_per_unit(workload: str, mix_mode: int, key: str = "dram_bytes_per_voice_sample") -> float | None:
    """A per-voice-sample figure of the render kernel from the committed ncu
    summary of the render path this workload runs on
    (profiles/render_traffic.json): DRAM bytes read + written, or lane
    instructions issued. None for workloads with no captured path."""
    path = PROFILE_PATH.get(workload) if mix_mode == 0 else None
    p = ROOT / "profiles" / "render_traffic.json"
    if path and p.exists():
        try:
            return float(json.loads(p.read_text())["paths"][path][key])
        except Exception:
            return None
    return None


def torch_sm_count() -> int | None:
    try:
        import torch
        return torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    except Exception:
        return None


def issue_roofline(lane_instr_per_unit, units, launch_ms, sms, sm_mhz):
    if not (lane_instr_per_unit and launch_ms and sms and sm_mhz):
        return None
    achieved = lane_instr_per_unit * units / 32.0 / (launch_ms * 1e-3)
    peak = sms * 4 * sm_mhz * 1e6
    return {"bound": "issue", "achieved": achieved, "peak": peak, "unit": "warp-instr/s", "frac": achieved / peak,
            "lane_instructions_per_voice_sample": lane_instr_per_unit}


# ---- the CUDA arm ------------------------------------------------------------------

def run_cuda(args, world, rank, local):
    import torch
    from kestrel_b200 import host as H
    from kestrel_b200 import native as N
    from kestrel_b200.backend import CudaSynth

    torch.cuda.set_device(local)
    cfg, bs, ms = H.config_workload(args.workload, seed=args.seed + rank)
    cfg.device = local
    cfg.voices_per_lane = args.voices_per_lane
    cfg.strict_fp = args.strict_fp
    cfg.mix_mode = args.mix_mode
    cfg.unit_tile_frames = args.tile_frames
    cfg.sort_voices = args.sort_every
    bank = H.Bank(bs, cfg)
    drv = H.Driver(cfg, bank, ms)
    A = CudaSynth(cfg, bank.pool, bank.params, bank.regions, bank.max_sample_len)
    bf = cfg.block_frames
    tiles = bf // cfg.gate_frames
    out = np.empty(bf * 2, np.float32)
    preroll = args.preroll if args.preroll is not None else PREROLL[args.workload]

    # Pre-roll to the workload's steady state (untimed).
    t_pre = time.perf_counter()
    for _ in range(preroll):
        blk = drv.prepare(A.stats().active_voices)
        H.feed(A, blk)
        A.render(out)
        drv.finish(A.stats().active_voices)
    t_pre = time.perf_counter() - t_pre
    B = A.clone()
    C = A.clone()

    # The serial host-buffer form: W + K blocks through the C ABI as the
    # reference's loop makes them (kc_set_gates, kc_set_channels, kc_spawn,
    # kc_render per block); records the blocks' inputs.
    W, K = args.warmup, args.steps
    rec, ser_t, e2e_units, h2d, d2h = [], 0.0, 0, 0, 0
    outs_a = []
    for i in range(W + K):
        live = A.stats().active_voices
        blk = drv.prepare(live)
        n_render = live + len(blk.cmds)
        t0 = time.perf_counter()
        H.feed(A, blk)
        A.render(out)
        t1 = time.perf_counter()
        drv.finish(A.stats().active_voices)
        rec.append((blk, n_render))
        outs_a.append(out.copy())
        if i >= W:
            ser_t += t1 - t0
            e2e_units += n_render * bf
            h2d += blk.gates.nbytes + blk.chan.nbytes + blk.cmds.nbytes
            d2h += out.nbytes + 64

    # e2e: the same blocks' host buffers through the pipelined form of the
    # same calls on a second clone -- kc_render_begin returns once the block
    # is enqueued, and the next block's kc_set_* / kc_spawn stage its inputs
    # while this one renders (they wait only for its input copies), then
    # kc_render_end reads the block back. Every step's host-to-device copies
    # and its read-back are inside the timed region; the driver's
    # preparation is not (as in the serial form).
    outs_c = []
    for i in range(W):
        H.feed(C, rec[i][0])
        C.render(out)
        outs_c.append(out.copy())
    t0 = time.perf_counter()
    if K:
        H.feed(C, rec[W][0])
        C.render_begin()
        for i in range(W + 1, W + K):
            H.feed(C, rec[i][0])
            C.render_end(out)
            outs_c.append(out.copy())
            C.render_begin()
        C.render_end(out)
        outs_c.append(out.copy())
    e2e_t = time.perf_counter() - t0

    # value: replay the recorded blocks from HBM on the clone.
    dev = []
    for blk, n_render in rec:
        g = torch.from_numpy(blk.gates.view(np.int32)).cuda()
        c = torch.from_numpy(blk.chan.view(np.int32)).cuda()
        cm = torch.from_numpy(blk.cmds.view(np.uint8).copy()).cuda() if len(blk.cmds) else None
        o = torch.empty(bf * 2, dtype=torch.float32, device="cuda")
        dev.append((blk, n_render, g, c, cm, o))
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(B.stream())

    def enqueue(entry):
        blk, n_render, g, c, cm, o = entry
        for idx, data in blk.variants:
            B.set_params_variant(idx, data)
        B.enqueue_block_device(g.data_ptr(), c.data_ptr(), blk.bend, blk.gain, blk.variant,
                               cm.data_ptr() if cm is not None else 0, len(blk.cmds), o.data_ptr())

    for e in dev[:W]:
        enqueue(e)
    B.synchronize()
    B.set_profile(True)
    launches0 = B.launches_total()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for e in dev[W:]:
        enqueue(e)
    ev1.record(stream)
    B.synchronize()
    torch.cuda.synchronize()
    clk = clocks.stop()
    dt_ms = ev0.elapsed_time(ev1)
    passes, nblocks = B.timings_total()
    ut, at = B.last_block_tiles()
    units = sum(n for _, n, *_ in dev[W:]) * bf
    # determinism: the replay must equal the host-buffer render byte for byte
    same = all(np.array_equal(e[5].cpu().numpy(), outs_a[i]) for i, e in enumerate(dev))
    same = same and all(np.array_equal(o, outs_a[i]) for i, o in enumerate(outs_c))
    launches = B.launches_total() - launches0  # kernel launches of the K timed blocks

    res = {
        "units": units, "ms": dt_ms, "e2e_units": e2e_units, "e2e_s": e2e_t, "serial_s": ser_t,
        "h2d": h2d // max(K, 1),
        "d2h": d2h // max(K, 1), "render_ms": passes["render"] / max(nblocks, 1), "passes": passes,
        "nblocks": nblocks, "mean_live": float(np.mean([n for _, n, *_ in dev[W:]])),
        "same": same, "clocks": clk, "launches": launches, "preroll_s": t_pre, "preroll": preroll,
        "tiles": tiles, "bf": bf, "max_voices": cfg.max_voices, "sample_rate": cfg.sample_rate,
        "steal_percent": cfg.max_steal_percent, "stolen": B.stats().stolen, "dropped": B.stats().dropped,
        "hot_share": ut / at if at else None,
    }
    C.close()
    B.close()
    A.close()
    return res


# ---- the CPU restatement ---------------------------------------------------------------

def run_oracle(workload, seed, threads, max_blocks, max_seconds):
    """Time the CPU restatement of src/cpu.rs over the workload's first blocks."""
    from kestrel_b200 import host as H
    from oracle.binding import OracleSynth
    cfg, bs, ms = H.config_workload(workload, seed=seed)
    bank = H.Bank(bs, cfg)
    drv = H.Driver(cfg, bank, ms)
    orc = OracleSynth(cfg, bank.pool, bank.params, threads=threads)
    out = np.empty(cfg.block_frames * 2, np.float32)
    t_sum, units, blocks, live_max = 0.0, 0, 0, 0
    per_block = []
    while blocks < max_blocks and t_sum < max_seconds:
        live = orc.stats().active_voices
        blk = drv.prepare(live)
        n_render = live + len(blk.cmds)
        t0 = time.perf_counter()
        H.feed(orc, blk)
        orc.render(out, keep_mix64=False)
        dt = time.perf_counter() - t0
        drv.finish(orc.stats().active_voices)
        t_sum += dt
        units += n_render * cfg.block_frames
        blocks += 1
        live_max = max(live_max, n_render)
        per_block.append((n_render, dt))
    orc.close()
    return {"value": units / t_sum if t_sum > 0 else 0.0, "blocks": blocks, "seconds": t_sum, "units": units,
            "live_max": live_max, "per_block": per_block, "block_frames": cfg.block_frames,
            "sample_rate": cfg.sample_rate}


def _served_cpu_job(n_jobs, seed, served_seconds, index, budget_s):
    """One served job through the CPU restatement of src/cpu.rs, one thread,
    for at most its block bound or `budget_s` of CPU: (voice-samples, s)."""
    from kestrel_b200 import host as H
    from kestrel_b200 import serve as S
    from oracle.binding import OracleSynth
    sp = S.served_jobs(n_jobs, seed=seed, max_seconds=served_seconds)[index]
    bank = H.Bank(sp.bank, sp.cfg, sp.opt)
    drv = H.Driver(sp.cfg, bank, sp.midi)
    orc = OracleSynth(sp.cfg, bank.pool, bank.params, threads=1)
    out = np.empty(sp.cfg.block_frames * 2, np.float32)
    units, t_sum, blocks = 0, 0.0, 0
    while (not sp.max_blocks or blocks < sp.max_blocks) and t_sum < budget_s:
        live = orc.stats().active_voices
        blk = drv.prepare(live)
        t0 = time.perf_counter()
        H.feed(orc, blk)
        orc.render(out, keep_mix64=False)
        t_sum += time.perf_counter() - t0
        units += (live + len(blk.cmds)) * sp.cfg.block_frames
        blocks += 1
        if not drv.finish(orc.stats().active_voices):
            break
    orc.close()
    drv.close()
    return units, t_sum


def served_cpu_baseline(n_jobs, seed, served_seconds, workers, budget_s):
    """The served job mix as independent jobs on `workers` host cores (the
    CPU baseline of the batched configuration), each job a bounded sample of
    its render: summed voice-samples over summed render seconds, times the
    workers that ran at once."""
    import concurrent.futures as cf
    import multiprocessing as mp
    # spawn: the parent may already hold a CUDA context
    with cf.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
        res = list(ex.map(_served_cpu_job, [n_jobs] * n_jobs, [seed] * n_jobs, [served_seconds] * n_jobs,
                          range(n_jobs), [budget_s] * n_jobs))
    units = sum(u for u, _ in res)
    secs = sum(t for _, t in res)
    per_core = units / secs if secs > 0 else 0.0
    return {"value": per_core * min(workers, n_jobs), "unit": "voice-samples/s", "cores": min(workers, n_jobs),
            "kind": "port",
            "sample": f"the served mix's {n_jobs} jobs, each rendered by the C++ restatement of src/cpu.rs on one "
                      f"thread for its first blocks (at most {budget_s:g} s of CPU each), as independent jobs on "
                      f"{min(workers, n_jobs)} cores: the per-core rate x the cores"}


def run_served(args):
    """The batched-and-served configuration: the same seeded job mix through
    the render server twice -- continuous batching (one kc_batch_render per
    step for every resident job, graph-replayed) and the plain path (one job
    at a time through kc_render) -- end to end through ks_serve, host driver
    included. Returns one JSON line."""
    import torch
    from kestrel_b200 import serve as S

    torch.cuda.set_device(0)
    jobs = S.served_jobs(args.served_jobs, seed=args.seed, max_seconds=args.served_seconds)
    queued = args.served_arrivals == "queued"
    # warm-up: module load, graph capture paths, host pools
    S.serve(S.served_jobs(3, seed=args.seed + 99, max_seconds=0.2, notes=(10_000, 20_000),
                          pools=(16_384, 32_768)), mode=S.MODE_BATCHED, max_jobs=4, realtime_arrivals=False)
    S.serve(S.served_jobs(1, seed=args.seed + 98, max_seconds=0.2, notes=(10_000, 20_000),
                          pools=(16_384, 32_768)), mode=S.MODE_SEQUENTIAL, realtime_arrivals=False)
    clocks = ClockSampler(0)
    clocks.start()
    bat = S.serve(jobs, mode=S.MODE_BATCHED, max_jobs=256, realtime_arrivals=not queued)
    clk = clocks.stop()
    seq = S.serve(jobs, mode=S.MODE_SEQUENTIAL, realtime_arrivals=not queued)
    # The plain path on as many host threads as the batched server uses, one
    # context and stream per job: many contexts at once, none batched.
    par = S.serve(jobs, mode=S.MODE_PARALLEL, host_threads=int(bat.stats.host_threads),
                  realtime_arrivals=not queued)

    def summary(r):
        lat = r.latencies()
        vs = r.stats.voice_samples
        return {"voice_samples_per_s": vs / r.stats.wall_s, "wall_s": r.stats.wall_s,
                "gpu_s": r.stats.gpu_ms * 1e-3 if r.stats.gpu_ms else None,
                "device_voice_samples_per_s": vs / (r.stats.gpu_ms * 1e-3) if r.stats.gpu_ms else None,
                "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
                "mean_latency_s": float(lat.mean()), "steps": int(r.stats.steps),
                "max_resident": int(r.stats.max_resident), "host_threads": int(r.stats.host_threads),
                "peak_device_gb": r.stats.peak_device_bytes / 1e9, "voice_samples": int(vs),
                "failed_jobs": sum(1 for j in r.jobs if j.status != 0)}

    b, s = summary(bat), summary(seq)
    p = summary(par)
    same = bat.hashes() == seq.hashes() == par.hashes()
    audio_s = sum(j.blocks for j in bat.jobs) * 4096 / 48000
    blocks = sum(j.blocks for j in bat.jobs)
    line = {
        "metric": "aggregate voice-samples/s of the served job mix (p50/p99 job latency beside)",
        "value": b["voice_samples_per_s"], "unit": "voice-samples/s", "n_gpus": 1,
        "steps": int(bat.stats.steps), "warmup": 1, "ms_per_step": b["wall_s"] * 1e3 / max(bat.stats.steps, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "impl": "cuda-batched-served",
        "config": {"workload": f"served: {len(jobs)} jobs, Poisson arrivals at 20 jobs/s"
                               f"{' (all queued at start)' if queued else ''}, notes log-uniform 10k-20M, "
                               f"durations U[5,300] s, pools log-uniform 16k-2M, 1-128 presets per job; "
                               f"each job bounded to its first {args.served_seconds:g} s of audio",
                   "jobs": len(jobs), "job_audio_s": audio_s, "job_blocks": blocks,
                   "arrivals": "queued" if queued else "poisson-realtime"},
        "batched": b, "sequential_plain_path": s, "parallel_plain_path": p,
        "ratio_vs_plain_path": b["voice_samples_per_s"] / s["voice_samples_per_s"],
        "ratio_vs_parallel_plain_path": b["voice_samples_per_s"] / p["voice_samples_per_s"],
        # Device time alone: the batch's launch sequences against the same
        # jobs' blocks rendered one context at a time (each summed on the
        # device with CUDA events), so host threads drop out of the ratio.
        "device_ratio_vs_plain_path": (b["device_voice_samples_per_s"] / s["device_voice_samples_per_s"]
                                       if b["device_voice_samples_per_s"] and s["device_voice_samples_per_s"]
                                       else None),
        "p50_latency_s": b["p50_latency_s"], "p99_latency_s": b["p99_latency_s"],
        "outputs_identical_to_plain_path": same,
        "e2e": {"value": b["voice_samples_per_s"], "unit": "voice-samples/s", "h2d_bytes_per_step": None,
                "d2h_bytes_per_step": 32832, "note": "the served run is itself end to end: ks_serve with "
                                                    "host drivers, host buffers and per-block readback"},
        "clocks": clk,
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = served_cpu_baseline(len(jobs), args.seed, args.served_seconds,
                                                   os.cpu_count() or 1, max(args.cpu_seconds / 10, 0.5))
    return line


def reduce_over_ranks(units, e2e_units, ms_t, e2e_s, device):
    """Replicas: every rank rendered its own job. The job's work is the sum of
    the ranks' voice-samples; its time is the slowest rank's."""
    import torch
    t = torch.tensor([float(units), float(e2e_units)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t)
    m = torch.tensor([float(ms_t), float(e2e_s)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(m, op=torch.distributed.ReduceOp.MAX)
    return float(t[0]), float(t[1]), float(m[0]), float(m[1])


def workload_desc(name):
    return {
        "steal": "steal-saturation: 200M notes / 120 s, log-normal durations (median 6 s, sigma 0.5), "
                 "1 preset x 128 zones, max_voices 8,388,608, steal-percent 10",
        "steal-bent": "steal-saturation with a pitch-bend, CC7 and CC11 curve per channel every 10 ms (every voice "
                      "at a fractional step): 200M notes / 120 s, log-normal durations (median 6 s, sigma 0.5), "
                      "1 preset x 128 zones, max_voices 8,388,608, steal-percent 10",
        "black": "black-midi: 20M notes / 180 s, 60% in 1 ms clusters of 1k-50k, 128 presets, "
                 "bend+CC7+CC11 every 10 ms, max_voices 1,048,576",
        "plain": "plain: 100k notes / 30 s, 1 preset, max_voices 65,536",
    }[name]


# The reference arm renders the steal workloads at this fraction of their
# pool and note count: the same per-voice work (durations, steal percent,
# bank) at a size whose pre-roll to the steady state and timed blocks fit in
# minutes on the host's cores.
REFERENCE_SCALE = {"steal": 8, "steal-bent": 8}


def bench_config(args, world):
    """The workload the line is quoted on; both arms print this object."""
    from kestrel_b200 import host as H
    cfg, _, _ = H.config_workload(args.workload, seed=args.seed)
    return {"workload": workload_desc(args.workload), "block_frames": cfg.block_frames,
            "sample_rate": cfg.sample_rate, "max_voices": cfg.max_voices,
            "mix": ["f32 tree", "two-sum", "f64"][args.mix_mode], "pool_sort_every": args.sort_every,
            "parallelism": "replicas" if world > 1 else "single",
            "l2": "inputs larger than L2 (voice pool >= 1.8 GB at 8.4M voices)"
                  if args.workload.startswith("steal") else "inputs smaller than L2 between blocks"}


def run_reference(args, world):
    """The reference arm: the CPU restatement of src/cpu.rs (the oracle) on
    every host thread, on steady-state blocks of the workload. For the steal
    workloads a bounded sample: the same workload at 1/REFERENCE_SCALE of its
    pool and notes, pre-rolled on the oracle until its pool is saturated and
    stealing, then W untimed and K timed blocks; one more block on a single
    thread gives the reference's own (single-threaded) figure."""
    from kestrel_b200 import host as H
    from oracle.binding import OracleSynth
    threads = os.cpu_count() or 1
    cfg, bs, ms = H.config_workload(args.workload, seed=args.seed)
    scale = REFERENCE_SCALE.get(args.workload, 1)
    cfg.max_voices //= scale
    ms.notes //= scale
    cfg.mix_mode = args.mix_mode
    bank = H.Bank(bs, cfg)
    drv = H.Driver(cfg, bank, ms)
    orc = OracleSynth(cfg, bank.pool, bank.params, threads=threads)
    out = np.empty(cfg.block_frames * 2, np.float32)

    def block():
        live = orc.stats().active_voices
        blk = drv.prepare(live)
        t0 = time.perf_counter()
        H.feed(orc, blk)
        orc.render(out, keep_mix64=False)
        dt = time.perf_counter() - t0
        drv.finish(orc.stats().active_voices)
        return live + len(blk.cmds), dt

    t_pre = time.perf_counter()
    pre, stealing = 0, 0
    while pre < 160 and (pre < PREROLL.get(args.workload, 0) if scale == 1 else stealing < 2):
        before = orc.stats().stolen
        block()
        pre += 1
        stealing += orc.stats().stolen > before
    t_pre = time.perf_counter() - t_pre
    for _ in range(args.warmup):
        block()
    timed = [block() for _ in range(args.steps)]
    orc.threads = 1
    n1, t1 = block()
    st = orc.stats()
    orc.close()
    secs = sum(dt for _, dt in timed)
    units = sum(n for n, _ in timed) * cfg.block_frames
    return {"value": units / secs if secs > 0 else 0.0, "secs": secs, "timed": timed, "threads": threads,
            "single": n1 * cfg.block_frames / t1 if t1 > 0 else 0.0, "single_voices": n1, "preroll": pre,
            "preroll_s": t_pre, "scale": scale, "max_voices": cfg.max_voices, "notes": ms.notes,
            "stolen": st.stolen, "block_frames": cfg.block_frames, "sample_rate": cfg.sample_rate}


def main(argv=None):
    args = parse_args(argv)
    world, rank, local = dist_env()
    metric = "voice-samples/s (x-realtime beside) at 1M-8M voices"
    unit = "voice-samples/s"

    if args.impl == "reference":
        if rank != 0:
            return 0
        r = run_reference(args, world)
        value, secs, K = r["value"], r["secs"], len(r["timed"])
        mean_v = float(np.mean([n for n, _ in r["timed"]])) if K else 0.0
        sample = (f"the workload at 1/{r['scale']} of its pool and notes ({r['max_voices']:,}-voice pool, "
                  f"{r['notes']:,} notes, same durations, bank and steal percent), pre-rolled on the oracle for "
                  f"{r['preroll']} blocks until saturated and stealing, then {args.warmup} untimed and {K} timed "
                  f"steady-state blocks (mean {mean_v:,.0f} voices rendered per block)" if r["scale"] > 1 else
                  f"blocks {r['preroll'] + args.warmup}..{r['preroll'] + args.warmup + K - 1} of the workload after "
                  f"a {r['preroll']}-block pre-roll (mean {mean_v:,.0f} voices per block)")
        line = {
            "metric": metric, "value": value, "unit": unit, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs * 1e3 / max(K, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "x_realtime": (K * r["block_frames"] / r["sample_rate"]) / secs if secs > 0 else 0.0,
            "config": bench_config(args, world),
            "cpu_baseline": {"value": value, "unit": unit, "cores": r["threads"], "kind": "port",
                             "sample": sample + f"; C++ restatement of src/cpu.rs, voice loop split over "
                                                f"{r['threads']} threads"},
            # The reference backend is single-threaded (README.md:113-117):
            # the next steady-state block on one thread.
            "single_thread": {"value": r["single"], "unit": unit, "cores": 1,
                              "voices_rendered": r["single_voices"]},
            "preroll_s": r["preroll_s"], "stolen": r["stolen"],
            "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
        return 0

    if args.workload == "served":
        if rank == 0:
            print(json.dumps(run_served(args)), flush=True)
        return 0

    if world > 1:
        import datetime

        import torch
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    r = run_cuda(args, world, rank, local)

    units, ms_t, e2e_units, e2e_s = r["units"], r["ms"], r["e2e_units"], r["e2e_s"]
    if world > 1:
        units, e2e_units, ms_t, e2e_s = reduce_over_ranks(units, e2e_units, ms_t, e2e_s, "cuda")

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        c = run_oracle(args.workload, args.seed, 1, 1 << 30, args.cpu_seconds)
        cpu = {"value": c["value"], "unit": unit, "cores": 1, "kind": "port",
               "sample": f"first {c['blocks']} blocks of the workload (up to {c['live_max']} voices, "
                         f"{c['seconds']:.1f} s of CPU), C++ restatement of src/cpu.rs, one thread"}

    if rank == 0:
        K = args.steps
        peak, peak_kind = measured_peaks()
        n_render_mean = r["mean_live"]
        bytes_launch = render_algorithmic_bytes(int(round(n_render_mean)), r["bf"], r["tiles"])
        achieved = bytes_launch / (r["render_ms"] * 1e-3) / 1e9 if r["render_ms"] > 0 else 0.0
        tpu = render_profile_per_unit(args.workload, args.mix_mode)
        ipu = render_profile_per_unit(args.workload, args.mix_mode, "lane_instructions_per_voice_sample")
        sms = torch_sm_count()
        value = units / (ms_t * 1e-3)
        line = {
            "metric": metric, "value": value, "unit": unit, "n_gpus": world, "steps": K,
            "warmup": args.warmup, "ms_per_step": ms_t / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "x_realtime": (K * r["bf"] / r["sample_rate"]) / (ms_t * 1e-3),
            "config": bench_config(args, world),
            "measured": {"mean_voices_rendered": round(n_render_mean), "preroll_blocks": r["preroll"],
                         "replay_equals_host_render": r["same"], "stolen": r["stolen"],
                         "hot_path_share": r["hot_share"],
                         # the host-buffer blocks one at a time (kc_render per
                         # block, no staging ahead), rank 0
                         "e2e_serial": r["e2e_units"] / r["serial_s"] if r["serial_s"] > 0 else None},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind, "kernel": "k_render",
                         "algorithmic_bytes_per_launch": bytes_launch,
                         "launch_ms": r["render_ms"],
                         "traffic": (tpu * n_render_mean * r["bf"]) if tpu else None},
            # The same launch against instruction issue, its tighter bound: the
            # profiled instructions per voice-sample x the voice-samples of the
            # launch / its CUDA-event time, against one warp instruction per
            # scheduler per cycle (4 per SM) at the SM clock sampled meanwhile.
            "issue_roofline": issue_roofline(ipu, n_render_mean * r["bf"], r["render_ms"], sms,
                                             r["clocks"].get("sm_mhz") if r["clocks"] else None),
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_units / e2e_s if e2e_s > 0 else 0.0, "unit": unit,
                    "h2d_bytes_per_step": r["h2d"], "d2h_bytes_per_step": r["d2h"]},
            "clocks": r["clocks"],
            "gpu_launches": r["launches"],
            "passes_ms_per_block": {k: v / max(r["nblocks"], 1) for k, v in r["passes"].items()},
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
