"""The precision sweep: mix arithmetic and low-cutoff biquad design.

    python -m kestrel_b200.precision [--voices 4194304] [--blocks 6] [--json out.json]

Part 1, dense mix. The black-MIDI workload's bank (128 presets, per-preset
envelopes and filters) and a dense event stream that fills a pool of up to
`voices` concurrent voices. Three contexts render the identical blocks (one
driver feeds all three, so every voice's f32 contribution is the same bits in
each): the fixed-order f32 tree, the compensated two-sum tree, and the FP64
accumulation of the same f32 terms, which is the FP64 mix oracle (on the
device: the CPU oracle's f64 mix at this size would take minutes per block).
Reported per block: peak and RMS |mix - f64 mix| in dBFS and relative to the
block's peak.

Part 2, biquad design at cutoffs 20-200 Hz and Q up to 20. Coefficients from
the reference's f32 design (biquad_lowpass, src/bank.rs:956-979, restated in
the host library) and from the FP64 design on the device
(kc_design_lowpass_f64), each run through the f32 TDF-II recursion the
render uses, against the exact design run in f64. Reported: DC-gain error and
the output error on a test signal.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import sys
import time

import numpy as np

from . import host as H
from . import native as N
from .backend import CudaSynth


def _db(x: float) -> float:
    return -np.inf if x <= 0 else 20.0 * np.log10(x)


def dense_mix(voices: int, blocks: int, seed: int = 1) -> list[dict]:
    cfg, bs, ms = H.config_workload("black", seed=seed)
    cfg.max_voices = voices
    # Dense: twice `voices` note-ons per second with 2 s notes, so the pool
    # fills within about six blocks and then stays full.
    ms.notes = int(voices * 16)
    ms.seconds = 8.0
    ms.dur_median_s = 2.0
    ms.dur_sigma = 0.5
    ms.cluster_share = 0.0
    bank = H.Bank(bs, cfg)
    drv = H.Driver(cfg, bank, ms)
    ctx = {}
    for name, mode in (("f32_tree", N.MIX_F32_TREE), ("two_sum", N.MIX_TWO_SUM), ("f64", N.MIX_F64)):
        c = N.default_config(**{f: getattr(cfg, f) for f, _ in N.KcConfig._fields_ if f != "reserved"})
        c.mix_mode = mode
        ctx[name] = CudaSynth(c, bank.pool, bank.params, bank.regions, bank.max_sample_len)
    rows = []
    for b in range(blocks):
        live = ctx["f64"].stats().active_voices
        blk = drv.prepare(live)
        outs = {}
        for name, s in ctx.items():
            H.feed(s, blk)
            outs[name] = s.render().astype(np.float64)
        counts = {s.stats().active_voices for s in ctx.values()}
        assert len(counts) == 1, "contexts diverged"
        ref = outs["f64"]
        peak = float(np.max(np.abs(ref)))
        row = {"block": b, "voices_rendered": int(live + len(blk.cmds)), "ref_peak": peak}
        for name in ("f32_tree", "two_sum"):
            d = outs[name] - ref
            row[name] = {"peak_dbfs": _db(float(np.max(np.abs(d)))), "rms_dbfs": _db(float(np.sqrt(np.mean(d * d)))),
                         "peak_rel_db": _db(float(np.max(np.abs(d))) / peak) if peak > 0 else None}
        rows.append(row)
        drv.finish(live)
    for s in ctx.values():
        s.close()
    return rows


def _tdf2_f32(x: np.ndarray, coefs: np.ndarray) -> np.ndarray:
    """The render's f32 TDF-II recursion (src/cpu.rs:564-572), vectorised over
    filters: every operation is an elementwise f32 op, rounded like the
    device's strict path."""
    b0, b1, a1, a2 = (coefs[:, i].astype(np.float32) for i in range(4))
    z1 = np.zeros(coefs.shape[0], np.float32)
    z2 = np.zeros(coefs.shape[0], np.float32)
    y = np.empty((coefs.shape[0], x.size), np.float32)
    for t, xv in enumerate(x.astype(np.float32)):
        yt = b0 * xv + z1
        z1 = b1 * xv - a1 * yt + z2
        z2 = b0 * xv - a2 * yt
        y[:, t] = yt
    return y


def _tdf2_f64(x: np.ndarray, coefs: np.ndarray) -> np.ndarray:
    b0, b1, a1, a2 = (coefs[:, i] for i in range(4))
    z1 = np.zeros(coefs.shape[0])
    z2 = np.zeros(coefs.shape[0])
    y = np.empty((coefs.shape[0], x.size))
    for t, xv in enumerate(x.astype(np.float64)):
        yt = b0 * xv + z1
        z1 = b1 * xv - a1 * yt + z2
        z2 = b0 * xv - a2 * yt
        y[:, t] = yt
    return y


def _design_exact(fc, q_cb, sr):
    q = np.maximum(10.0 ** ((q_cb / 10.0 - 3.01) / 20.0), 0.001)
    gain = np.sqrt(np.sqrt(0.5) / q)
    w0 = 2 * np.pi * np.clip(fc / sr, 1e-5, 0.49)
    omc = 2 * np.sin(w0 / 2) ** 2
    alpha = np.sin(w0) / (2 * q)
    a0 = 1 + alpha
    return np.stack([gain * omc * 0.5 / a0, gain * omc / a0, -2 * np.cos(w0) / a0, (1 - alpha) / a0], axis=1)


def biquad_sweep(sr: float = 48000.0, seconds: float = 1.0, device: int = 0) -> list[dict]:
    fcs = np.geomspace(20.0, 200.0, 8)
    qs = np.array([0.7071, 2.0, 5.0, 10.0, 20.0])
    grid = [(f, q) for f in fcs for q in qs]
    fc = np.array([g[0] for g in grid], np.float32)
    q_cb = np.array([(20 * np.log10(g[1]) + 3.01) * 10 for g in grid], np.float32)
    f32 = np.array([H.biquad_lowpass(float(f), float(q), sr) for f, q in zip(fc, q_cb)], np.float32)
    f64 = np.empty((len(grid), 4), np.float32)
    lib = N.cuda_lib()
    N.check(lib.kc_design_lowpass_f64(N.ptr(fc), N.ptr(q_cb), len(grid), sr, N.ptr(f64), device), lib)
    exact = _design_exact(fc.astype(np.float64), q_cb.astype(np.float64), sr)
    rng = np.random.default_rng(3)
    n = int(sr * seconds)
    x = (0.25 * rng.standard_normal(n) + 0.5 * np.sin(2 * np.pi * 55.0 * np.arange(n) / sr)).astype(np.float32)
    y_ref = _tdf2_f64(x, exact)
    y32 = _tdf2_f32(x, f32).astype(np.float64)
    y64 = _tdf2_f32(x, f64).astype(np.float64)

    def dc(c):
        c = c.astype(np.float64)
        return (2 * c[:, 0] + c[:, 1]) / (1 + c[:, 2] + c[:, 3])

    dc_ref, dc32, dc64 = dc(exact), dc(f32), dc(f64)
    rows = []
    for i, (f, q) in enumerate(grid):
        pk = float(np.max(np.abs(y_ref[i])))
        e32, e64 = y32[i] - y_ref[i], y64[i] - y_ref[i]
        rows.append({
            "fc_hz": round(float(f), 2), "q": float(q),
            "dc_gain_err_db_f32_design": float(20 * np.log10(abs(dc32[i] / dc_ref[i]))),
            "dc_gain_err_db_f64_design": float(20 * np.log10(abs(dc64[i] / dc_ref[i]))),
            "out_peak_err_rel_db_f32_design": _db(float(np.max(np.abs(e32))) / pk),
            "out_peak_err_rel_db_f64_design": _db(float(np.max(np.abs(e64))) / pk),
            "out_rms_err_rel_db_f32_design": _db(float(np.sqrt(np.mean(e32 ** 2))) / pk),
            "out_rms_err_rel_db_f64_design": _db(float(np.sqrt(np.mean(e64 ** 2))) / pk),
        })
    return rows


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--voices", type=int, default=4 * 1024 * 1024)
    ap.add_argument("--blocks", type=int, default=10)
    ap.add_argument("--json", default=None)
    ap.add_argument("--skip-mix", action="store_true")
    args = ap.parse_args(argv)
    res = {}
    t = time.time()
    if not args.skip_mix:
        res["dense_mix"] = dense_mix(args.voices, args.blocks)
    res["biquad"] = biquad_sweep()
    res["seconds"] = time.time() - t
    text = json.dumps(res, indent=1)
    if args.json:
        with open(args.json, "w") as f:
            f.write(text)
    print(text)
    return 0


if __name__ == "__main__":
    sys.exit(main())
