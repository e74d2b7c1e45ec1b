"""The load-time resampler on the device against the host loop.

kc_resample_i16_batch must reproduce SincBank::process (src/resample.rs:
51-107, restated in the host library) bit for bit: edge taps clamped at the
ends of short sources, downsampling with the narrowed cutoff, saturation of
over-range sums, several ratios (and so several sinc tables) in one batch.
Installed as the bank builder's resampler, it must leave a bank's pool
byte-identical.
"""
import ctypes as C

import numpy as np
import pytest

from kestrel_b200 import host as H
from kestrel_b200 import native as N

gpu = pytest.mark.gpu


def _out_len(n, ratio):
    """max(round(n * ratio), 1) with f64::round, which rounds halves away from zero."""
    return max(int(np.floor(n * ratio + 0.5)), 1)


def _host(src, ratio):
    out = np.empty(_out_len(src.size, ratio) + 1, np.int16)
    n = H.lib().kh_resample_i16(N.ptr(src), src.size, ratio, N.ptr(out), out.size)
    return out[:n].copy()


def test_sinc_table_rows_sum_to_one():
    for ratio in (48000 / 44100, 44100 / 48000, 0.5):
        t = H.sinc_table(ratio).astype(np.float64)
        assert t.shape == (512, 32)
        assert np.all(np.abs(t.sum(axis=1) - 1.0) < 1e-5)


@gpu
def test_device_batch_matches_host_loop():
    rng = np.random.default_rng(7)
    ratios = [48000 / 44100, 44100 / 48000, 2.0, 0.5, 48000 / 22050, 0.37, 3.3]
    lengths = [1, 2, 5, 31, 32, 33, 1000, 40000]
    srcs, rs = [], []
    for i, n in enumerate(lengths * 2):
        kind = i % 3
        if kind == 0:
            x = rng.integers(-32768, 32768, n)
        elif kind == 1:  # full-scale square: sums overshoot and must saturate
            x = np.where((np.arange(n) // 7) % 2 == 0, 32767, -32768)
        else:
            x = np.round(20000 * np.sin(np.arange(n) * 0.05))
        srcs.append(x.astype(np.int16))
        rs.append(ratios[i % len(ratios)])
    tabs = [H.sinc_table(r) for r in rs]
    outs = [np.empty(_out_len(s.size, r), np.int16) for s, r in zip(srcs, rs)]
    n = len(srcs)
    P = C.c_void_p * n
    src_p = P(*[s.ctypes.data for s in srcs])
    tab_p = P(*[t.ctypes.data for t in tabs])
    dst_p = P(*[o.ctypes.data for o in outs])
    src_len = np.array([s.size for s in srcs], np.uint32)
    dst_len = np.array([o.size for o in outs], np.uint32)
    rat = np.array(rs, np.float64)
    lib = N.cuda_lib()
    N.check(lib.kc_resample_i16_batch(None, n, src_p, N.ptr(src_len), N.ptr(rat), tab_p, dst_p, N.ptr(dst_len)), lib)
    for s, r, o in zip(srcs, rs, outs):
        np.testing.assert_array_equal(o, _host(s, r), err_msg=f"len {s.size} ratio {r}")


@gpu
def test_device_resampler_rejects_wrong_output_length():
    s = np.zeros(100, np.int16)
    o = np.empty(50, np.int16)
    t = H.sinc_table(2.0)
    P = C.c_void_p * 1
    lib = N.cuda_lib()
    rc = lib.kc_resample_i16_batch(None, 1, P(s.ctypes.data), N.ptr(np.array([100], np.uint32)),
                                   N.ptr(np.array([2.0])), P(t.ctypes.data), P(o.ctypes.data),
                                   N.ptr(np.array([50], np.uint32)))
    assert rc == 1 and b"round" in lib.kc_last_error()


@gpu
def test_bank_built_with_the_device_resampler_is_identical():
    cfg = N.default_config(max_voices=65536)
    for spec in (H.bank_spec(presets=1, seed=4), H.bank_spec(presets=16, random_generators=1, sample_rate=22050,
                                                             sample_frames=12000, loop_frames=3000, seed=5)):
        ref = H.Bank(spec, cfg)
        H.use_device_resampler(0)
        try:
            dev = H.Bank(spec, cfg)
        finally:
            H.use_device_resampler(None)
        assert ref.pool.tobytes() == dev.pool.tobytes()
        assert ref.params.tobytes() == dev.params.tobytes()
        assert ref.max_sample_len == dev.max_sample_len
