"""End to end: the render loop writes WAV files (driver -> backend -> output
stage -> writer, src/bin/kestrel.rs:311-365). The CUDA render and the CPU
reference render of the same workload, both through the default brickwall,
null below -100 dBFS on every sample of the file; a CUDA rerun is byte
for byte the same file.
"""
import numpy as np
import pytest

from kestrel_b200 import host as H
from kestrel_b200.render import render_file

gpu = pytest.mark.gpu


def _oracle(cfg, bank):
    from oracle.binding import OracleSynth
    return OracleSynth(cfg, bank.pool, bank.params)


def _payload(path, fmt):
    raw = path.read_bytes()
    return np.frombuffer(raw[44:], "<f4" if fmt == H.WAV_FLOAT32 else "<i2")


def test_cpu_render_loop_writes_a_wav(tmp_path):
    cfg, bs, ms = H.config_workload("plain", seed=2)
    st = render_file(tmp_path / "cpu.wav", cfg, bs, ms, backend=_oracle, max_seconds=0.5)
    x = _payload(tmp_path / "cpu.wav", H.WAV_FLOAT32)
    assert st.blocks == 6 and x.size == 6 * cfg.block_frames * 2
    assert float(np.max(np.abs(x))) <= 1.0 and np.any(x != 0)
    assert st.latency_frames == 96 + 3   # 2 ms lookahead + the detector's group delay


@gpu
@pytest.mark.parametrize("limiter", [H.LIMITER_BRICKWALL, H.LIMITER_OMNI, H.LIMITER_OFF])
def test_cuda_wav_nulls_against_the_cpu_reference(tmp_path, limiter):
    cfg, bs, ms = H.config_workload("plain", seed=4)
    a = render_file(tmp_path / "cuda.wav", cfg, bs, ms, limiter=limiter, max_seconds=2.0)
    b = render_file(tmp_path / "cpu.wav", cfg, bs, ms, backend=_oracle, limiter=limiter, max_seconds=2.0)
    assert a.blocks == b.blocks and a.clipped == b.clipped
    x, y = _payload(tmp_path / "cuda.wav", H.WAV_FLOAT32), _payload(tmp_path / "cpu.wav", H.WAV_FLOAT32)
    assert x.size == y.size
    d = float(np.max(np.abs(x.astype(np.float64) - y.astype(np.float64))))
    assert d == 0.0 or 20 * np.log10(d) <= -100.0
    c = render_file(tmp_path / "cuda2.wav", cfg, bs, ms, limiter=limiter, max_seconds=2.0)
    assert (tmp_path / "cuda.wav").read_bytes() == (tmp_path / "cuda2.wav").read_bytes()
    assert c.blocks == a.blocks


@gpu
def test_pcm16_render(tmp_path):
    cfg, bs, ms = H.config_workload("plain", seed=5)
    render_file(tmp_path / "a.wav", cfg, bs, ms, fmt=H.WAV_PCM16, max_seconds=1.0)
    render_file(tmp_path / "b.wav", cfg, bs, ms, backend=_oracle, fmt=H.WAV_PCM16, max_seconds=1.0)
    x, y = _payload(tmp_path / "a.wav", H.WAV_PCM16), _payload(tmp_path / "b.wav", H.WAV_PCM16)
    # A -100 dB null is far below one pcm16 step: the files differ by at most one code, rarely
    assert np.max(np.abs(x.astype(np.int32) - y.astype(np.int32))) <= 1


def test_cli_maps_the_reference_render_flags(tmp_path, monkeypatch):
    """`python -m kestrel_b200.render song.mid -s bank.sf2 -o out.wav ...`
    takes `kestrel render`'s options (src/bin/kestrel.rs:72-187, spellings
    of src/config.rs:20-150) to the config, the driver options and the
    output stage."""
    from kestrel_b200 import native as N
    from kestrel_b200 import render as R
    seen = {}

    def fake(path, cfg, bank, midi, backend, limiter, fmt, max_seconds, pipelined, options, limiter_opts, block_csv,
             nan_guard, progress):
        seen.update(path=path, cfg=cfg, bank=bank, midi=midi, limiter=limiter, fmt=fmt, seconds=max_seconds,
                    pipelined=pipelined, opt=options, lim=limiter_opts, csv=block_csv, nan=nan_guard, prog=progress)
        return R.RenderStats(1, 0.1, 0.1, 0, 0, 0, 0)

    monkeypatch.setattr(R, "render_file", fake)
    R.main(["song.mid", "-s", "bank.sf2", "-o", str(tmp_path / "o.wav"), "--rate", "44100", "--block", "2048",
            "--max-voices", "5000", "--interp", "hermite", "--decay-curve", "lin", "--steal", "drop-new",
            "--admit", "spread", "--steal-percent", "50", "--format", "pcm16", "--volume", "0.5", "--layers", "4",
            "--ceiling-db", "-1", "--no-true-peak", "--no-filter", "--no-sort", "--no-resample-pool",
            "--pool-budget", "64", "--seconds", "3", "--serial", "--block-csv", "b.csv", "--nan-guard", "--quiet"])
    c, o = seen["cfg"], seen["opt"]
    assert seen["midi"] == "song.mid" and seen["bank"] == "bank.sf2"
    assert (c.sample_rate, c.block_frames, c.max_voices, c.max_steal_percent) == (44100, 2048, 5000, 50)
    assert (c.interpolation, c.decay_curve, c.steal_rule, c.admit_rule, c.sort_voices) == \
        (N.INTERP_CUBIC, N.CURVE_LINEAR, N.STEAL_DROP_NEW, N.ADMIT_EVEN, 0)
    assert (o.filter_enabled, o.resample_pool, o.sample_pool_budget, o.max_layers) == (0, 0, 64 << 20, 4)
    assert abs(o.master_volume - 0.5) < 1e-7
    assert seen["fmt"] == H.WAV_PCM16 and seen["seconds"] == 3.0 and seen["pipelined"] is False
    assert seen["lim"]["ceiling_db"] == -1.0 and seen["lim"]["true_peak"] is False and seen["csv"] == "b.csv"
    assert seen["nan"] is True and seen["prog"] is None
    R.main(["-o", str(tmp_path / "o.wav"), "--no-limiter"])
    assert seen["limiter"] == H.LIMITER_OFF and seen["pipelined"] is None
    with pytest.raises(SystemExit):
        R.main(["x.mid", "-o", "y.wav", "--steal", "loudest"])


def test_nan_guard_stops_at_a_non_finite_block(tmp_path):
    """--nan-guard: a block holding a NaN ends the render with an error (the
    NaN is planted in the CPU reference's output)."""
    class Planted:
        def __init__(self, cfg, bank):
            self.o, self.n = _oracle(cfg, bank), 0
            self.block_frames = cfg.block_frames

        def __getattr__(self, name):
            return getattr(self.o, name)

        def render(self):
            out = self.o.render()
            self.n += 1
            if self.n == 3:
                out[5] = np.nan
            return out

    cfg, bs, ms = H.config_workload("plain", seed=2)
    render_file(tmp_path / "ok.wav", cfg, bs, ms, backend=Planted, max_seconds=0.3)   # unguarded: runs on
    with pytest.raises(FloatingPointError, match="block 2"):
        render_file(tmp_path / "x.wav", cfg, bs, ms, backend=Planted, max_seconds=0.3, nan_guard=True)
