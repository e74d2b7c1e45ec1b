"""A second, independent restatement of src/cpu.rs in plain Python.

Test infrastructure for small cases only (pure-Python loops). It exists to
check the C++ oracle: two restatements written separately from the same
source must agree bit for bit. f32 arithmetic is done with numpy float32
scalars, which round every operation to f32 as Rust does; nothing is ever
promoted to a Python float inside the voice loop.
"""
from __future__ import annotations

import numpy as np

from kestrel_b200 import native as N

f32 = np.float32
ATTACK, DECAY, SUSTAIN, RELEASE, DEAD = 0, 1, 2, 3, 4
FRAC = f32(1.0 / 4294967296.0)
INV = f32(1.0) / f32(32767.0)
M64 = (1 << 64) - 1


class PyCpuSynth:
    def __init__(self, cfg, pool, params):
        self.cfg = cfg
        self.pool_data = np.asarray(pool, np.int16)
        self.params = params
        self.variants = {}
        self.tiles = cfg.block_frames // cfg.gate_frames
        self.tf = cfg.gate_frames
        self.voices = []  # list of dicts, pool order (src/cpu.rs:24-52)
        self.gate_rows = np.zeros(self.tiles * 2048, np.uint32)
        self.chan_rows = np.zeros(self.tiles * 64, np.uint32)
        self.bend = self.gain = self.var = False
        self.stolen = self.dropped = 0

    def set_gates(self, rows):
        self.gate_rows = np.asarray(rows, np.uint32).copy()

    def set_channels(self, rows, bend, gain, variant):
        self.chan_rows = np.asarray(rows, np.uint32).copy()
        self.bend, self.gain, self.var = bend, gain, variant

    def set_params_variant(self, index, data):
        if index:
            self.variants[index] = data.copy()

    def params_of(self, variant, base):  # cpu.rs:227-238
        if variant == 0:
            return self.params[base]
        t = self.variants.get(variant)
        if t is not None and base < len(t):
            return t[base]
        return self.params[base]

    def fetch(self, base, idx):  # cpu.rs:190-194
        i = (base + idx) & 0xFFFFFFFF
        v = self.pool_data[i] if i < self.pool_data.size else 0
        return max(f32(v) * INV, f32(-1.0))

    @staticmethod
    def adv(idx, off, looping, ls, le, ln):  # cpu.rs:243-259
        raw = idx + off
        if looping:
            if raw >= le:
                span = max(le - ls, 1)
                return ls + (raw - ls) % span
            return 0 if raw < 0 else raw
        return min(max(raw, 0), ln - 1)

    def steal_key(self, v):  # cpu.rs:213-221
        if self.cfg.steal_rule != N.STEAL_QUIETEST:
            return v["id"]
        lv = v["level"]
        lv = f32(0.0) if lv < 0 else (f32(1.0) if lv > 1 else lv)
        q = int(lv * f32(65535.0)) if not np.isnan(lv) else 0
        return (q << 48) | (v["id"] & 0xFFFFFFFFFFFF)

    def _push(self, c):  # cpu.rs:59-82
        self.voices.append(dict(
            phase=(int(c["phase_hi"]) << 32) | int(c["phase_lo"]), step=(int(c["step_hi"]) << 32) | int(c["step_lo"]),
            base=int(c["smp_base"]), len=int(c["smp_len"]), ls=int(c["loop_start"]), le=int(c["loop_end"]),
            flags=int(c["flags"]), stage=ATTACK, level=f32(0.0), gl=f32(c["gain_l"]), gr=f32(c["gain_r"]),
            z1=f32(0.0), z2=f32(0.0), params=int(c["params"]), slot=int(c["gate_slot"]), ordinal=int(c["ordinal"]),
            start=int(c["start_rel"]), born=int(c["variant"]) + 1, stop=0,
            id=(int(c["note_id_hi"]) << 32) | int(c["note_id_lo"])))

    def spawn(self, cmds):  # cpu.rs:330-390
        cap, live, want = self.cfg.max_voices, len(self.voices), len(cmds)
        pick = (lambda i, w, t: i) if self.cfg.admit_rule == N.ADMIT_LOUDEST else (lambda i, w, t: i * w // t)
        if live + want > cap:
            if self.cfg.steal_rule == N.STEAL_DROP_NEW:
                take = min(want, max(cap - live, 0))
            else:
                ms = max(self.cfg.max_voices * self.cfg.max_steal_percent // 100, 1)
                need = min(live + want - cap, live, ms)
                if need:
                    order = sorted(range(live), key=lambda i: self.steal_key(self.voices[i]))[:need]
                    span = max(self.cfg.block_frames - self.cfg.steal_fade_frames, 1)
                    for i in order:
                        self.voices[i]["stop"] = (self.voices[i]["id"] & 0xFFFFFFFF) % span + 1
                    self.stolen += need
                take = min(want, cap - (live - need))
            self.dropped += want - take
            for i in range(take):
                self._push(cmds[pick(i, want, take)])
            return
        for c in cmds:
            self._push(c)

    def render(self):  # cpu.rs:392-639
        cfg = self.cfg
        bf = cfg.block_frames
        mix = np.zeros(bf * 2, np.float64)
        floor = f32(cfg.env_floor)
        fade = cfg.steal_fade_frames
        exp_d = cfg.decay_curve == N.CURVE_EXPONENTIAL
        exp_r = cfg.release_curve == N.CURVE_EXPONENTIAL
        interp = cfg.interpolation
        for v in self.voices:
            if v["stage"] == DEAD:
                continue
            born = v["born"]
            variant = born - 1 if born else 0
            p = self.params_of(variant, v["params"])
            use_filter = bool(p["flags"] & 1)
            looping_en, lur = bool(v["flags"] & 1), bool(v["flags"] & 2)
            ch = (v["slot"] >> 7) & 15
            gain_l, gain_r = v["gl"], v["gr"]
            step = v["step"]
            phase, stage, level, z1, z2 = v["phase"], v["stage"], v["level"], v["z1"], v["z2"]
            born_tile = v["start"] // self.tf
            dead_break = False
            for tile in range(self.tiles):
                if stage < RELEASE and self.gate_rows[tile * 2048 + v["slot"]] >= v["ordinal"]:
                    stage = RELEASE
                    level = min(level, f32(1.0))
                if self.bend or self.gain or self.var:
                    ci = (tile * 16 + ch) * 4
                    if self.bend:
                        step = min((v["step"] * int(self.chan_rows[ci])) >> 24, M64)
                    if self.gain:
                        gain_l = v["gl"] * self.chan_rows[ci + 1:ci + 2].view(np.float32)[0]
                        gain_r = v["gr"] * self.chan_rows[ci + 2:ci + 3].view(np.float32)[0]
                    if self.var:
                        want = int(self.chan_rows[ci + 3])
                        born_here = born != 0 and tile <= born_tile
                        if want != variant and not born_here:
                            variant = want
                            p = self.params_of(variant, v["params"])
                            use_filter = bool(p["flags"] & 1)
                for i in range(self.tf):
                    f = tile * self.tf + i
                    if f < v["start"]:
                        continue
                    if stage == DEAD:
                        dead_break = True
                        break
                    looping = looping_en and not (lur and stage >= RELEASE)
                    idx = phase >> 32
                    if not looping and idx >= v["len"]:
                        stage = DEAD
                        dead_break = True
                        break
                    if stage == ATTACK:
                        level = level + p["attack_rate"]
                        if level >= p["attack_end"]:
                            stage, level = DECAY, f32(1.0)
                    elif stage == DECAY:
                        level = level * p["decay_coef"] if exp_d else level - p["decay_coef"]
                        if level <= p["decay_target"]:
                            if p["sustain"] <= floor:
                                stage, level = DEAD, f32(0.0)
                            else:
                                stage, level = SUSTAIN, p["sustain"]
                    elif stage == RELEASE:
                        level = level * p["release_coef"] if exp_r else level - p["release_coef"]
                        if level <= floor:
                            stage, level = DEAD, f32(0.0)
                    frac = f32(phase & 0xFFFFFFFF) * FRAC
                    args = (looping, v["ls"], v["le"], v["len"])
                    if interp == N.INTERP_NEAREST:
                        s = self.fetch(v["base"], idx)
                    elif interp == N.INTERP_LINEAR:
                        s0 = self.fetch(v["base"], idx)
                        s1 = self.fetch(v["base"], self.adv(idx, 1, *args))
                        s = s0 + (s1 - s0) * frac
                    else:
                        sm1 = self.fetch(v["base"], self.adv(idx, -1, *args))
                        s0 = self.fetch(v["base"], idx)
                        s1 = self.fetch(v["base"], self.adv(idx, 1, *args))
                        s2 = self.fetch(v["base"], self.adv(idx, 2, *args))
                        a = f32(-0.5) * sm1 + f32(1.5) * s0 - f32(1.5) * s1 + f32(0.5) * s2
                        b = sm1 - f32(2.5) * s0 + f32(2.0) * s1 - f32(0.5) * s2
                        c = f32(-0.5) * sm1 + f32(0.5) * s1
                        s = ((a * frac + b) * frac + c) * frac + s0
                    x = s * min(level, f32(1.0))
                    if use_filter:
                        y = p["b0"] * x + z1
                        z1 = p["b1"] * x - p["a1"] * y + z2
                        z2 = p["b0"] * x - p["a2"] * y
                    else:
                        y = x
                    if v["stop"] and f + 1 >= v["stop"]:
                        d = f + 1 - v["stop"]
                        if d >= fade:
                            stage, y = DEAD, f32(0.0)
                        else:
                            y = y * (f32(1.0) - f32(d) / f32(fade))
                    mix[2 * f] += float(y * gain_l)
                    mix[2 * f + 1] += float(y * gain_r)
                    phase = (phase + step) & M64
                    if looping:
                        hi = phase >> 32
                        if hi >= v["le"]:
                            span = max((v["le"] - v["ls"]) & 0xFFFFFFFF, 1)
                            phase = (((v["ls"] + (hi - v["ls"]) % span) & 0xFFFFFFFF) << 32) | (phase & 0xFFFFFFFF)
                if dead_break:
                    break
            v.update(phase=phase, stage=stage, level=level, z1=z1, z2=z2, start=0, born=0, stop=0)
        out = mix.astype(np.float32)
        self.voices = [v for v in self.voices if v["stage"] != DEAD]
        return out, mix

    def read_pool(self):
        n = len(self.voices)
        a = np.zeros((24, n), np.uint32)
        for k, v in enumerate(self.voices):
            a[:, k] = [v["phase"] & 0xFFFFFFFF, v["phase"] >> 32, v["step"] & 0xFFFFFFFF, v["step"] >> 32, v["base"],
                       v["len"], v["ls"], v["le"], v["flags"], v["stage"], f32(v["level"]).view(np.uint32),
                       f32(v["gl"]).view(np.uint32), f32(v["gr"]).view(np.uint32), f32(v["z1"]).view(np.uint32),
                       f32(v["z2"]).view(np.uint32), v["params"], 0, v["slot"], v["ordinal"], v["start"],
                       v["id"] & 0xFFFFFFFF, v["id"] >> 32, v["born"], v["stop"]]
        return a
