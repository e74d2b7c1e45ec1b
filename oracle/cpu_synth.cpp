// cpu_synth.cpp -- CPU restatement of Kestrel's reference backend (src/cpu.rs).
//
// TEST INFRASTRUCTURE: the checker, never the thing measured or shipped. Only
// tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs load it.
//
// Compiled with -O2 -ffp-contract=off (never -ffast-math) so every f32
// expression rounds exactly where the Rust source rounds: Rust never contracts
// a*b+c into an FMA, and neither may this file. Rust's float->int `as` casts
// saturate (NaN -> 0); the helpers below reproduce that explicitly because the
// C++ casts are undefined out of range.
//
// Parity status: pinned against the reference's in-module known-answer tests
// and analytic answers only (see oracle.h); block-level parity with the Rust
// binary is unpinned because the crate cannot be built in this image.

#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

namespace {

constexpr uint32_t ENV_ATTACK = 0, ENV_DECAY = 1, ENV_SUSTAIN = 2, ENV_RELEASE = 3,
                   ENV_DEAD = 4;
constexpr size_t GATE_SLOTS = 2048;
constexpr size_t BEND_CHANNELS = 16, CHAN_FIELDS = 4;
constexpr uint32_t VF_LOOP = 1, VF_LOOP_UNTIL_RELEASE = 2, RP_FILTER = 1;
constexpr float FRAC_SCALE_F32 = 1.0f / 4294967296.0f;  // src/fixed.rs:15

// f32::max / f32::min: IEEE maxNum/minNum, the non-NaN operand wins.
inline float rmax(float a, float b) { return std::fmax(a, b); }
inline float rmin(float a, float b) { return std::fmin(a, b); }
// f32::clamp: NaN stays NaN (src/cpu.rs:218 relies on `as u32` mapping it to 0).
inline float rclamp(float v, float lo, float hi) {
    if (v < lo) v = lo;
    if (v > hi) v = hi;
    return v;
}
// `f as u32`, saturating.
inline uint32_t f32_as_u32(float v) {
    if (!(v > 0.0f)) return 0;  // NaN and <= 0
    if (v >= 4294967296.0f) return 0xFFFFFFFFu;
    return (uint32_t)v;
}

// ---- fixed.rs ---------------------------------------------------------------

// Fixed::scale, src/fixed.rs:83-90: (u128 product) >> 24, saturating.
inline uint64_t fixed_scale(uint64_t v, uint32_t factor) {
    unsigned __int128 p = ((unsigned __int128)v * factor) >> 24;
    if (p > (unsigned __int128)UINT64_MAX) return UINT64_MAX;
    return (uint64_t)p;
}

// ---- config.rs ---------------------------------------------------------------

// Config::max_steal, src/config.rs:549-552.
inline uint32_t max_steal(const kc_config& c) {
    uint64_t n = (uint64_t)c.max_voices * c.max_steal_percent / 100;
    uint32_t v = (uint32_t)n;
    return v > 1 ? v : 1;
}
// Config::steal_span, src/config.rs:534-536.
inline uint32_t steal_span(const kc_config& c) {
    uint32_t s = c.block_frames > c.steal_fade_frames ? c.block_frames - c.steal_fade_frames : 0;
    return s > 1 ? s : 1;
}

// voice::spawn_pick, src/voice.rs:71-75.
inline size_t spawn_pick(size_t i, size_t want, size_t take) {
    return (size_t)((uint64_t)i * (uint64_t)want / (uint64_t)take);
}

// catmull_rom, src/cpu.rs:295-302. Left-to-right evaluation, no contraction.
inline float catmull_rom(float sm1, float s0, float s1, float s2, float t) {
    float a = -0.5f * sm1 + 1.5f * s0 - 1.5f * s1 + 0.5f * s2;
    float b = sm1 - 2.5f * s0 + 2.0f * s1 - 0.5f * s2;
    float c = -0.5f * sm1 + 0.5f * s1;
    return ((a * t + b) * t + c) * t + s0;
}

// Pool, src/cpu.rs:21-142: one vector per field; phase/step as u64.
struct Pool {
    std::vector<uint64_t> phase, step;
    std::vector<uint32_t> smp_base, smp_len, loop_start, loop_end, flags, env_stage;
    std::vector<float> env_level, gain_l, gain_r, filt_z1, filt_z2;
    std::vector<uint32_t> params, region, gate_slot, ordinal, start_rel, born_variant, stop_rel;
    std::vector<uint64_t> note_id;

    size_t len() const { return phase.size(); }

    // Pool::push, src/cpu.rs:59-82.
    void push(const kc_spawn_cmd& c) {
        phase.push_back(((uint64_t)c.phase_hi << 32) | c.phase_lo);
        step.push_back(((uint64_t)c.step_hi << 32) | c.step_lo);
        smp_base.push_back(c.smp_base);
        smp_len.push_back(c.smp_len);
        loop_start.push_back(c.loop_start);
        loop_end.push_back(c.loop_end);
        flags.push_back(c.flags);
        env_stage.push_back(ENV_ATTACK);
        env_level.push_back(0.0f);
        gain_l.push_back(c.gain_l);
        gain_r.push_back(c.gain_r);
        filt_z1.push_back(0.0f);
        filt_z2.push_back(0.0f);
        params.push_back(c.params);
        region.push_back(c.region);
        gate_slot.push_back(c.gate_slot);
        ordinal.push_back(c.ordinal);
        start_rel.push_back(c.start_rel);
        born_variant.push_back(c.variant + 1);
        stop_rel.push_back(0);
        note_id.push_back(((uint64_t)c.note_id_hi << 32) | c.note_id_lo);
    }

    template <class V>
    static void keep_into(V& v, const std::vector<char>& keep) {
        size_t w = 0;
        for (size_t r = 0; r < keep.size(); ++r)
            if (keep[r]) v[w++] = v[r];
        v.resize(w);
    }

    // Pool::swap_remove_compact, src/cpu.rs:84-117: stable, order-preserving.
    void compact(const std::vector<char>& keep) {
        keep_into(phase, keep); keep_into(step, keep); keep_into(smp_base, keep);
        keep_into(smp_len, keep); keep_into(loop_start, keep); keep_into(loop_end, keep);
        keep_into(flags, keep); keep_into(env_stage, keep); keep_into(env_level, keep);
        keep_into(gain_l, keep); keep_into(gain_r, keep); keep_into(filt_z1, keep);
        keep_into(filt_z2, keep); keep_into(params, keep); keep_into(region, keep);
        keep_into(gate_slot, keep); keep_into(ordinal, keep); keep_into(start_rel, keep);
        keep_into(born_variant, keep); keep_into(stop_rel, keep); keep_into(note_id, keep);
    }
};

}  // namespace

struct ko_synth {
    kc_config cfg;
    std::vector<int16_t> pool_data;
    std::vector<kc_region_params> bank_params;
    Pool pool;
    std::vector<double> mix;
    std::vector<uint32_t> gate_rows, chan_rows;
    std::vector<std::vector<kc_region_params>> variants;  // entry i holds variant i+1
    bool bend_active = false, gain_active = false, variant_active = false;
    size_t tiles = 0, tile_frames = 0;
    uint64_t stolen = 0, dropped = 0;
    float peak = 0.0f;

    // CpuSynth::fetch, src/cpu.rs:187-194: out of range reads as 0.
    inline float fetch(uint32_t base, uint32_t idx) const {
        size_t i = (size_t)(uint32_t)(base + idx);
        int16_t v = i < pool_data.size() ? pool_data[i] : 0;
        return rmax((float)v * (1.0f / 32767.0f), -1.0f);
    }

    // CpuSynth::pick, src/cpu.rs:200-206.
    inline size_t pick(size_t i, size_t want, size_t take) const {
        return cfg.admit_rule == KC_ADMIT_LOUDEST ? i : spawn_pick(i, want, take);
    }

    // CpuSynth::steal_key, src/cpu.rs:212-221.
    inline uint64_t steal_key(size_t i) const {
        uint64_t id = pool.note_id[i];
        if (cfg.steal_rule != KC_STEAL_QUIETEST) return id;
        float level = rclamp(pool.env_level[i], 0.0f, 1.0f);
        uint64_t q = (uint64_t)f32_as_u32(level * 65535.0f);
        return (q << 48) | (id & 0x0000FFFFFFFFFFFFull);
    }

    // CpuSynth::params_of, src/cpu.rs:227-238.
    inline kc_region_params params_of(uint32_t variant, size_t base) const {
        if (variant == 0) return bank_params[base];
        size_t i = variant - 1;
        if (i < variants.size() && base < variants[i].size()) return variants[i][base];
        return bank_params[base];
    }

    // CpuSynth::advance_index, src/cpu.rs:242-259.
    static inline uint32_t advance_index(uint32_t idx, int32_t off, bool looping,
                                         uint32_t loop_start, uint32_t loop_end, uint32_t len) {
        int64_t raw = (int64_t)idx + off;
        if (looping) {
            int64_t ls = loop_start, le = loop_end;
            if (raw >= le) {
                int64_t span = std::max<int64_t>(le - ls, 1);
                return (uint32_t)(ls + (raw - ls) % span);
            } else if (raw < 0) {
                return 0;
            }
            return (uint32_t)raw;
        }
        return (uint32_t)std::clamp<int64_t>(raw, 0, (int64_t)len - 1);
    }

    // CpuSynth::interpolate, src/cpu.rs:261-292.
    inline float interpolate(uint32_t base, uint32_t idx, float frac, bool looping,
                             uint32_t ls, uint32_t le, uint32_t len) const {
        switch (cfg.interpolation) {
            case KC_INTERP_NEAREST:
                return fetch(base, idx);
            case KC_INTERP_LINEAR: {
                uint32_t i1 = advance_index(idx, 1, looping, ls, le, len);
                float s0 = fetch(base, idx);
                float s1 = fetch(base, i1);
                return s0 + (s1 - s0) * frac;
            }
            default: {
                uint32_t im1 = advance_index(idx, -1, looping, ls, le, len);
                uint32_t i1 = advance_index(idx, 1, looping, ls, le, len);
                uint32_t i2 = advance_index(idx, 2, looping, ls, le, len);
                return catmull_rom(fetch(base, im1), fetch(base, idx), fetch(base, i1),
                                   fetch(base, i2), frac);
            }
        }
    }

    // One voice of CpuSynth::render, src/cpu.rs:403-613, accumulating into `mix`.
    void render_voice(size_t v, double* mix) {
        const uint32_t stage0 = pool.env_stage[v];
        if (stage0 == ENV_DEAD) return;
        const bool exp_decay = cfg.decay_curve == KC_CURVE_EXPONENTIAL;
        const bool exp_release = cfg.release_curve == KC_CURVE_EXPONENTIAL;
        const float floor = cfg.env_floor;
        const size_t fade = cfg.steal_fade_frames;

        const size_t params_base = pool.params[v];
        const uint32_t born_variant = pool.born_variant[v];
        uint32_t variant = born_variant > 0 ? born_variant - 1 : 0;
        kc_region_params p = params_of(variant, params_base);
        bool use_filter = (p.flags & RP_FILTER) != 0;

        const uint32_t base = pool.smp_base[v];
        const uint32_t len = pool.smp_len[v];
        const uint32_t loop_start = pool.loop_start[v];
        const uint32_t loop_end = pool.loop_end[v];
        const uint32_t vflags = pool.flags[v];
        const bool loop_enabled = (vflags & VF_LOOP) != 0;
        const bool loop_until_release = (vflags & VF_LOOP_UNTIL_RELEASE) != 0;
        const size_t gate_slot = pool.gate_slot[v];
        const uint32_t ordinal = pool.ordinal[v];
        const float base_gain_l = pool.gain_l[v];
        const float base_gain_r = pool.gain_r[v];
        float gain_l = base_gain_l, gain_r = base_gain_r;
        const uint64_t base_step = pool.step[v];
        const size_t channel = (gate_slot >> 7) & 15;  // ChannelTable::channel_of
        uint64_t step = base_step;

        uint64_t phase = pool.phase[v];
        uint32_t stage = stage0;
        float level = pool.env_level[v];
        float z1 = pool.filt_z1[v], z2 = pool.filt_z2[v];
        const size_t start_rel = pool.start_rel[v];
        const size_t stop_rel = pool.stop_rel[v];
        const size_t born_tile = start_rel / tile_frames;

        for (size_t tile = 0; tile < tiles; ++tile) {
            // Note-off gate, src/cpu.rs:450-456.
            if (stage < ENV_RELEASE && gate_rows[tile * GATE_SLOTS + gate_slot] >= ordinal) {
                stage = ENV_RELEASE;
                level = rmin(level, 1.0f);
            }
            // Channel controller path, src/cpu.rs:458-487.
            if (bend_active || gain_active || variant_active) {
                size_t ci = (tile * BEND_CHANNELS + channel) * CHAN_FIELDS;
                if (bend_active) step = fixed_scale(base_step, chan_rows[ci + KC_CHAN_BEND]);
                if (gain_active) {
                    float gl, gr;
                    std::memcpy(&gl, &chan_rows[ci + KC_CHAN_GAIN_L], 4);
                    std::memcpy(&gr, &chan_rows[ci + KC_CHAN_GAIN_R], 4);
                    gain_l = base_gain_l * gl;
                    gain_r = base_gain_r * gr;
                }
                if (variant_active) {
                    uint32_t want = chan_rows[ci + KC_CHAN_VARIANT];
                    bool born_here = born_variant != 0 && tile <= born_tile;
                    if (want != variant && !born_here) {
                        variant = want;
                        p = params_of(variant, params_base);
                        use_filter = (p.flags & RP_FILTER) != 0;
                    }
                }
            }

            const size_t f0 = tile * tile_frames;
            for (size_t i = 0; i < tile_frames; ++i) {
                const size_t f = f0 + i;
                if (f < start_rel) continue;
                if (stage == ENV_DEAD) goto done;

                const bool looping = loop_enabled && !(loop_until_release && stage >= ENV_RELEASE);
                const uint32_t idx = (uint32_t)(phase >> 32);
                if (!looping && idx >= len) {
                    stage = ENV_DEAD;
                    goto done;
                }

                // Envelope before the sample, src/cpu.rs:508-549.
                switch (stage) {
                    case ENV_ATTACK:
                        level += p.attack_rate;
                        if (level >= p.attack_end) {
                            stage = ENV_DECAY;
                            level = 1.0f;
                        }
                        break;
                    case ENV_DECAY:
                        level = exp_decay ? level * p.decay_coef : level - p.decay_coef;
                        if (level <= p.decay_target) {
                            if (p.sustain <= floor) {
                                stage = ENV_DEAD;
                                level = 0.0f;
                            } else {
                                stage = ENV_SUSTAIN;
                                level = p.sustain;
                            }
                        }
                        break;
                    case ENV_RELEASE:
                        level = exp_release ? level * p.release_coef : level - p.release_coef;
                        if (level <= floor) {
                            stage = ENV_DEAD;
                            level = 0.0f;
                        }
                        break;
                    default:
                        break;
                }

                const float s = interpolate(base, idx, (float)(uint32_t)phase * FRAC_SCALE_F32,
                                            looping, loop_start, loop_end, len);
                const float g = rmin(level, 1.0f);
                const float x = s * g;
                // Transposed direct form II, b2 == b0 (src/cpu.rs:564-572).
                float y;
                if (use_filter) {
                    y = p.b0 * x + z1;
                    z1 = p.b1 * x - p.a1 * y + z2;
                    z2 = p.b0 * x - p.a2 * y;
                } else {
                    y = x;
                }
                // Steal fade after the filter, src/cpu.rs:574-587.
                if (stop_rel != 0 && f + 1 >= stop_rel) {
                    size_t d = f + 1 - stop_rel;
                    if (d >= fade) {
                        stage = ENV_DEAD;
                        y = 0.0f;
                    } else {
                        y = y * (1.0f - (float)d / (float)fade);
                    }
                }
                mix[f * 2] += (double)(y * gain_l);
                mix[f * 2 + 1] += (double)(y * gain_r);

                // Phase advance and loop wrap, src/cpu.rs:592-601.
                phase = phase + step;
                if (looping) {
                    uint32_t hi = (uint32_t)(phase >> 32);
                    if (hi >= loop_end) {
                        uint32_t span = std::max<uint32_t>(loop_end - loop_start, 1);
                        uint32_t wrapped = loop_start + (hi - loop_start) % span;
                        phase = ((uint64_t)wrapped << 32) | (uint32_t)phase;
                    }
                }
            }
        }
    done:
        // Writeback, src/cpu.rs:605-612.
        pool.phase[v] = phase;
        pool.env_stage[v] = stage;
        pool.env_level[v] = level;
        pool.filt_z1[v] = z1;
        pool.filt_z2[v] = z2;
        pool.start_rel[v] = 0;
        pool.born_variant[v] = 0;
        pool.stop_rel[v] = 0;
    }
};

extern "C" {

uint32_t ko_max_steal(const kc_config* c) { return max_steal(*c); }
uint32_t ko_steal_span(const kc_config* c) { return steal_span(*c); }
// Config::pool_slots, src/config.rs:542-544 (saturating add).
uint32_t ko_pool_slots(const kc_config* c) {
    uint64_t s = (uint64_t)c->max_voices + max_steal(*c);
    return s > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)s;
}
// Config::admit_take, src/config.rs:120-131.
uint32_t ko_admit_take(const kc_config* c, uint32_t live, uint32_t queued) {
    uint32_t cap = c->max_voices;
    uint32_t want = std::min(queued, cap);
    if (live + want <= cap) return want;
    uint32_t need = c->steal_rule == KC_STEAL_DROP_NEW
                        ? 0
                        : std::min(std::min(live + want - cap, live), max_steal(*c));
    return std::min(want, cap - (live - need));
}

// Fixed::from_f64, src/fixed.rs:24-38.
uint64_t ko_fixed_from_f64(double v) {
    double scaled = v * 18446744073709551616.0 / 4294967296.0;
    if (std::isnan(scaled) || scaled <= 0.0) return 0;
    if (scaled >= 18446744073709551615.0) return UINT64_MAX;
    return (uint64_t)scaled;
}
uint64_t ko_fixed_scale(uint64_t v, uint32_t factor) { return fixed_scale(v, factor); }
// bend_factor, src/fixed.rs:101-113.
uint32_t ko_bend_factor(double semitones) {
    if (!std::isfinite(semitones)) return 1u << 24;
    double f = std::exp2(semitones / 12.0) * (double)(1u << 24);
    if (f <= 0.0) return 1;
    if (f >= 4294967295.0) return 0xFFFFFFFFu;
    return (uint32_t)std::round(f);
}
float ko_catmull_rom(float sm1, float s0, float s1, float s2, float t) {
    return catmull_rom(sm1, s0, s1, s2, t);
}

// CpuSynth::new, src/cpu.rs:166-185.
ko_synth* ko_create(const kc_config* cfg, const int16_t* pool, uint64_t pool_len,
                    const kc_region_params* params, uint32_t params_len) {
    if (!cfg || cfg->gate_frames == 0 || cfg->block_frames % cfg->gate_frames != 0) return nullptr;
    ko_synth* s = new ko_synth();
    s->cfg = *cfg;
    s->pool_data.assign(pool, pool + pool_len);
    s->bank_params.assign(params, params + params_len);
    s->tiles = cfg->block_frames / cfg->gate_frames;
    s->tile_frames = cfg->gate_frames;
    s->mix.assign((size_t)cfg->block_frames * 2, 0.0);
    s->gate_rows.assign(s->tiles * GATE_SLOTS, 0);
    s->chan_rows.assign(s->tiles * BEND_CHANNELS * CHAN_FIELDS, 0);
    return s;
}

void ko_destroy(ko_synth* s) { delete s; }

int ko_set_gates(ko_synth* s, const uint32_t* rows, size_t n) {
    if (n != s->gate_rows.size()) return KC_ERR_INVALID;
    std::memcpy(s->gate_rows.data(), rows, n * 4);
    return KC_OK;
}

// CpuSynth::set_channels, src/cpu.rs:305-311.
int ko_set_channels(ko_synth* s, const uint32_t* rows, size_t n, int bend, int gain,
                    int variant) {
    if (n != s->chan_rows.size()) return KC_ERR_INVALID;
    std::memcpy(s->chan_rows.data(), rows, n * 4);
    s->bend_active = bend != 0;
    s->gain_active = gain != 0;
    s->variant_active = variant != 0;
    return KC_OK;
}

// CpuSynth::set_params_variant, src/cpu.rs:313-323.
int ko_set_params_variant(ko_synth* s, uint32_t index, const kc_region_params* data, size_t n) {
    if (index == 0) return KC_OK;
    size_t i = index - 1;
    if (s->variants.size() <= i) s->variants.resize(i + 1);
    s->variants[i].assign(data, data + n);
    return KC_OK;
}

// CpuSynth::spawn, src/cpu.rs:330-390.
int ko_spawn(ko_synth* s, const kc_spawn_cmd* cmds, size_t want) {
    const size_t cap = s->cfg.max_voices;
    const size_t live = s->pool.len();
    if (live + want > cap) {
        if (s->cfg.steal_rule == KC_STEAL_DROP_NEW) {
            size_t take = std::min(want, cap > live ? cap - live : 0);
            s->dropped += want - take;
            for (size_t i = 0; i < take; ++i) s->pool.push(cmds[s->pick(i, want, take)]);
            return KC_OK;
        }
        size_t need = live + want - cap;
        need = std::min(need, live);
        need = std::min(need, (size_t)max_steal(s->cfg));
        if (need > 0) {
            // select_nth_unstable_by_key(need - 1, steal_key): the keys are a
            // total order, so the victim *set* is unique; nth_element gives it.
            std::vector<uint32_t> order(live);
            for (size_t i = 0; i < live; ++i) order[i] = (uint32_t)i;
            std::nth_element(order.begin(), order.begin() + (need - 1), order.end(),
                             [s](uint32_t a, uint32_t b) { return s->steal_key(a) < s->steal_key(b); });
            const uint32_t span = steal_span(s->cfg);
            for (size_t j = 0; j < need; ++j) {
                uint32_t i = order[j];
                uint32_t id = (uint32_t)s->pool.note_id[i];
                s->pool.stop_rel[i] = id % span + 1;
            }
            s->stolen += need;
        }
        size_t take = std::min(want, cap - (live - need));
        s->dropped += want - take;
        for (size_t i = 0; i < take; ++i) s->pool.push(cmds[s->pick(i, want, take)]);
        return KC_OK;
    }
    for (size_t i = 0; i < want; ++i) s->pool.push(cmds[i]);
    return KC_OK;
}

// CpuSynth::render, src/cpu.rs:392-639.
int ko_render(ko_synth* s, float* out, size_t n, double* mix64, int threads) {
    const size_t block = s->cfg.block_frames;
    if (n != block * 2) return KC_ERR_INVALID;
    std::fill(s->mix.begin(), s->mix.end(), 0.0);
    const size_t nv = s->pool.len();
    if (threads <= 1 || nv < 1024) {
        for (size_t v = 0; v < nv; ++v) s->render_voice(v, s->mix.data());
    } else {
        std::vector<std::vector<double>> part(threads, std::vector<double>(block * 2, 0.0));
        std::vector<std::thread> th;
        for (int t = 0; t < threads; ++t) {
            th.emplace_back([s, t, threads, nv, &part]() {
                size_t lo = nv * t / threads, hi = nv * (t + 1) / threads;
                for (size_t v = lo; v < hi; ++v) s->render_voice(v, part[t].data());
            });
        }
        for (auto& x : th) x.join();
        for (int t = 0; t < threads; ++t)
            for (size_t j = 0; j < block * 2; ++j) s->mix[j] += part[t][j];
    }
    float peak = 0.0f;
    for (size_t j = 0; j < block * 2; ++j) {
        float v = (float)s->mix[j];
        out[j] = v;
        float a = std::fabs(v);
        if (a > peak) peak = a;
    }
    if (mix64) std::memcpy(mix64, s->mix.data(), block * 2 * sizeof(double));
    s->peak = peak;
    // Compaction, src/cpu.rs:627-636.
    std::vector<char> keep(nv);
    bool any_dead = false;
    for (size_t v = 0; v < nv; ++v) {
        keep[v] = s->pool.env_stage[v] != ENV_DEAD;
        any_dead |= !keep[v];
    }
    if (any_dead) s->pool.compact(keep);
    return KC_OK;
}

int ko_stats(const ko_synth* s, kc_block_stats* out) {
    out->active_voices = s->pool.len();
    out->stolen = s->stolen;
    out->dropped = s->dropped;
    out->peak = s->peak;
    out->pad = 0;
    return KC_OK;
}

int ko_read_pool(const ko_synth* s, uint32_t* fields, size_t cap_words, uint32_t* live) {
    const size_t n = s->pool.len();
    *live = (uint32_t)n;
    if (cap_words < n * 24) return KC_ERR_INVALID;
    const Pool& p = s->pool;
    for (size_t i = 0; i < n; ++i) {
        uint32_t w[24];
        w[0] = (uint32_t)p.phase[i];
        w[1] = (uint32_t)(p.phase[i] >> 32);
        w[2] = (uint32_t)p.step[i];
        w[3] = (uint32_t)(p.step[i] >> 32);
        w[4] = p.smp_base[i];
        w[5] = p.smp_len[i];
        w[6] = p.loop_start[i];
        w[7] = p.loop_end[i];
        w[8] = p.flags[i];
        w[9] = p.env_stage[i];
        std::memcpy(&w[10], &p.env_level[i], 4);
        std::memcpy(&w[11], &p.gain_l[i], 4);
        std::memcpy(&w[12], &p.gain_r[i], 4);
        std::memcpy(&w[13], &p.filt_z1[i], 4);
        std::memcpy(&w[14], &p.filt_z2[i], 4);
        w[15] = p.params[i];
        w[16] = p.region[i];
        w[17] = p.gate_slot[i];
        w[18] = p.ordinal[i];
        w[19] = p.start_rel[i];
        w[20] = (uint32_t)p.note_id[i];
        w[21] = (uint32_t)(p.note_id[i] >> 32);
        w[22] = p.born_variant[i];
        w[23] = p.stop_rel[i];
        for (int f = 0; f < 24; ++f) fields[(size_t)f * n + i] = w[f];
    }
    return KC_OK;
}

int ko_load_pool(ko_synth* s, const uint32_t* fields, uint32_t live, uint64_t stolen, uint64_t dropped) {
    if (!s || (live && !fields)) return KC_ERR_INVALID;
    Pool p;
    const size_t n = live;
    auto col = [&](int f, size_t i) { return fields[(size_t)f * n + i]; };
    auto colf = [&](int f, size_t i) {
        float x;
        const uint32_t w = col(f, i);
        std::memcpy(&x, &w, 4);
        return x;
    };
    for (size_t i = 0; i < n; ++i) {
        p.phase.push_back(((uint64_t)col(1, i) << 32) | col(0, i));
        p.step.push_back(((uint64_t)col(3, i) << 32) | col(2, i));
        p.smp_base.push_back(col(4, i));
        p.smp_len.push_back(col(5, i));
        p.loop_start.push_back(col(6, i));
        p.loop_end.push_back(col(7, i));
        p.flags.push_back(col(8, i));
        p.env_stage.push_back(col(9, i));
        p.env_level.push_back(colf(10, i));
        p.gain_l.push_back(colf(11, i));
        p.gain_r.push_back(colf(12, i));
        p.filt_z1.push_back(colf(13, i));
        p.filt_z2.push_back(colf(14, i));
        p.params.push_back(col(15, i));
        p.region.push_back(col(16, i));
        p.gate_slot.push_back(col(17, i));
        p.ordinal.push_back(col(18, i));
        p.start_rel.push_back(col(19, i));
        p.note_id.push_back(((uint64_t)col(21, i) << 32) | col(20, i));
        p.born_variant.push_back(col(22, i));
        p.stop_rel.push_back(col(23, i));
    }
    s->pool = std::move(p);
    s->stolen = stolen;
    s->dropped = dropped;
    return KC_OK;
}

}  // extern "C"
