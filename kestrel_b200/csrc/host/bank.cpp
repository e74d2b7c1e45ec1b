// bank.cpp -- src/bank.rs and src/resample.rs, restated in C++17. Every f32
// expression is evaluated in the order the Rust source writes it (the file is
// built with -ffp-contract=off).
#include "bank.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <set>
#include <unordered_map>

namespace kh {

namespace {
constexpr float PI_F = 3.14159265358979323846f;  // std::f32::consts::PI
constexpr float FRAC_1_SQRT_2_F = 0.70710678118654752440f;

// Sound controller constants, src/bank.rs:283-326.
constexpr float CC_CUTOFF_CENTS_PER_STEP = 75.0f;
constexpr float CC_Q_CB_PER_STEP = 240.0f / 63.0f;
constexpr float CC_ENV_STEPS_PER_OCTAVE = 8.0f;
constexpr float CC_ENV_ADD_PER_CUBE = 6.0e-5f;
constexpr float CC_MIN_FADE_SECS = 0.004f;
}  // namespace

// timecents_to_secs, src/bank.rs:451-459.
float timecents_to_secs(float tc) {
    if (tc <= -12000.0f) return 0.0f;
    return std::pow(2.0f, tc / 1200.0f);
}
// cents_to_hz, src/bank.rs:461-464.
float cents_to_hz(float cents) { return 8.176f * std::pow(2.0f, cents / 1200.0f); }
// cb_to_gain, src/bank.rs:466-469.
float cb_to_gain(float cb) { return std::pow(10.0f, -cb / 200.0f); }

// velocity_atten_cb, src/bank.rs:491-511.
float velocity_atten_cb(uint8_t vel, float veltrack) {
    const float v = (float)std::max<uint8_t>(vel, 1) / 127.0f;
    const float t = rclamp(veltrack, -100.0f, 100.0f) / 100.0f;
    if (t == 1.0f) return rclamp(-400.0f * std::log10(v), 0.0f, 960.0f);
    const float gain = t >= 0.0f ? 1.0f - t * (1.0f - v * v) : 1.0f + t * v * v;
    if (gain <= 0.0f) return 960.0f;
    return rclamp(-200.0f * std::log10(gain), 0.0f, 960.0f);
}

// TimeMod::from_controller, src/bank.rs:241-252.
TimeMod TimeMod::from_controller(uint8_t v) {
    const float d = (float)v - 64.0f;
    TimeMod t;
    if (d <= 0.0f) {
        t.scale = std::exp2(d / CC_ENV_STEPS_PER_OCTAVE);
        t.add = 0.0f;
    } else {
        t.scale = 1.0f;
        t.add = CC_ENV_ADD_PER_CUBE * d * d * d;
    }
    return t;
}

// ParamMod::from_controllers, src/bank.rs:336-348.
ParamMod ParamMod::from_controllers(uint8_t cc71, uint8_t cc72, uint8_t cc73, uint8_t cc74, uint8_t cc75) {
    ParamMod m;
    m.cutoff_cents = ((float)cc74 - 64.0f) * CC_CUTOFF_CENTS_PER_STEP;
    m.q_cb = rmax((float)cc71 - 64.0f, 0.0f) * CC_Q_CB_PER_STEP;
    m.attack = TimeMod::from_controller(cc73);
    m.decay = TimeMod::from_controller(cc75);
    m.release = TimeMod::from_controller(cc72);
    return m;
}

// Preset::build_key_index, src/bank.rs:364-381.
void Preset::build_key_index(const std::vector<Region>& rg) {
    std::vector<std::vector<uint32_t>> per_key(128);
    for (uint32_t r : regions) {
        const Region& reg = rg[r];
        for (int k = reg.key_lo; k <= std::min<int>(reg.key_hi, 127); ++k) per_key[k].push_back(r);
    }
    key_index.clear();
    key_regions.clear();
    for (auto& list : per_key) {
        key_index.push_back((uint32_t)key_regions.size());
        key_regions.insert(key_regions.end(), list.begin(), list.end());
    }
    key_index.push_back((uint32_t)key_regions.size());
}

// Bank::finish, src/bank.rs:514-525.
void Bank::finish() {
    for (auto& p : presets) p.build_key_index(regions);
    index.clear();
    for (uint32_t i = 0; i < presets.size(); ++i)
        index.push_back({((uint32_t)presets[i].bank << 16) | presets[i].program, i});
    std::stable_sort(index.begin(), index.end(),
                     [](const auto& a, const auto& b) { return a.first < b.first; });
}

// Bank::find_preset, src/bank.rs:527-544.
bool Bank::find_preset(uint16_t bank, uint16_t program, uint32_t* out) const {
    auto find = [&](uint32_t key) -> int64_t {
        auto it = std::lower_bound(index.begin(), index.end(), key,
                                   [](const auto& e, uint32_t k) { return e.first < k; });
        if (it != index.end() && it->first == key) return (int64_t)it->second;
        return -1;
    };
    int64_t i = find(((uint32_t)bank << 16) | program);
    if (i < 0) i = find(program);
    if (i < 0 && bank == 128) {
        for (const auto& e : index)
            if ((e.first >> 16) == 128) {
                i = e.second;
                break;
            }
    }
    if (i < 0 && !index.empty()) i = index.front().second;
    if (i < 0) return false;
    *out = (uint32_t)i;
    return true;
}

// Bank::build_voice, src/bank.rs:596-686.
bool Bank::build_voice(const Region& r, uint32_t region_idx, uint8_t key, uint8_t vel, const BankConfig& cfg,
                       VoiceSpawn* out) const {
    if (r.sample >= samples.size()) return false;
    const SampleInfo& s = samples[r.sample];
    if (s.len == 0) return false;
    const uint8_t eff_key = r.fixed_key >= 0 ? (uint8_t)r.fixed_key : key;
    const uint8_t eff_vel = r.fixed_vel >= 0 ? (uint8_t)r.fixed_vel : vel;
    const double root = r.root_key_override >= 0 ? (double)r.root_key_override : (double)s.root_key;
    const double cents = ((double)eff_key - root) * (double)r.scale_tuning + (double)r.coarse_tune * 100.0 +
                         (double)r.fine_tune + (double)s.correction_cents;
    double ratio = std::exp2(cents / 1200.0);
    if (pool_rate == 0)
        ratio *= (double)s.rate / (double)cfg.sample_rate;
    else
        ratio *= (double)pool_rate / (double)cfg.sample_rate;
    if (!(std::isfinite(ratio) && ratio > 0.0)) return false;

    const float atten = r.attenuation_cb + velocity_atten_cb(eff_vel, r.amp_veltrack);
    const float gain = cb_to_gain(atten) * cfg.master_volume;
    const float theta = (rclamp(r.pan, -1.0f, 1.0f) + 1.0f) * 0.5f * (PI_F * 0.5f);
    const float gain_l = gain * std::cos(theta);
    const float gain_r = gain * std::sin(theta);

    auto scale = [&](int32_t v) -> int64_t { return sat_cast<int64_t>(rroundf((float)v * s.resample_ratio)); };
    const int64_t len = s.len;
    const uint32_t start_offset = (uint32_t)std::clamp<int64_t>(scale(r.addr_start), 0, len - 1);
    const uint32_t smp_len = (uint32_t)std::clamp<int64_t>(len + scale(r.addr_end), 1, len);
    const uint32_t loop_start =
        (uint32_t)std::clamp<int64_t>((int64_t)s.loop_start + scale(r.addr_loop_start), 0, (int64_t)smp_len - 1);
    const uint32_t loop_end =
        (uint32_t)std::clamp<int64_t>((int64_t)s.loop_end + scale(r.addr_loop_end), 0, (int64_t)smp_len);

    const uint32_t keys = r.params_stride != 0 ? 128u : 1u;
    const uint32_t ki = r.params_stride != 0 ? (uint32_t)eff_key : 0u;
    uint32_t vi = 0;
    if (r.params_vel_span > 1) {
        const uint32_t d = vel > r.vel_lo ? (uint32_t)(vel - r.vel_lo) : 0u;
        vi = std::min(d, r.params_vel_span - 1);
    }
    uint32_t flags = r.loop_mode == LoopMode::NoLoop        ? 0u
                     : r.loop_mode == LoopMode::Continuous ? VF_LOOP
                                                           : (VF_LOOP | VF_LOOP_UNTIL_RELEASE);
    if (r.loop_mode != LoopMode::NoLoop && loop_end <= loop_start + 1) flags = 0;

    out->phase = (uint64_t)start_offset << 32;
    out->step = fixed_from_f64(ratio);
    out->smp_base = s.start;
    out->smp_len = smp_len;
    out->loop_start = loop_start;
    out->loop_end = loop_end;
    out->flags = flags;
    out->params = r.params_base + vi * keys + ki;
    out->region = region_idx;
    out->gain_l = gain_l;
    out->gain_r = gain_r;
    out->delay_frames = sat_cast<uint32_t>(r.delay * (float)cfg.sample_rate);
    out->exclusive_class = r.exclusive_class;
    return true;
}

// Bank::build_layer, src/bank.rs:585-594.
bool Bank::build_layer(uint32_t region, uint8_t key, uint8_t vel, const BankConfig& cfg, VoiceSpawn* out) const {
    if (region >= regions.size()) return false;
    return build_voice(regions[region], region, std::min<uint8_t>(key, 127), vel, cfg, out);
}

// make_params, src/bank.rs:876-954.
static kc_region_params make_params(const Region& r, uint8_t key, uint8_t vel, float sr, const BankConfig& cfg,
                                    const ParamMod& m) {
    const float key_delta = 60.0f - (float)key;
    const float hold = r.hold * std::pow(2.0f, (float)r.keynum_to_hold * key_delta / 1200.0f);
    const float decay = r.decay * std::pow(2.0f, (float)r.keynum_to_decay * key_delta / 1200.0f);
    auto floor_fn = [](float t, float base) { return rmax(t, rmin(CC_MIN_FADE_SECS, base)); };
    const float attack_frames = rmax(m.attack.apply(r.attack) * sr, 0.0f);
    const float hold_frames = rmax(hold * sr, 0.0f);
    const float decay_frames = rmax(floor_fn(m.decay.apply(decay), decay) * sr, 1.0f);
    const float release_frames = rmax(floor_fn(m.release.apply(r.release), r.release) * sr, 1.0f);
    const float attack_rate = attack_frames < 1.0f ? 1.0f : 1.0f / attack_frames;
    const float attack_end = 1.0f + hold_frames * attack_rate;
    const float sustain = rclamp(r.sustain, 0.0f, 1.0f);
    const float floor = cfg.env_floor;
    const float exp_rel = std::pow(10.0f, -100.0f / (20.0f * release_frames));
    const float lin_rel = 1.0f / release_frames;
    float decay_coef, release_coef;
    if (cfg.exp_decay) {
        decay_coef = std::pow(10.0f, -100.0f / (20.0f * decay_frames));
    } else {
        decay_coef = 1.0f / decay_frames;
    }
    release_coef = cfg.exp_release ? exp_rel : lin_rel;
    const float fc_cents = r.filter_fc_cents + r.filter_veltrack_cents * ((float)vel / 127.0f) + m.cutoff_cents;
    const float fc = cents_to_hz(fc_cents);
    const float nyq_guard = sr * 0.49f;
    const bool use_filter = cfg.filter_enabled && fc_cents < 13500.0f && fc < nyq_guard && fc > 20.0f;
    kc_region_params p{};
    if (use_filter) {
        biquad_lowpass(fc, r.filter_q_cb + m.q_cb, sr, &p.b0, &p.b1, &p.a1, &p.a2);
    } else {
        p.b0 = 1.0f;
        p.b1 = 0.0f;
        p.a1 = 0.0f;
        p.a2 = 0.0f;
    }
    p.attack_rate = attack_rate;
    p.attack_end = attack_end;
    p.decay_coef = decay_coef;
    p.decay_target = rmax(sustain, floor);
    p.sustain = sustain;
    p.release_coef = release_coef;
    p.flags = use_filter ? RP_FILTER : 0u;
    p.pad = 0;
    return p;
}

// biquad_lowpass, src/bank.rs:956-979 (RBJ, normalised against the default Q).
void biquad_lowpass(float fc, float q_cb, float sr, float* b0, float* b1, float* a1, float* a2) {
    const float q_db = q_cb / 10.0f - 3.01f;
    const float q = rmax(std::pow(10.0f, q_db / 20.0f), 0.001f);
    const float gain = std::sqrt(FRAC_1_SQRT_2_F / q);
    const float w0 = 2.0f * PI_F * rclamp(fc / sr, 1.0e-5f, 0.49f);
    const float sin_w0 = std::sin(w0), cos_w0 = std::cos(w0);
    const float alpha = sin_w0 / (2.0f * q);
    const float a0 = 1.0f + alpha;
    *b0 = gain * (1.0f - cos_w0) * 0.5f / a0;
    *b1 = gain * (1.0f - cos_w0) / a0;
    *a1 = -2.0f * cos_w0 / a0;
    *a2 = (1.0f - alpha) / a0;
}

// Bank::build_params, src/bank.rs:688-713.
void Bank::build_params(const BankConfig& cfg) {
    uint32_t n = 0;
    for (auto& r : regions) {
        const bool per_key = r.keynum_to_decay != 0 || r.keynum_to_hold != 0;
        const uint32_t vel_span =
            r.filter_veltrack_cents != 0.0f
                ? std::min<uint32_t>((uint32_t)(r.vel_hi > r.vel_lo ? r.vel_hi - r.vel_lo : 0) + 1, 128)
                : 1;
        r.params_base = n;
        r.params_stride = per_key ? 1 : 0;
        r.params_vel_span = vel_span;
        n += vel_span * (per_key ? 128 : 1);
    }
    params = build_variant(cfg, ParamMod{});
    build_admission_tables(cfg);
}

// Bank::build_admission_tables, src/bank.rs:723-778.
void Bank::build_admission_tables(const BankConfig& cfg) {
    const size_t n = regions.size();
    gain_table.assign(n * 128 * 2, 0.0f);
    key_ok.assign((n * 128 + 63) / 64, 0);
    delay_frames.resize(n);
    for (size_t i = 0; i < n; ++i) delay_frames[i] = sat_cast<uint32_t>(regions[i].delay * (float)cfg.sample_rate);
    for (size_t ri = 0; ri < n; ++ri) {
        const Region& r = regions[ri];
        const float theta = (rclamp(r.pan, -1.0f, 1.0f) + 1.0f) * 0.5f * (PI_F * 0.5f);
        const float pan_l = std::cos(theta), pan_r = std::sin(theta);
        for (int v = 0; v < 128; ++v) {
            const uint8_t eff_vel = r.fixed_vel >= 0 ? (uint8_t)r.fixed_vel : (uint8_t)v;
            const float atten = r.attenuation_cb + velocity_atten_cb(eff_vel, r.amp_veltrack);
            const float gain = cb_to_gain(atten) * cfg.master_volume;
            gain_table[(ri * 128 + v) * 2] = gain * pan_l;
            gain_table[(ri * 128 + v) * 2 + 1] = gain * pan_r;
        }
        if (r.sample >= samples.size()) continue;
        const SampleInfo& s = samples[r.sample];
        if (s.len == 0) continue;
        for (int k = 0; k < 128; ++k) {
            const uint8_t eff_key = r.fixed_key >= 0 ? (uint8_t)r.fixed_key : (uint8_t)k;
            const double root = r.root_key_override >= 0 ? (double)r.root_key_override : (double)s.root_key;
            const double cents = ((double)eff_key - root) * (double)r.scale_tuning + (double)r.coarse_tune * 100.0 +
                                 (double)r.fine_tune + (double)s.correction_cents;
            double ratio = std::exp2(cents / 1200.0);
            if (pool_rate == 0)
                ratio *= (double)s.rate / (double)cfg.sample_rate;
            else
                ratio *= (double)pool_rate / (double)cfg.sample_rate;
            if (std::isfinite(ratio) && ratio > 0.0) {
                const size_t bit = ri * 128 + k;
                key_ok[bit / 64] |= 1ull << (bit % 64);
            }
        }
    }
}

bool Bank::region_key_ok(uint32_t region, uint8_t key) const {
    const size_t bit = (size_t)region * 128 + key;
    return (key_ok[bit / 64] >> (bit % 64)) & 1;
}

// Bank::preview_note_on, src/bank.rs:793-829.
void Bank::preview_note_on(uint32_t preset, uint8_t key, uint8_t vel, size_t max_layers,
                           std::vector<PreviewLayer>& out) const {
    if (preset >= presets.size()) return;
    const Preset& p = presets[preset];
    key = std::min<uint8_t>(key, 127);
    const uint32_t lo = p.key_index[key], hi = p.key_index[key + 1];
    size_t layers = 0;
    for (uint32_t j = lo; j < hi; ++j) {
        if (layers >= max_layers) break;
        const uint32_t ri = p.key_regions[j];
        const Region& r = regions[ri];
        if (vel < r.vel_lo || vel > r.vel_hi) continue;
        if (!region_key_ok(ri, key)) continue;
        PreviewLayer l;
        l.region = ri;
        l.gain_l = gain_table[((size_t)ri * 128 + vel) * 2];
        l.gain_r = gain_table[((size_t)ri * 128 + vel) * 2 + 1];
        l.delay_frames = delay_frames[ri];
        out.push_back(l);
        ++layers;
    }
}

// Bank::build_variant, src/bank.rs:836-853.
std::vector<kc_region_params> Bank::build_variant(const BankConfig& cfg, const ParamMod& m) const {
    const float sr = (float)cfg.sample_rate;
    std::vector<kc_region_params> out;
    out.reserve(params.size());
    for (const auto& r : regions) {
        const bool per_key = r.params_stride != 0;
        for (uint32_t v = 0; v < r.params_vel_span; ++v) {
            const uint8_t vel = (uint8_t)std::min<uint32_t>(r.vel_lo + v, 127);
            if (per_key) {
                for (uint32_t k = 0; k < 128; ++k) out.push_back(make_params(r, (uint8_t)k, vel, sr, cfg, m));
            } else {
                out.push_back(make_params(r, 60, vel, sr, cfg, m));
            }
        }
    }
    return out;
}

void Bank::filter_inputs(const BankConfig& cfg, const ParamMod& m, std::vector<float>& fc, std::vector<float>& q_cb,
                         std::vector<uint8_t>& on) const {
    const float sr = (float)cfg.sample_rate;
    fc.clear();
    q_cb.clear();
    on.clear();
    auto one = [&](const Region& r, uint8_t vel) {
        // make_params, src/bank.rs:922-938: the cutoff, its guard, and the Q.
        const float fc_cents = r.filter_fc_cents + r.filter_veltrack_cents * ((float)vel / 127.0f) + m.cutoff_cents;
        const float f = cents_to_hz(fc_cents);
        const bool use = cfg.filter_enabled && fc_cents < 13500.0f && f < sr * 0.49f && f > 20.0f;
        fc.push_back(f);
        q_cb.push_back(r.filter_q_cb + m.q_cb);
        on.push_back(use ? 1 : 0);
    };
    for (const auto& r : regions) {
        const bool per_key = r.params_stride != 0;
        for (uint32_t v = 0; v < r.params_vel_span; ++v) {
            const uint8_t vel = (uint8_t)std::min<uint32_t>(r.vel_lo + v, 127);
            const int reps = per_key ? 128 : 1;
            for (int k = 0; k < reps; ++k) one(r, vel);
        }
    }
}

uint32_t Bank::max_sample_len() const {
    uint32_t m = 1;
    for (const auto& s : samples) m = std::max(m, s.len);
    return m;
}

// ---- resample.rs ------------------------------------------------------------

namespace {
constexpr size_t TAPS = 32, PHASES = 512;

double sinc(double x) {
    if (std::fabs(x) < 1e-9) return 1.0;
    const double px = M_PI * x;
    return std::sin(px) / px;
}

}  // namespace

// SincBank::new, src/resample.rs:15-49.
std::vector<float> sinc_table(double ratio) {
    const double cutoff = (ratio < 1.0 ? ratio : 1.0) * 0.95;
    std::vector<float> table(PHASES * TAPS, 0.0f);
    const double half = (double)TAPS / 2.0;
    for (size_t p = 0; p < PHASES; ++p) {
        const double frac = (double)p / (double)PHASES;
        double sum = 0.0;
        for (size_t k = 0; k < TAPS; ++k) {
            const double x = (double)k - half + 1.0 - frac;
            const double s = sinc(x * cutoff) * cutoff;
            double t = ((double)k - frac + 1.0) / (double)TAPS;
            t = rclampd(t, 0.0, 1.0);
            const double w = 0.42 - 0.5 * std::cos(2.0 * M_PI * t) + 0.08 * std::cos(4.0 * M_PI * t);
            const double v = s * w;
            table[p * TAPS + k] = (float)v;
            sum += v;
        }
        if (std::fabs(sum) > 1e-9) {
            const float inv = (float)(1.0 / sum);
            for (size_t k = 0; k < TAPS; ++k) table[p * TAPS + k] *= inv;
        }
    }
    return table;
}

namespace {
std::atomic<kh_resample_fn> g_resample_fn{nullptr};
std::atomic<void*> g_resample_user{nullptr};
}  // namespace

void set_resample_hook(kh_resample_fn fn, void* user) {
    g_resample_user.store(user);
    g_resample_fn.store(fn);
}

ResampleHook resample_hook() {
    ResampleHook h;
    h.fn = g_resample_fn.load();
    h.user = g_resample_user.load();
    return h;
}

// SincBank::process + resample_i16, src/resample.rs:51-107.
std::vector<int16_t> resample_i16(const std::vector<int16_t>& src, double ratio) {
    if (std::fabs(ratio - 1.0) < 1e-12) return src;
    if (src.empty()) return {};
    const std::vector<float> table = sinc_table(ratio);
    const int64_t n = (int64_t)src.size();
    const size_t out_len = std::max<size_t>(sat_cast<size_t>(std::round((double)src.size() * ratio)), 1);
    std::vector<int16_t> out;
    out.reserve(out_len);
    const int64_t half = (int64_t)TAPS / 2;
    const double inv_ratio = 1.0 / ratio;
    for (size_t j = 0; j < out_len; ++j) {
        const double t = (double)j * inv_ratio;
        const int64_t i = (int64_t)std::floor(t);
        const double frac = t - (double)i;
        const size_t p = std::min<size_t>(sat_cast<size_t>(frac * (double)PHASES), PHASES - 1);
        const float* coeffs = &table[p * TAPS];
        const int64_t base = i - half + 1;
        float acc = 0.0f;
        if (base >= 0 && base + (int64_t)TAPS <= n) {
            for (size_t k = 0; k < TAPS; ++k) acc += coeffs[k] * (float)src[base + k];
        } else {
            for (size_t k = 0; k < TAPS; ++k) {
                const int64_t idx = std::clamp<int64_t>(base + (int64_t)k, 0, n - 1);
                acc += coeffs[k] * (float)src[idx];
            }
        }
        out.push_back(sat_cast<int16_t>(rclamp(acc, -32768.0f, 32767.0f)));
    }
    return out;
}

// testkit::noise, src/testkit.rs:41-53.
std::vector<int16_t> noise(size_t n, uint64_t seed) {
    uint64_t s = seed | 1;
    std::vector<int16_t> v(n);
    for (size_t i = 0; i < n; ++i) {
        s ^= s << 13;
        s ^= s >> 7;
        s ^= s << 17;
        v[i] = (int16_t)((int32_t)(s >> 40) - 8192);
    }
    return v;
}

}  // namespace kh
