// bank.h -- the format-independent instrument bank (src/bank.rs), its SF2
// generator flattening (src/sf2.rs) and the load-time resampler
// (src/resample.rs), restated in C++17 for the host side.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../../include/kestrel_host.h"
#include "rust.h"

namespace kh {

constexpr uint32_t VF_LOOP = 1, VF_LOOP_UNTIL_RELEASE = 2, RP_FILTER = 1;

enum class LoopMode { NoLoop, Continuous, UntilRelease };

// bank::SampleInfo (src/bank.rs:34-54).
struct SampleInfo {
    uint32_t start = 0, len = 0, loop_start = 0, loop_end = 0, rate = 0;
    uint8_t root_key = 60;
    float correction_cents = 0.0f;
    float resample_ratio = 1.0f;
};

// bank::Region (src/bank.rs:56-160), defaults included.
struct Region {
    uint32_t sample = 0;
    uint8_t key_lo = 0, key_hi = 127, vel_lo = 0, vel_hi = 127;
    int16_t root_key_override = -1, fixed_key = -1, fixed_vel = -1;
    int16_t coarse_tune = 0, fine_tune = 0, scale_tuning = 100;
    float attenuation_cb = 0.0f, amp_veltrack = 100.0f, pan = 0.0f;
    LoopMode loop_mode = LoopMode::NoLoop;
    int32_t addr_start = 0, addr_end = 0, addr_loop_start = 0, addr_loop_end = 0;
    uint8_t exclusive_class = 0;
    float delay = 0.0f, attack = 0.001f, hold = 0.0f, decay = 0.001f, sustain = 1.0f, release = 0.001f;
    int16_t keynum_to_hold = 0, keynum_to_decay = 0;
    float filter_fc_cents = 13500.0f, filter_q_cb = 0.0f, filter_veltrack_cents = 0.0f;
    uint32_t params_base = 0, params_stride = 0, params_vel_span = 1;
};

// bank::TimeMod / ParamMod (src/bank.rs:192-349).
struct TimeMod {
    float scale = 1.0f, add = 0.0f;
    float apply(float secs) const { return secs * scale + add; }
    static TimeMod from_controller(uint8_t v);
    bool operator==(const TimeMod& o) const { return scale == o.scale && add == o.add; }
};
struct ParamMod {
    float cutoff_cents = 0.0f, q_cb = 0.0f;
    TimeMod attack, decay, release;
    static ParamMod from_controllers(uint8_t cc71, uint8_t cc72, uint8_t cc73, uint8_t cc74, uint8_t cc75);
};

struct Preset {
    uint16_t bank = 0, program = 0;
    std::vector<uint32_t> regions, key_index, key_regions;
    void build_key_index(const std::vector<Region>& regions);
};

// bank::VoiceSpawn (src/bank.rs:432-449).
struct VoiceSpawn {
    uint64_t phase = 0, step = 0;
    uint32_t smp_base = 0, smp_len = 0, loop_start = 0, loop_end = 0, flags = 0, params = 0, region = 0;
    float gain_l = 0.0f, gain_r = 0.0f;
    uint32_t delay_frames = 0;
    uint8_t exclusive_class = 0;
};

// bank::PreviewLayer (src/bank.rs:418-430).
struct PreviewLayer {
    uint32_t region = 0;
    float gain_l = 0.0f, gain_r = 0.0f;
    uint32_t delay_frames = 0;
};

struct BankConfig {
    uint32_t sample_rate = 48000;
    float env_floor = 1.0e-5f;
    bool exp_decay = true, exp_release = true;
    bool filter_enabled = true;
    float master_volume = 1.0f;
    bool resample_pool = true;
    uint64_t sample_pool_budget = 2ull << 30;
};

struct Bank {
    std::vector<int16_t> pool;
    uint32_t pool_rate = 0;
    std::vector<SampleInfo> samples;
    std::vector<Region> regions;
    std::vector<kc_region_params> params;
    std::vector<Preset> presets;
    std::vector<std::pair<uint32_t, uint32_t>> index;  // ((bank << 16) | program, preset)
    std::vector<float> gain_table;                     // region * 128 + vel -> (l, r) pairs
    std::vector<uint32_t> delay_frames;
    std::vector<uint64_t> key_ok;

    void finish();
    bool find_preset(uint16_t bank, uint16_t program, uint32_t* out) const;
    bool build_voice(const Region& r, uint32_t region_idx, uint8_t key, uint8_t vel, const BankConfig& cfg,
                     VoiceSpawn* out) const;
    bool build_layer(uint32_t region, uint8_t key, uint8_t vel, const BankConfig& cfg, VoiceSpawn* out) const;
    void build_params(const BankConfig& cfg);
    void build_admission_tables(const BankConfig& cfg);
    bool region_key_ok(uint32_t region, uint8_t key) const;
    void preview_note_on(uint32_t preset, uint8_t key, uint8_t vel, size_t max_layers,
                         std::vector<PreviewLayer>& out) const;
    std::vector<kc_region_params> build_variant(const BankConfig& cfg, const ParamMod& m) const;
    // The (cutoff Hz, Q cB, filter on) each entry of build_variant's table was
    // designed from, in the same order.
    void filter_inputs(const BankConfig& cfg, const ParamMod& m, std::vector<float>& fc, std::vector<float>& q_cb,
                       std::vector<uint8_t>& on) const;
    uint32_t max_sample_len() const;
};

float timecents_to_secs(float tc);
float cents_to_hz(float cents);
float cb_to_gain(float cb);
float velocity_atten_cb(uint8_t vel, float veltrack);
void biquad_lowpass(float fc, float q_cb, float sr, float* b0, float* b1, float* a1, float* a2);

// ---- SF2 generator flattening (src/sf2.rs:221-579) ------------------------
constexpr int GEN_COUNT = 60;
using GenArray = std::array<int16_t, GEN_COUNT>;

struct Sf2Sample {
    std::vector<int16_t> data;
    uint32_t rate = 44100, loop_start = 0, loop_end = 0;
    uint8_t root = 60;
    int8_t correction = 0;
};
struct Sf2Zone {
    uint16_t sample = 0;
    uint8_t key_lo = 0, key_hi = 127, vel_lo = 0, vel_hi = 127;
    std::vector<std::pair<uint16_t, int16_t>> gens;
};
struct Sf2Preset {
    uint16_t bank = 0, program = 0, instrument = 0;
    std::vector<std::pair<uint16_t, int16_t>> gens;
};
struct Sf2 {
    std::vector<Sf2Sample> samples;
    std::vector<std::vector<Sf2Zone>> instruments;
    std::vector<Sf2Preset> presets;
};

// sf2::load (src/sf2.rs:221-505): walk the RIFF tree, flatten presets into
// regions, pull the used samples into the pool (resampled to the pool rate),
// build params and the admission tables. load_sf2 writes the in-memory
// soundfont in the test kit's layout first, so both go through one loader.
bool load_sf2_file(const std::string& path, const BankConfig& cfg, Bank* out, std::string* err);
bool load_sf2(const Sf2& sf, const BankConfig& cfg, Bank* out, std::string* err);
// Sf2Builder::write's layout (src/testkit.rs:173-318) as bytes; false when
// the soundfont does not fit the format's indexes.
bool write_sf2(const Sf2& sf, std::vector<uint8_t>* out, std::string* err);

// sfz::load (src/sfz.rs:262-415): an SFZ instrument and the WAV files it
// names. `report` receives the warnings (unreadable samples, unsupported
// opcodes with their counts).
bool load_sfz_file(const std::string& path, const BankConfig& cfg, Bank* out, std::string* err,
                   std::vector<std::string>* report);
// parse_note_name and find_value_end (src/sfz.rs:88-116, 233-260).
bool sfz_note_name(const std::string& s, int32_t* out);
size_t sfz_value_end(const std::string& s);

// resample::resample_i16 (src/resample.rs:102-107).
std::vector<int16_t> resample_i16(const std::vector<int16_t>& src, double ratio);
// SincBank::new (src/resample.rs:18-49): 512 phases x 32 taps, phase-major.
std::vector<float> sinc_table(double ratio);
// The batch resampler kh_set_resampler installed, or null.
struct ResampleHook {
    kh_resample_fn fn = nullptr;
    void* user = nullptr;
};
ResampleHook resample_hook();
void set_resample_hook(kh_resample_fn fn, void* user);

// testkit waveforms (src/testkit.rs:19-53).
std::vector<int16_t> noise(size_t n, uint64_t seed);

}  // namespace kh
