// limiter.cpp -- the output stage Driver::next_block runs after the backend's
// render (src/driver.rs:596-606), and the WAV writer (src/wav.rs:50-159).
//
// Both run on the host on the mixed stereo block, not per voice: a 4096-frame
// block costs them a fraction of a millisecond at any voice count. They are
// restated statement for statement in f64 (the reference's own precision),
// so a block that the CUDA backend and the CPU backend mix to within the null
// comes out of the limiter the same way.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <string>
#include <utility>
#include <vector>

#include "../../../include/kestrel_host.h"

namespace kh {
std::string& last_error();  // driver.cpp
}  // namespace kh

namespace {

constexpr size_t TP_PHASES = 4, TP_TAPS = 8;

// Limiter (src/limiter.rs:13-116): the OmniConverter loudness follower.
struct Omni {
    double loudness_l = 1.0, loudness_r = 1.0, velocity_l = 0.0, velocity_r = 0.0;
    double attack = 100.0, falloff;
    double min_thresh = 0.4, strength = 1.0;
    bool reduce_high_pitch = false;
    double velocity_thresh = 1.0;
    bool first_sample = true;

    explicit Omni(uint32_t sample_rate) : falloff((double)sample_rate / 3.0) {}

    static double follow(double state, double x, double falloff, double attack) {
        return state > x ? (state * falloff + x) / (falloff + 1.0) : (state * attack + x) / (attack + 1.0);
    }

    void process(float* buf, size_t n) {
        for (size_t i = 0; i + 1 < n; i += 2) {
            const double in_l = buf[i], in_r = buf[i + 1];
            const double l_abs = std::fabs(in_l), r_abs = std::fabs(in_r);
            loudness_l = follow(loudness_l, l_abs, falloff, attack);
            loudness_r = follow(loudness_r, r_abs, falloff, attack);
            if (loudness_l < min_thresh) loudness_l = min_thresh;
            if (loudness_r < min_thresh) loudness_r = min_thresh;
            double l = in_l / (loudness_l * strength + 2.0 * (1.0 - strength)) / 2.0;
            double r = in_r / (loudness_r * strength + 2.0 * (1.0 - strength)) / 2.0;
            if (!first_sample) {
                const double dl = std::fabs(in_l - l), dr = std::fabs(in_r - r);
                velocity_l = follow(velocity_l, dl, falloff, attack);
                velocity_r = follow(velocity_r, dr, falloff, attack);
            }
            first_sample = false;
            if (reduce_high_pitch) {
                if (velocity_l > velocity_thresh) l = l / velocity_l * velocity_thresh;
                if (velocity_r > velocity_thresh) r = r / velocity_r * velocity_thresh;
            }
            buf[i] = (float)l;
            buf[i + 1] = (float)r;
        }
    }
};

// design_polyphase (src/limiter.rs:445-470): 4 phases x 8 taps of a
// Blackman-windowed sinc, each phase normalised to unity gain.
void design_polyphase(double out[TP_PHASES][TP_TAPS]) {
    const double n = (double)(TP_TAPS * TP_PHASES);
    for (size_t p = 0; p < TP_PHASES; ++p) {
        for (size_t t = 0; t < TP_TAPS; ++t) {
            const double x = (double)t - ((double)TP_TAPS / 2.0 - 1.0) - (double)p / (double)TP_PHASES;
            const double sinc = std::fabs(x) < 1e-12 ? 1.0 : std::sin(M_PI * x) / (M_PI * x);
            const double k = (double)(t * TP_PHASES + p);
            const double w = 0.42 - 0.5 * std::cos(2.0 * M_PI * k / (n - 1.0)) + 0.08 * std::cos(4.0 * M_PI * k / (n - 1.0));
            out[p][t] = sinc * w;
        }
        double sum = 0.0;
        for (size_t t = 0; t < TP_TAPS; ++t) sum += out[p][t];
        if (std::fabs(sum) > 1e-12)
            for (size_t t = 0; t < TP_TAPS; ++t) out[p][t] /= sum;
    }
}

// Brickwall (src/limiter.rs:164-441): lookahead true-peak limiter. The audio
// is delayed by the lookahead plus the detector's group delay; the gain is at
// most the moving average, over the lookahead window, of ceiling / (sliding
// maximum of the detected peak), which bounds every emitted sample by the
// ceiling; a two-stage release follows it.
struct Brickwall {
    double ceiling;
    size_t look;
    double release_coef, sustain_atk = 0.0, sustain_rel = 0.0;
    double g_slow = 1.0, g_fast = 1.0;
    std::vector<float> delay;
    size_t dpos = 0;
    std::deque<std::pair<double, uint64_t>> dq;
    std::vector<double> gr_ring;
    size_t gr_pos = 0;
    double gr_sum;
    double gain = 1.0;
    double hist[2][TP_TAPS] = {};
    double poly[TP_PHASES][TP_TAPS];
    size_t delay_frames;
    bool true_peak;
    uint64_t idx = 0;
    double peak_in = 0.0, min_gain = 1.0;

    Brickwall(uint32_t sample_rate, double ceiling_, double lookahead_ms, double release_ms, double sustain_ms,
              bool true_peak_)
        : ceiling(ceiling_), true_peak(true_peak_) {
        const double sr = (double)sample_rate;
        const double lk = std::round(lookahead_ms * 1e-3 * sr);
        look = std::max<size_t>(lk > 0.0 ? (size_t)lk : 0, 1);
        const double rel = std::max(release_ms * 1e-3 * sr, 1.0);
        if (sustain_ms > 0.0) {
            const double a = std::max(sustain_ms * 1e-3 * sr, 1.0);
            sustain_atk = 1.0 - std::exp(-1.0 / a);
            sustain_rel = 1.0 - std::exp(-1.0 / (a * 4.0));
        }
        release_coef = 1.0 - std::exp(-1.0 / rel);
        const size_t group = true_peak ? TP_TAPS / 2 - 1 : 0;
        delay_frames = look + group;
        delay.assign(delay_frames * 2, 0.0f);
        gr_ring.assign(look + 1, 1.0);
        gr_sum = (double)(look + 1);
        design_polyphase(poly);
    }

    double detect(double l, double r) {
        if (!true_peak) return std::max(std::fabs(l), std::fabs(r));
        double peak = 0.0;
        const double v2[2] = {l, r};
        for (int ch = 0; ch < 2; ++ch) {
            double* h = hist[ch];
            std::memmove(h + 1, h, (TP_TAPS - 1) * sizeof(double));
            h[0] = v2[ch];
            for (size_t p = 0; p < TP_PHASES; ++p) {
                double acc = 0.0;
                for (size_t t = 0; t < TP_TAPS; ++t) acc += poly[p][t] * h[t];
                const double a = std::fabs(acc);
                if (a > peak) peak = a;
            }
        }
        return peak;
    }

    void process(float* buf, size_t n) {
        for (size_t i = 0; i + 1 < n; i += 2) {
            const double in_l = buf[i], in_r = buf[i + 1];
            const size_t d = dpos * 2;
            const double out_l = delay[d], out_r = delay[d + 1];
            delay[d] = buf[i];
            delay[d + 1] = buf[i + 1];
            dpos = (dpos + 1) % delay_frames;

            const double det = detect(in_l, in_r);
            if (det > peak_in) peak_in = det;
            while (!dq.empty() && dq.back().first <= det) dq.pop_back();
            dq.emplace_back(det, idx);
            const uint64_t oldest = idx >= look ? idx - look : 0;
            while (!dq.empty() && dq.front().second < oldest) dq.pop_front();
            const double env = dq.empty() ? 0.0 : dq.front().first;

            const double gr = env > ceiling ? ceiling / env : 1.0;
            gr_sum += gr - gr_ring[gr_pos];
            gr_ring[gr_pos] = gr;
            gr_pos = (gr_pos + 1) % gr_ring.size();
            const double ma = gr_sum / (double)gr_ring.size();

            if (sustain_atk > 0.0) {
                const double c = ma < g_slow ? sustain_atk : sustain_rel;
                g_slow += (ma - g_slow) * c;
                g_slow = g_slow < 1e-9 ? 1e-9 : (g_slow > 1.0 ? 1.0 : g_slow);
            }
            const double q = ma / g_slow;
            const double req = q < 1.0 ? q : 1.0;  // f64::min: a NaN quotient gives 1
            if (req < g_fast) {
                g_fast = req;
            } else {
                g_fast += (req - g_fast) * release_coef;
                if (g_fast > req) g_fast = req;
            }
            gain = g_slow * g_fast;
            if (gain > ma) gain = ma;
            if (gain < min_gain) min_gain = gain;  // reporting only (the reference declares it, never sets it)

            buf[i] = (float)(out_l * gain);
            buf[i + 1] = (float)(out_r * gain);
            ++idx;
        }
    }
};

}  // namespace

struct kh_limiter {
    uint32_t mode = KH_LIMITER_OFF;
    Omni* omni = nullptr;
    Brickwall* bw = nullptr;
    ~kh_limiter() {
        delete omni;
        delete bw;
    }
};

struct kh_wav {
    FILE* f = nullptr;
    uint32_t format = KH_WAV_FLOAT32;
    uint16_t channels = 2;
    uint64_t data_bytes = 0;
    std::vector<uint8_t> buf;
};

extern "C" {

// clamp_block, src/limiter.rs:120-129.
uint64_t kh_clamp_block(float* buf, size_t n) {
    uint64_t c = 0;
    for (size_t i = 0; i < n; ++i) {
        const float v = buf[i];
        if (v > 1.0f || v < -1.0f) {
            ++c;
            buf[i] = v > 1.0f ? 1.0f : -1.0f;
        }
    }
    return c;
}

kh_limiter* kh_limiter_create(uint32_t mode, uint32_t sample_rate, double ceiling_db, double lookahead_ms,
                              double release_ms, double sustain_ms, int true_peak) {
    if (mode > KH_LIMITER_BRICKWALL || sample_rate == 0) {
        kh::last_error() = "limiter: unknown mode or zero sample rate";
        return nullptr;
    }
    // Config::validate's ranges (src/config.rs:472-494).
    if (mode == KH_LIMITER_BRICKWALL &&
        (!(ceiling_db >= -24.0 && ceiling_db <= 0.0) || !(lookahead_ms >= 0.05 && lookahead_ms <= 100.0) ||
         !(sustain_ms >= 0.0 && sustain_ms <= 10000.0) || !(release_ms >= 0.1 && release_ms <= 5000.0))) {
        kh::last_error() = "limiter: ceiling_db, lookahead_ms, release_ms or sustain_ms out of range";
        return nullptr;
    }
    kh_limiter* l = new kh_limiter();
    l->mode = mode;
    if (mode == KH_LIMITER_OMNI) l->omni = new Omni(sample_rate);
    if (mode == KH_LIMITER_BRICKWALL)
        l->bw = new Brickwall(sample_rate, std::pow(10.0, ceiling_db / 20.0), lookahead_ms, release_ms, sustain_ms,
                              true_peak != 0);
    return l;
}

void kh_limiter_destroy(kh_limiter* l) { delete l; }

uint32_t kh_limiter_latency(const kh_limiter* l) { return l && l->bw ? (uint32_t)l->bw->delay_frames : 0u; }

uint64_t kh_limiter_process(kh_limiter* l, float* buf, size_t n) {
    if (l && l->omni) l->omni->process(buf, n);
    if (l && l->bw) l->bw->process(buf, n);
    return kh_clamp_block(buf, n);
}

int kh_limiter_report(const kh_limiter* l, double* peak_in, double* min_gain) {
    if (!l || !l->bw) return 1;
    if (peak_in) *peak_in = l->bw->peak_in;
    if (min_gain) *min_gain = l->bw->min_gain;
    return 0;
}

kh_wav* kh_wav_create(const char* path, uint32_t sample_rate, uint16_t channels, uint32_t format) {
    if (!path || channels == 0 || format > KH_WAV_FLOAT32) {
        kh::last_error() = "wav: null path, zero channels or unknown format";
        return nullptr;
    }
    FILE* f = std::fopen(path, "wb");
    if (!f) {
        kh::last_error() = std::string("wav: cannot create ") + path;
        return nullptr;
    }
    kh_wav* w = new kh_wav();
    w->f = f;
    w->format = format;
    w->channels = channels;
    std::setvbuf(f, nullptr, _IOFBF, 1 << 20);
    // WavWriter::create, src/wav.rs:63-79: the sizes are patched at finish.
    const uint16_t bits = format == KH_WAV_PCM16 ? 16 : 32;
    const uint16_t tag = format == KH_WAV_PCM16 ? 1 : 3;
    const uint32_t block_align = (uint32_t)channels * (bits / 8);
    uint8_t h[44];
    auto put32 = [&](int o, uint32_t v) { std::memcpy(h + o, &v, 4); };
    auto put16 = [&](int o, uint16_t v) { std::memcpy(h + o, &v, 2); };
    std::memcpy(h, "RIFF", 4);
    put32(4, 0);
    std::memcpy(h + 8, "WAVEfmt ", 8);
    put32(16, 16);
    put16(20, tag);
    put16(22, channels);
    put32(24, sample_rate);
    put32(28, sample_rate * block_align);
    put16(32, (uint16_t)block_align);
    put16(34, bits);
    std::memcpy(h + 36, "data", 4);
    put32(40, 0);
    std::fwrite(h, 1, 44, f);
    return w;
}

// WavWriter::write_block, src/wav.rs:84-101.
int kh_wav_write(kh_wav* w, const float* samples, size_t n) {
    if (!w || (n && !samples)) return 1;
    if (w->format == KH_WAV_FLOAT32) {
        if (std::fwrite(samples, 4, n, w->f) != n) return 1;
        w->data_bytes += (uint64_t)n * 4;
        return 0;
    }
    w->buf.resize(n * 2);
    for (size_t i = 0; i < n; ++i) {
        float s = samples[i];
        s = s < -1.0f ? -1.0f : (s > 1.0f ? 1.0f : s);  // NaN stays NaN: the cast below makes it 0
        const float r = std::round(s * 32767.0f);
        const int16_t v = std::isnan(r) ? (int16_t)0 : (int16_t)r;
        std::memcpy(&w->buf[2 * i], &v, 2);
    }
    if (std::fwrite(w->buf.data(), 1, n * 2, w->f) != n * 2) return 1;
    w->data_bytes += (uint64_t)n * 2;
    return 0;
}

// WavWriter::finish, src/wav.rs:112-139: the RIFF and data sizes, saturated
// at 4 GiB.
int kh_wav_finish(kh_wav* w, uint64_t* data_bytes) {
    if (!w) return 1;
    int rc = 0;
    const uint64_t riff = 36 + w->data_bytes;
    const uint32_t riff32 = (uint32_t)std::min<uint64_t>(riff, 0xFFFFFFFFull);
    const uint32_t data32 = (uint32_t)std::min<uint64_t>(w->data_bytes, 0xFFFFFFFFull);
    if (std::fflush(w->f) != 0) rc = 1;
    if (std::fseek(w->f, 4, SEEK_SET) != 0 || std::fwrite(&riff32, 4, 1, w->f) != 1) rc = 1;
    if (std::fseek(w->f, 40, SEEK_SET) != 0 || std::fwrite(&data32, 4, 1, w->f) != 1) rc = 1;
    if (std::fclose(w->f) != 0) rc = 1;
    if (data_bytes) *data_bytes = w->data_bytes;
    delete w;
    return rc;
}

}  // extern "C"
