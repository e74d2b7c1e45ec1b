// sfz.cpp -- src/sfz.rs and the WAV reader it loads samples with
// (src/wav.rs:160-356), restated in C++17.
//
// An SFZ file is a list of <header> sections of opcode=value pairs. Regions
// inherit from the <global>, <master> and <group> in force where they are
// written; every referenced WAV is read once per channel into the pool
// (resampled to the pool rate), stereo files becoming two mono regions
// panned hard left and right; the regions form one preset (bank 0, program
// 0). Opcodes outside the implemented set are counted and reported.
#include "bank.h"

#include <dirent.h>
#include <sys/stat.h>

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>

namespace kh {

namespace {

// ---- the WAV reader (src/wav.rs:164-356) -------------------------------------

struct WavData {
    uint32_t sample_rate = 0;
    uint16_t channels = 0;
    std::vector<float> interleaved;
    bool has_loop = false;
    uint32_t loop_start = 0, loop_end = 0;  // the smpl chunk's first loop, frames
    bool has_root = false;
    uint8_t root_key = 60;
    float fine_tune_cents = 0.0f;

    // WavData::channel_i16: channel ch, scaled to i16 with rounding.
    std::vector<int16_t> channel_i16(size_t ch) const {
        const size_t nch = channels;
        ch = std::min(ch, nch > 0 ? nch - 1 : 0);
        std::vector<int16_t> out;
        const size_t step = std::max<size_t>(nch, 1);
        for (size_t i = ch; i < interleaved.size(); i += step) {
            const float s = interleaved[i];
            const float c = std::isnan(s) ? s : std::min(std::max(s, -1.0f), 1.0f);
            const float v = std::round(c * 32767.0f);
            out.push_back(std::isnan(v) ? (int16_t)0 : (int16_t)v);
        }
        return out;
    }
};

uint16_t le16(const uint8_t* p) { return (uint16_t)(p[0] | p[1] << 8); }
uint32_t le32(const uint8_t* p) { return (uint32_t)p[0] | (uint32_t)p[1] << 8 | (uint32_t)p[2] << 16 | (uint32_t)p[3] << 24; }

bool decode_samples(const std::vector<uint8_t>& d, uint16_t tag, uint16_t bits, std::vector<float>& out) {
    out.clear();
    if (tag == 1 && bits == 8) {
        for (uint8_t b : d) out.push_back(((float)b - 128.0f) / 128.0f);
    } else if (tag == 1 && bits == 16) {
        for (size_t i = 0; i + 2 <= d.size(); i += 2) out.push_back((float)(int16_t)le16(&d[i]) / 32768.0f);
    } else if (tag == 1 && bits == 24) {
        for (size_t i = 0; i + 3 <= d.size(); i += 3) {
            const int32_t v = (int32_t)((uint32_t)d[i] << 8 | (uint32_t)d[i + 1] << 16 | (uint32_t)d[i + 2] << 24) >> 8;
            out.push_back((float)v / 8388608.0f);
        }
    } else if (tag == 1 && bits == 32) {
        for (size_t i = 0; i + 4 <= d.size(); i += 4) out.push_back((float)(int32_t)le32(&d[i]) / 2147483648.0f);
    } else if (tag == 3 && bits == 32) {
        for (size_t i = 0; i + 4 <= d.size(); i += 4) {
            float f;
            std::memcpy(&f, &d[i], 4);
            out.push_back(f);
        }
    } else if (tag == 3 && bits == 64) {
        for (size_t i = 0; i + 8 <= d.size(); i += 8) {
            double f;
            std::memcpy(&f, &d[i], 8);
            out.push_back((float)f);
        }
    } else {
        return false;
    }
    return true;
}

// wav::read: the fmt, data and smpl chunks; every other chunk is skipped.
bool read_wav(const std::string& path, WavData* w, std::string* err) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) {
        *err = "opening " + path + ": " + std::strerror(errno);
        return false;
    }
    std::vector<uint8_t> b;
    {
        uint8_t buf[1 << 16];
        size_t n;
        while ((n = std::fread(buf, 1, sizeof(buf), f)) > 0) b.insert(b.end(), buf, buf + n);
        std::fclose(f);
    }
    const uint64_t file_len = b.size();
    if (b.size() < 4 || std::memcmp(b.data(), "RIFF", 4) != 0) {
        *err = path + ": not a RIFF file";
        return false;
    }
    if (b.size() < 12 || std::memcmp(b.data() + 8, "WAVE", 4) != 0) {
        *err = path + ": not a WAVE file";
        return false;
    }
    uint16_t tag = 0, bits = 0;
    bool have_data = false;
    std::vector<uint8_t> data;
    size_t pos = 12;
    while (pos + 4 <= b.size()) {
        const uint8_t* id = &b[pos];
        if (pos + 8 > b.size()) {
            *err = path + ": truncated chunk header";
            return false;
        }
        const uint64_t size = le32(&b[pos + 4]);
        const uint64_t padded = size + (size & 1);
        if (size > file_len) {
            *err = path + ": chunk " + std::string((const char*)id, 4) + " claims " + std::to_string(size) + " bytes";
            return false;
        }
        const size_t body = pos + 8;
        if (std::memcmp(id, "fmt ", 4) == 0) {
            if (body + 16 > b.size()) {
                *err = path + ": truncated fmt chunk";
                return false;
            }
            tag = le16(&b[body]);
            w->channels = le16(&b[body + 2]);
            w->sample_rate = le32(&b[body + 4]);
            bits = le16(&b[body + 14]);
            if (tag == 0xFFFE && size >= 40) {
                // WAVE_FORMAT_EXTENSIBLE: the sub-format GUID starts with the tag
                if (body + 26 > b.size()) {
                    *err = path + ": truncated fmt chunk";
                    return false;
                }
                tag = le16(&b[body + 24]);
            }
        } else if (std::memcmp(id, "data", 4) == 0) {
            if (body + size > b.size()) {
                *err = path + ": truncated data chunk";
                return false;
            }
            data.assign(b.begin() + (ptrdiff_t)body, b.begin() + (ptrdiff_t)(body + size));
            have_data = true;
        } else if (std::memcmp(id, "smpl", 4) == 0) {
            if (body + padded > b.size()) {
                *err = path + ": truncated smpl chunk";
                return false;
            }
            if (padded >= 36) {
                const uint8_t* s = &b[body];
                const uint32_t midi_note = le32(s + 20), pitch_frac = le32(s + 24), num_loops = le32(s + 28);
                if (midi_note < 128) {
                    w->has_root = true;
                    w->root_key = (uint8_t)midi_note;
                }
                // MIDIPitchFraction: a 0.32 fraction of a semitone
                w->fine_tune_cents = (float)((double)pitch_frac / 4294967296.0 * 100.0);
                if (num_loops > 0 && padded >= 36 + 24) {
                    w->has_loop = true;
                    w->loop_start = le32(s + 44);
                    w->loop_end = le32(s + 48);
                }
            }
        }
        pos = body + (size_t)padded;
    }
    if (!have_data) {
        *err = path + ": no data chunk";
        return false;
    }
    if (w->channels == 0) {
        *err = path + ": no fmt chunk";
        return false;
    }
    if (!decode_samples(data, tag, bits, w->interleaved)) {
        *err = path + ": unsupported format tag " + std::to_string(tag) + " / " + std::to_string(bits) + " bits";
        return false;
    }
    return true;
}

// ---- text helpers ------------------------------------------------------------------

bool is_ws(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\f'; }

std::string trim(const std::string& s) {
    size_t a = 0, b = s.size();
    while (a < b && is_ws(s[a])) ++a;
    while (b > a && is_ws(s[b - 1])) --b;
    return s.substr(a, b - a);
}

std::string lower(std::string s) {
    for (auto& c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

bool parse_i32(const std::string& v, int32_t* out) {
    // str::parse::<i32>: an optional sign, then digits only
    if (v.empty()) return false;
    size_t i = (v[0] == '+' || v[0] == '-') ? 1 : 0;
    if (i == v.size()) return false;
    for (size_t k = i; k < v.size(); ++k)
        if (!std::isdigit((unsigned char)v[k])) return false;
    errno = 0;
    const long long x = std::strtoll(v.c_str(), nullptr, 10);
    if (errno == ERANGE || x < INT32_MIN || x > INT32_MAX) return false;
    *out = (int32_t)x;
    return true;
}

bool parse_f32(const std::string& v, float* out) {
    // str::parse::<f32>: decimal digits with an optional sign, point and
    // exponent, or inf / infinity / nan (any case); no hex, no surrounding text
    if (v.empty()) return false;
    size_t i = (v[0] == '+' || v[0] == '-') ? 1 : 0;
    const std::string rest = lower(v.substr(i));
    if (rest == "inf" || rest == "infinity" || rest == "nan") {
        const float x = rest == "nan" ? NAN : INFINITY;
        *out = v[0] == '-' ? -x : x;
        return true;
    }
    bool digits = false, point = false;
    size_t k = i;
    for (; k < v.size(); ++k) {
        const char c = v[k];
        if (std::isdigit((unsigned char)c)) digits = true;
        else if (c == '.' && !point) point = true;
        else break;
    }
    if (!digits) return false;
    if (k < v.size() && (v[k] == 'e' || v[k] == 'E')) {
        size_t e = k + 1;
        if (e < v.size() && (v[e] == '+' || v[e] == '-')) ++e;
        if (e == v.size()) return false;
        for (; e < v.size(); ++e)
            if (!std::isdigit((unsigned char)v[e])) return false;
        k = v.size();
    }
    if (k != v.size()) return false;
    *out = std::strtof(v.c_str(), nullptr);
    return true;
}

// Saturating f32 -> i32, NaN to 0 (Rust's `as`).
int32_t sat_i32(float f) {
    if (std::isnan(f)) return 0;
    if (f >= 2147483647.0f) return INT32_MAX;
    if (f <= -2147483648.0f) return INT32_MIN;
    return (int32_t)f;
}
uint32_t sat_u32(double f) {
    if (!(f > 0.0)) return 0;
    if (f >= 4294967295.0) return UINT32_MAX;
    return (uint32_t)f;
}

}  // namespace

// parse_note_name (src/sfz.rs:88-116): `c4` = 60, sharps `#`, flats `b`,
// octave -1 written `c-1`.
bool sfz_note_name(const std::string& s, int32_t* out) {
    if (s.empty()) return false;
    int32_t step;
    switch (std::tolower((unsigned char)s[0])) {
        case 'c': step = 0; break;
        case 'd': step = 2; break;
        case 'e': step = 4; break;
        case 'f': step = 5; break;
        case 'g': step = 7; break;
        case 'a': step = 9; break;
        case 'b': step = 11; break;
        default: return false;
    }
    size_t i = 1;
    int32_t acc = 0;
    while (i < s.size() && (s[i] == '#' || s[i] == 'b' || (s[i] == '-' && i == 1))) {
        if (s[i] == '#') acc += 1;
        else if (s[i] == 'b') acc -= 1;
        else break;
        ++i;
    }
    int32_t octave;
    if (!parse_i32(trim(s.substr(i)), &octave)) return false;
    *out = (octave + 1) * 12 + step + acc;
    return true;
}

// find_value_end (src/sfz.rs:233-260): a value runs to just before the last
// whitespace-separated token that holds an `=` (or a `<`), so file names
// with spaces survive.
size_t sfz_value_end(const std::string& s) {
    size_t i = 0;
    bool have_ws = false;
    size_t last_ws = 0;
    while (i < s.size()) {
        if (s[i] == '=') return have_ws ? last_ws : i;
        if (s[i] == '<') return have_ws ? last_ws : i;
        if (is_ws(s[i])) {
            size_t j = i;
            while (j < s.size() && is_ws(s[j])) ++j;
            have_ws = true;
            last_ws = i;
            i = j;
            continue;
        }
        ++i;
    }
    return s.size();
}

namespace {

// OpcodeSet (src/sfz.rs:24-86).
struct Ops {
    std::map<std::string, std::string> m;
    Ops merged(const Ops& o) const {
        Ops r = *this;
        for (const auto& [k, v] : o.m) r.m[k] = v;
        return r;
    }
    const std::string* get(const std::string& k) const {
        auto it = m.find(k);
        return it == m.end() ? nullptr : &it->second;
    }
    // Aliases collapse to one name at the level that wrote them, before any
    // inheritance; an explicit sibling at the same level wins.
    void canonicalise() {
        if (auto it = m.find("key"); it != m.end()) {
            const std::string k = it->second;
            m.erase(it);
            for (const char* alias : {"lokey", "hikey", "pitch_keycenter"}) m.emplace(alias, k);
        }
        for (auto [from, to] : {std::pair<const char*, const char*>{"loopmode", "loop_mode"},
                                {"loopstart", "loop_start"},
                                {"loopend", "loop_end"},
                                {"pitch", "tune"}}) {
            if (auto it = m.find(from); it != m.end()) {
                const std::string v = it->second;
                m.erase(it);
                m.emplace(to, v);
            }
        }
    }
    bool f32(const std::string& k, float* out) const {
        const std::string* v = get(k);
        return v && parse_f32(trim(*v), out);
    }
    bool i32(const std::string& k, int32_t* out) const {
        const std::string* v = get(k);
        if (!v) return false;
        const std::string t = trim(*v);
        if (parse_i32(t, out)) return true;
        float f;
        if (!parse_f32(t, &f)) return false;
        *out = sat_i32(f);
        return true;
    }
    bool key(const std::string& k, int32_t* out) const {
        const std::string* v = get(k);
        if (!v) return false;
        const std::string t = trim(*v);
        return parse_i32(t, out) || sfz_note_name(t, out);
    }
};

bool path_exists(const std::string& p) {
    struct stat st;
    return ::stat(p.c_str(), &st) == 0;
}

std::string join(const std::string& a, const std::string& b) {
    if (b.empty()) return a;
    if (!b.empty() && b[0] == '/') return b;
    if (a.empty()) return b;
    return a.back() == '/' ? a + b : a + "/" + b;
}

std::string dirname_of(const std::string& p) {
    const size_t s = p.rfind('/');
    return s == std::string::npos ? std::string() : p.substr(0, s);
}

std::string basename_of(const std::string& p) {
    const size_t s = p.rfind('/');
    return s == std::string::npos ? p : p.substr(s + 1);
}

struct Parser {
    std::string root;
    std::map<std::string, uint32_t> unknown;
    uint32_t depth = 0;
    std::vector<std::string> warnings;

    // Parser::resolve: backslashes to slashes, relative to the file's
    // directory, with a case-insensitive match on the file name as a fallback.
    std::string resolve(const std::string& default_path, const std::string& rel_in) const {
        std::string rel = rel_in;
        std::replace(rel.begin(), rel.end(), '\\', '/');
        const std::string cand = join(root, join(default_path, rel));
        if (path_exists(cand)) return cand;
        const std::string parent = dirname_of(cand);
        const std::string name = lower(basename_of(cand));
        if (DIR* d = ::opendir(parent.empty() ? "." : parent.c_str())) {
            std::string found;
            while (dirent* e = ::readdir(d)) {
                if (lower(e->d_name) == name) {
                    found = join(parent, e->d_name);
                    break;
                }
            }
            ::closedir(d);
            if (!found.empty()) return found;
        }
        return cand;
    }

    // Parser::parse_file: headers and opcodes in file order, #include
    // followed in place (16 levels at most), #define lines skipped.
    bool parse_file(const std::string& path, std::vector<std::pair<std::string, Ops>>& out, std::string* err) {
        if (depth > 16) {
            *err = "#include nesting is too deep at " + path;
            return false;
        }
        FILE* f = std::fopen(path.c_str(), "rb");
        if (!f) {
            *err = "reading " + path + ": " + std::strerror(errno);
            return false;
        }
        std::string text;
        {
            char buf[1 << 16];
            size_t n;
            while ((n = std::fread(buf, 1, sizeof(buf), f)) > 0) text.append(buf, n);
            std::fclose(f);
        }
        std::string header = "global";
        Ops current;
        bool started = false;
        size_t p = 0;
        while (p <= text.size()) {
            size_t nl = text.find('\n', p);
            if (nl == std::string::npos) nl = text.size();
            std::string raw = text.substr(p, nl - p);
            p = nl + 1;
            if (!raw.empty() && raw.back() == '\r') raw.pop_back();
            if (const size_t c = raw.find("//"); c != std::string::npos) raw.resize(c);
            const std::string line = trim(raw);
            if (line.empty()) {
                if (nl == text.size()) break;
                continue;
            }
            if (line.rfind("#include", 0) == 0) {
                std::string inc = trim(line.substr(8));
                size_t a = 0, b = inc.size();
                while (a < b && inc[a] == '"') ++a;
                while (b > a && inc[b - 1] == '"') --b;
                inc = trim(inc.substr(a, b - a));
                const std::string ip = resolve("", inc);
                if (started) {
                    out.push_back({header, std::move(current)});
                    current = Ops{};
                    started = false;
                }
                ++depth;
                std::string e2;
                if (!parse_file(ip, out, &e2)) warnings.push_back(e2);
                --depth;
                if (nl == text.size()) break;
                continue;
            }
            if (line.rfind("#define", 0) == 0) {
                if (nl == text.size()) break;
                continue;
            }
            std::string rest = line;
            while (!rest.empty()) {
                size_t a = 0;
                while (a < rest.size() && is_ws(rest[a])) ++a;
                rest = rest.substr(a);
                if (rest.empty()) break;
                if (rest[0] == '<') {
                    const size_t end = rest.find('>', 1);
                    if (end == std::string::npos) break;
                    if (started) out.push_back({header, std::move(current)});
                    header = lower(trim(rest.substr(1, end - 1)));
                    current = Ops{};
                    started = true;
                    rest = rest.substr(end + 1);
                    continue;
                }
                const size_t eq = rest.find('=');
                if (eq == std::string::npos) break;
                const std::string key = lower(trim(rest.substr(0, eq)));
                const std::string after = rest.substr(eq + 1);
                const size_t ve = sfz_value_end(after);
                const std::string value = trim(after.substr(0, ve));
                rest = after.substr(ve);
                if (key.empty()) continue;
                current.m[key] = value;
                started = true;
            }
            if (nl == text.size()) break;
        }
        if (started) out.push_back({header, std::move(current)});
        return true;
    }
};

// The opcodes this loader reads (src/sfz.rs:462-505); the rest are counted.
const char* const KNOWN[] = {"sample", "lokey", "hikey", "key", "lovel", "hivel", "pitch_keycenter", "tune", "pitch",
                             "transpose", "volume", "amp_veltrack", "pan", "pitch_keytrack", "loop_mode", "loopmode",
                             "loop_start", "loop_end", "offset", "end", "ampeg_delay", "ampeg_attack", "ampeg_hold",
                             "ampeg_decay", "ampeg_sustain", "ampeg_release", "cutoff", "resonance", "fil_veltrack",
                             "fil_type", "group", "off_by", "default_path"};
const char* const UNIMPLEMENTED[] = {"amplfo_", "fillfo_", "pitchlfo_", "set_cc", "label_cc"};

void note_unhandled(const Ops& ops, std::map<std::string, uint32_t>& unknown) {
    for (const auto& [k, v] : ops.m) {
        if (std::find_if(std::begin(KNOWN), std::end(KNOWN), [&](const char* x) { return k == x; }) != std::end(KNOWN))
            continue;
        std::string key = k;
        for (const char* p : UNIMPLEMENTED)
            if (k.rfind(p, 0) == 0) {
                key = std::string(p) + "* (not implemented)";
                break;
            }
        unknown[key] += 1;
    }
}

// region_from_opcodes (src/sfz.rs:536-681).
Region region_from_opcodes(const Ops& ops, uint32_t sample, const SampleInfo& info, std::vector<std::string>& extra) {
    Region r;
    r.sample = sample;
    int32_t k;
    if (ops.key("lokey", &k)) r.key_lo = (uint8_t)std::clamp(k, 0, 127);
    if (ops.key("hikey", &k)) r.key_hi = (uint8_t)std::clamp(k, 0, 127);
    if (ops.key("pitch_keycenter", &k)) r.root_key_override = (int16_t)std::clamp(k, 0, 127);
    if (r.root_key_override < 0) r.root_key_override = (int16_t)info.root_key;
    if (ops.i32("lovel", &k)) r.vel_lo = (uint8_t)std::clamp(k, 0, 127);
    if (ops.i32("hivel", &k)) r.vel_hi = (uint8_t)std::clamp(k, 0, 127);

    float f = 0.0f;
    float tune = 0.0f;
    ops.f32("tune", &tune);
    r.fine_tune = (int16_t)std::clamp(std::round(tune), -32768.0f, 32767.0f);
    if (ops.i32("transpose", &k)) r.coarse_tune = (int16_t)std::clamp(k, -127, 127);
    if (ops.f32("pitch_keytrack", &f)) r.scale_tuning = (int16_t)std::clamp(std::round(f), -1200.0f, 1200.0f);

    if (ops.f32("volume", &f)) r.attenuation_cb = -f * 10.0f;
    if (ops.f32("pan", &f)) r.pan = std::clamp(f / 100.0f, -1.0f, 1.0f);
    if (ops.f32("amp_veltrack", &f)) r.amp_veltrack = std::clamp(f, -100.0f, 100.0f);

    const std::string* lm = ops.get("loop_mode");
    const std::string mode = lm ? *lm : std::string();
    if (mode == "loop_continuous") r.loop_mode = LoopMode::Continuous;
    else if (mode == "loop_sustain") r.loop_mode = LoopMode::UntilRelease;
    else if (mode == "one_shot" || mode == "no_loop") r.loop_mode = LoopMode::NoLoop;
    else r.loop_mode = info.loop_end > info.loop_start + 1 ? LoopMode::Continuous : LoopMode::NoLoop;

    if (ops.i32("offset", &k)) r.addr_start = std::max(k, 0);
    // Absolute positions in source frames; the region stores offsets from
    // the sample's own points, which are at the pool rate.
    auto to_source = [&](uint32_t resampled) -> int32_t {
        if (info.resample_ratio > 0.0f) return sat_i32(std::round((float)resampled / info.resample_ratio));
        return (int32_t)resampled;
    };
    if (ops.i32("end", &k) && k > 0) r.addr_end = k - to_source(info.len);
    if (ops.i32("loop_start", &k)) r.addr_loop_start = k - to_source(info.loop_start);
    if (ops.i32("loop_end", &k)) r.addr_loop_end = k - to_source(info.loop_end);

    auto env = [&](const char* name, float dflt) {
        float v = dflt;
        ops.f32(name, &v);
        return v;
    };
    r.delay = std::max(env("ampeg_delay", 0.0f), 0.0f);
    r.attack = std::max(env("ampeg_attack", 0.001f), 0.0f);
    r.hold = std::max(env("ampeg_hold", 0.0f), 0.0f);
    r.decay = std::max(env("ampeg_decay", 100.0f), 0.0f);
    r.sustain = std::clamp(env("ampeg_sustain", 100.0f) / 100.0f, 0.0f, 1.0f);
    r.release = std::max(env("ampeg_release", 0.05f), 0.0f);

    if (ops.f32("cutoff", &f) && f > 0.0f) r.filter_fc_cents = 1200.0f * std::log2(f / 8.176f);
    if (ops.f32("resonance", &f)) r.filter_q_cb = f * 10.0f;
    if (ops.f32("fil_veltrack", &f)) r.filter_veltrack_cents = std::clamp(f, -9600.0f, 9600.0f);
    // only lowpasses are implemented: any other type turns the filter off
    if (const std::string* t = ops.get("fil_type"); t && t->rfind("lpf", 0) != 0) {
        r.filter_fc_cents = 13500.0f;
        r.filter_veltrack_cents = 0.0f;
    }
    // `off_by` naming the region's own `group` is the self-exclusive case
    int32_t group_id = 0;
    ops.i32("group", &group_id);
    group_id = std::clamp(group_id, 0, 255);
    int32_t off;
    if (ops.i32("off_by", &off)) {
        if (std::clamp(off, 0, 255) == group_id && group_id > 0) r.exclusive_class = (uint8_t)group_id;
        else extra.push_back("off_by (cross-group, not implemented)");
    }
    return r;
}

constexpr uint32_t POOL_GUARD = 8;

struct SampleKey {
    std::string path;
    size_t ch;
    bool operator<(const SampleKey& o) const { return path != o.path ? path < o.path : ch < o.ch; }
};

// load_sample_channels (src/sfz.rs:417-486): one sample per channel (two at
// most), read once per path.
bool load_sample_channels(const std::string& spath, Bank& b, std::map<SampleKey, uint32_t>& cache, uint32_t pool_rate,
                          std::vector<uint32_t>& out, std::string* err) {
    out.clear();
    if (auto it = cache.find({spath, 0}); it != cache.end()) {
        out.push_back(it->second);
        if (auto j = cache.find({spath, 1}); j != cache.end()) out.push_back(j->second);
        return true;
    }
    WavData w;
    if (!read_wav(spath, &w, err)) return false;
    const size_t nch = std::clamp<size_t>(w.channels, 1, 2);
    for (size_t ch = 0; ch < nch; ++ch) {
        const std::vector<int16_t> raw = w.channel_i16(ch);
        const uint32_t src_rate = std::max<uint32_t>(w.sample_rate, 1);
        const double ratio = pool_rate != 0 && pool_rate != src_rate ? (double)pool_rate / (double)src_rate : 1.0;
        const std::vector<int16_t> data = std::fabs(ratio - 1.0) > 1e-12 ? resample_i16(raw, ratio) : raw;
        const uint32_t len = (uint32_t)data.size();
        uint32_t ls = 0, le = len > 0 ? len - 1 : 0;
        if (w.has_loop) {
            ls = w.loop_start;
            le = w.loop_end;
        }
        ls = sat_u32(std::round((double)ls * ratio));
        le = sat_u32(std::round((double)le * ratio));
        SampleInfo si;
        si.start = (uint32_t)b.pool.size();
        b.pool.insert(b.pool.end(), data.begin(), data.end());
        b.pool.insert(b.pool.end(), POOL_GUARD, 0);
        si.len = len;
        si.loop_start = std::min(ls, len > 0 ? len - 1 : 0);
        si.loop_end = std::min(le, len);
        si.rate = pool_rate != 0 ? pool_rate : src_rate;
        si.root_key = w.has_root ? w.root_key : 60;
        si.correction_cents = w.fine_tune_cents;
        si.resample_ratio = (float)ratio;
        const uint32_t idx = (uint32_t)b.samples.size();
        b.samples.push_back(si);
        cache[{spath, ch}] = idx;
        out.push_back(idx);
    }
    return true;
}

}  // namespace

// sfz::load (src/sfz.rs:262-415).
bool load_sfz_file(const std::string& path, const BankConfig& cfg, Bank* out, std::string* err,
                   std::vector<std::string>* report) {
    Parser parser;
    parser.root = dirname_of(path);
    std::vector<std::pair<std::string, Ops>> sections;
    if (!parser.parse_file(path, sections, err)) return false;
    for (auto& [h, ops] : sections) ops.canonicalise();

    // One walk in file order: each region inherits what is in force where it
    // is written, <control>'s default_path included.
    std::string default_path;
    Ops global, master, group;
    std::vector<std::pair<std::string, Ops>> region_sets;
    for (const auto& [h, ops] : sections) {
        if (h == "control") {
            if (const std::string* dp = ops.get("default_path")) {
                default_path = *dp;
                std::replace(default_path.begin(), default_path.end(), '\\', '/');
            }
        } else if (h == "global") {
            global = ops;
            master = Ops{};
            group = Ops{};
        } else if (h == "master") {
            master = ops;
            group = Ops{};
        } else if (h == "group") {
            group = ops;
        } else if (h == "region") {
            region_sets.push_back({default_path, global.merged(master).merged(group).merged(ops)});
        } else if (h == "curve" || h == "effect") {
        } else {
            parser.unknown["<" + h + ">"] += 1;
        }
    }
    if (region_sets.empty()) {
        *err = path + ": no <region> sections";
        return false;
    }

    Bank& b = *out;
    b = Bank{};
    const uint32_t pool_rate = cfg.resample_pool ? cfg.sample_rate : 0;
    std::map<SampleKey, uint32_t> cache;
    std::vector<uint32_t> region_ids;
    for (const auto& [dp, ops] : region_sets) {
        const std::string* rel = ops.get("sample");
        if (!rel) continue;
        int32_t end;
        if (ops.i32("end", &end) && end == -1) continue;  // the conventional way to disable a region
        const std::string spath = parser.resolve(dp, *rel);
        std::vector<uint32_t> channels;
        std::string e2;
        if (!load_sample_channels(spath, b, cache, pool_rate, channels, &e2)) {
            parser.warnings.push_back(e2);
            continue;
        }
        for (size_t ch = 0; ch < channels.size(); ++ch) {
            note_unhandled(ops, parser.unknown);
            std::vector<std::string> extra;
            Region r = region_from_opcodes(ops, channels[ch], b.samples[channels[ch]], extra);
            for (const auto& x : extra) parser.unknown[x] += 1;
            if (channels.size() == 2) r.pan = ch == 0 ? -1.0f : 1.0f;  // a stereo file's halves, hard panned
            region_ids.push_back((uint32_t)b.regions.size());
            b.regions.push_back(r);
        }
    }
    if (b.regions.empty()) {
        *err = path + ": every region was unusable";
        return false;
    }
    if (report) {
        *report = parser.warnings;
        for (const auto& [op, n] : parser.unknown)
            report->push_back("sfz: ignored unsupported " + op + " (" + std::to_string(n) + " times)");
    }
    Preset p;
    p.bank = 0;
    p.program = 0;
    p.regions = std::move(region_ids);
    b.presets.push_back(std::move(p));
    b.pool_rate = pool_rate;
    b.build_params(cfg);
    b.finish();
    return true;
}

}  // namespace kh
