// sf2.cpp -- src/sf2.rs restated in C++17: the RIFF walk, the pdta records,
// preset and instrument flattening into regions, and the pool build that
// pulls only the used samples out of smpl (resampled to the pool rate). Also
// a writer of the layout src/testkit.rs:130-318 writes, which the synthetic
// banks go through on their way to the same loader.
#include "bank.h"

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <set>
#include <unordered_map>

namespace kh {

namespace {
constexpr uint16_t G_START_ADDRS = 0, G_END_ADDRS = 1, G_STARTLOOP_ADDRS = 2, G_ENDLOOP_ADDRS = 3,
                   G_START_ADDRS_COARSE = 4, G_INITIAL_FILTER_FC = 8, G_INITIAL_FILTER_Q = 9,
                   G_END_ADDRS_COARSE = 12, G_PAN = 17, G_DELAY_VOL_ENV = 33, G_ATTACK_VOL_ENV = 34,
                   G_HOLD_VOL_ENV = 35, G_DECAY_VOL_ENV = 36, G_SUSTAIN_VOL_ENV = 37, G_RELEASE_VOL_ENV = 38,
                   G_KEYNUM_TO_HOLD = 39, G_KEYNUM_TO_DECAY = 40, G_INSTRUMENT = 41, G_KEY_RANGE = 43,
                   G_VEL_RANGE = 44, G_STARTLOOP_ADDRS_COARSE = 45, G_KEYNUM = 46, G_VELOCITY = 47,
                   G_INITIAL_ATTENUATION = 48, G_ENDLOOP_ADDRS_COARSE = 50, G_COARSE_TUNE = 51,
                   G_FINE_TUNE = 52, G_SAMPLE_ID = 53, G_SAMPLE_MODES = 54, G_SCALE_TUNING = 56,
                   G_EXCLUSIVE_CLASS = 57, G_OVERRIDING_ROOT_KEY = 58;
constexpr uint32_t POOL_GUARD = 8;  // src/sf2.rs:581-583

// is_absolute_only, src/sf2.rs:56-77.
bool is_absolute_only(uint16_t op) {
    switch (op) {
        case G_START_ADDRS: case G_END_ADDRS: case G_STARTLOOP_ADDRS: case G_ENDLOOP_ADDRS:
        case G_START_ADDRS_COARSE: case G_END_ADDRS_COARSE: case G_STARTLOOP_ADDRS_COARSE:
        case G_ENDLOOP_ADDRS_COARSE: case G_SAMPLE_ID: case G_SAMPLE_MODES: case G_EXCLUSIVE_CLASS:
        case G_OVERRIDING_ROOT_KEY: case G_KEYNUM: case G_VELOCITY: case G_INSTRUMENT: case G_KEY_RANGE:
        case G_VEL_RANGE:
            return true;
        default:
            return false;
    }
}

// default_generators, src/sf2.rs:79-103.
GenArray default_generators() {
    GenArray g{};
    g[G_INITIAL_FILTER_FC] = 13500;
    g[21] = -12000;
    g[23] = -12000;
    g[25] = -12000;
    g[26] = -12000;
    g[27] = -12000;
    g[28] = -12000;
    g[30] = -12000;
    g[G_DELAY_VOL_ENV] = -12000;
    g[G_ATTACK_VOL_ENV] = -12000;
    g[G_HOLD_VOL_ENV] = -12000;
    g[G_DECAY_VOL_ENV] = -12000;
    g[G_RELEASE_VOL_ENV] = -12000;
    g[G_KEY_RANGE] = (int16_t)0x7F00;
    g[G_VEL_RANGE] = (int16_t)0x7F00;
    g[G_KEYNUM] = -1;
    g[G_VELOCITY] = -1;
    g[G_SCALE_TUNING] = 100;
    g[G_OVERRIDING_ROOT_KEY] = -1;
    return g;
}

// range_of, src/sf2.rs:508-520.
std::pair<uint8_t, uint8_t> range_of(const GenArray& gen, bool set, uint16_t op) {
    if (!set) return {0, 127};
    const uint16_t raw = (uint16_t)gen[op];
    const uint8_t lo = raw & 0xFF, hi = raw >> 8;
    return lo > hi ? std::make_pair(hi, lo) : std::make_pair(lo, hi);
}

// build_region, src/sf2.rs:532-579.
Region build_region(const GenArray& g, uint32_t sample, std::pair<uint8_t, uint8_t> key,
                    std::pair<uint8_t, uint8_t> vel) {
    Region r;
    const float sustain_cb = (float)g[G_SUSTAIN_VOL_ENV];
    r.sample = sample;
    r.key_lo = key.first;
    r.key_hi = key.second;
    r.vel_lo = vel.first;
    r.vel_hi = vel.second;
    r.root_key_override = g[G_OVERRIDING_ROOT_KEY];
    r.fixed_key = g[G_KEYNUM];
    r.fixed_vel = g[G_VELOCITY];
    r.coarse_tune = g[G_COARSE_TUNE];
    r.fine_tune = g[G_FINE_TUNE];
    r.scale_tuning = g[G_SCALE_TUNING];
    r.attenuation_cb = (float)g[G_INITIAL_ATTENUATION];
    r.amp_veltrack = 100.0f;
    r.pan = rclamp((float)g[G_PAN] / 500.0f, -1.0f, 1.0f);
    switch (g[G_SAMPLE_MODES] & 3) {
        case 1: r.loop_mode = LoopMode::Continuous; break;
        case 3: r.loop_mode = LoopMode::UntilRelease; break;
        default: r.loop_mode = LoopMode::NoLoop; break;
    }
    r.addr_start = (int32_t)g[G_START_ADDRS] + (int32_t)g[G_START_ADDRS_COARSE] * 32768;
    r.addr_end = (int32_t)g[G_END_ADDRS] + (int32_t)g[G_END_ADDRS_COARSE] * 32768;
    r.addr_loop_start = (int32_t)g[G_STARTLOOP_ADDRS] + (int32_t)g[G_STARTLOOP_ADDRS_COARSE] * 32768;
    r.addr_loop_end = (int32_t)g[G_ENDLOOP_ADDRS] + (int32_t)g[G_ENDLOOP_ADDRS_COARSE] * 32768;
    r.exclusive_class = (uint8_t)std::clamp<int>(g[G_EXCLUSIVE_CLASS], 0, 255);
    r.delay = timecents_to_secs((float)g[G_DELAY_VOL_ENV]);
    r.attack = timecents_to_secs((float)g[G_ATTACK_VOL_ENV]);
    r.hold = timecents_to_secs((float)g[G_HOLD_VOL_ENV]);
    r.decay = timecents_to_secs((float)g[G_DECAY_VOL_ENV]);
    r.sustain = cb_to_gain(rmax(sustain_cb, 0.0f));
    r.release = timecents_to_secs((float)g[G_RELEASE_VOL_ENV]);
    r.keynum_to_hold = g[G_KEYNUM_TO_HOLD];
    r.keynum_to_decay = g[G_KEYNUM_TO_DECAY];
    r.filter_fc_cents = (float)g[G_INITIAL_FILTER_FC];
    r.filter_q_cb = (float)g[G_INITIAL_FILTER_Q];
    return r;
}

int16_t sat_add16(int16_t a, int16_t b) {
    const int32_t s = (int32_t)a + b;
    return (int16_t)std::clamp<int32_t>(s, -32768, 32767);
}

uint16_t le16(const uint8_t* p) { return (uint16_t)(p[0] | p[1] << 8); }
uint32_t le32(const uint8_t* p) { return (uint32_t)p[0] | (uint32_t)p[1] << 8 | (uint32_t)p[2] << 16 | (uint32_t)p[3] << 24; }

// The bytes of a soundfont: a file read by offset, or a buffer.
class Source {
   public:
    virtual ~Source() = default;
    virtual uint64_t size() const = 0;
    // false when fewer than n bytes are there (read_exact's error)
    virtual bool read(uint64_t off, void* dst, size_t n) = 0;
};

class FileSource : public Source {
   public:
    explicit FileSource(FILE* f) : f_(f) {
        if (std::fseek(f_, 0, SEEK_END) == 0) len_ = (uint64_t)ftello(f_);
    }
    ~FileSource() override { std::fclose(f_); }
    uint64_t size() const override { return len_; }
    bool read(uint64_t off, void* dst, size_t n) override {
        if (off > len_ || n > len_ - off) return false;
        if (fseeko(f_, (off_t)off, SEEK_SET) != 0) return false;
        return std::fread(dst, 1, n, f_) == n;
    }

   private:
    FILE* f_;
    uint64_t len_ = 0;
};

class MemSource : public Source {
   public:
    explicit MemSource(const std::vector<uint8_t>& b) : b_(b) {}
    uint64_t size() const override { return b_.size(); }
    bool read(uint64_t off, void* dst, size_t n) override {
        if (off > b_.size() || n > b_.size() - off) return false;
        std::memcpy(dst, b_.data() + off, n);
        return true;
    }

   private:
    const std::vector<uint8_t>& b_;
};

struct Chunk {
    char id[4];
    uint64_t offset, size;
};

bool chunk_header(Source& s, uint64_t pos, char id[4], uint32_t* size) {
    uint8_t h[8];
    if (!s.read(pos, h, 8)) return false;
    std::memcpy(id, h, 4);
    *size = le32(h + 4);
    return true;
}

std::string id_str(const char id[4]) { return std::string(id, 4); }

// scan_chunks, src/sf2.rs:153-207: the RIFF tree without its payloads. Sizes
// are clamped to what the file holds; an odd size is followed by a pad byte.
bool scan_chunks(Source& s, std::vector<Chunk>& sdta, std::vector<Chunk>& pdta, std::string* err) {
    const uint64_t file_len = s.size();
    char id[4];
    uint32_t sz;
    char form[4];
    if (!chunk_header(s, 0, id, &sz) || std::memcmp(id, "RIFF", 4) != 0) {
        *err = "not a RIFF file";
        return false;
    }
    if (!s.read(8, form, 4)) {
        *err = "truncated RIFF header";
        return false;
    }
    if (std::memcmp(form, "sfbk", 4) != 0) {
        *err = "RIFF form is " + id_str(form) + ", expected sfbk";
        return false;
    }
    uint64_t pos = 12;
    while (pos + 8 <= file_len) {
        if (!chunk_header(s, pos, id, &sz)) break;
        const uint64_t size = std::min<uint64_t>(sz, file_len - pos - 8);
        if (std::memcmp(id, "LIST", 4) == 0) {
            char list_id[4];
            if (!s.read(pos + 8, list_id, 4)) {
                *err = "truncated LIST chunk";
                return false;
            }
            std::vector<Chunk>* target = std::memcmp(list_id, "sdta", 4) == 0   ? &sdta
                                         : std::memcmp(list_id, "pdta", 4) == 0 ? &pdta
                                                                                : nullptr;
            if (target) {
                const uint64_t list_end = pos + 8 + size;
                uint64_t inner = pos + 12;
                while (inner + 8 <= list_end) {
                    char cid[4];
                    uint32_t csz;
                    if (!chunk_header(s, inner, cid, &csz)) break;
                    const uint64_t c = std::min<uint64_t>(csz, list_end - inner - 8);
                    Chunk ch;
                    std::memcpy(ch.id, cid, 4);
                    ch.offset = inner + 8;
                    ch.size = c;
                    target->push_back(ch);
                    inner += 8 + c + (c & 1);
                }
            }
        }
        pos += 8 + size + (size & 1);
    }
    return true;
}

const Chunk* find_chunk(const std::vector<Chunk>& v, const char* id) {
    for (const auto& c : v)
        if (std::memcmp(c.id, id, 4) == 0) return &c;
    return nullptr;
}

struct Bag {
    uint16_t gen_ndx;
};
struct Gen {
    uint16_t op;
    int16_t amount;
};
struct Shdr {
    uint32_t start, end, start_loop, end_loop, rate;
    uint8_t original_pitch;
    int8_t pitch_correction;
    uint16_t sample_type;
};
struct Phdr {
    uint16_t preset, bank, bag_ndx;
};

// The records of one pdta chunk, whole records only (chunks_exact).
template <class T, size_t N, class F>
bool load_records(Source& s, const std::vector<Chunk>& pdta, const char* id, F decode, std::vector<T>& out,
                  std::string* err) {
    const Chunk* c = find_chunk(pdta, id);
    if (!c) {
        *err = std::string("pdta is missing ") + id;
        return false;
    }
    std::vector<uint8_t> raw((size_t)c->size);
    if (!s.read(c->offset, raw.data(), raw.size())) {
        *err = std::string("reading ") + id;
        return false;
    }
    out.clear();
    for (size_t i = 0; i + N <= raw.size(); i += N) out.push_back(decode(raw.data() + i));
    return true;
}

// build_pool, src/sf2.rs:585-703, with the used samples' data already read:
// the pool rate halves until the pool fits the budget (down to 8 kHz), each
// used sample is resampled to it, and regions are remapped to the dense
// sample list.
void build_pool(const std::map<uint32_t, Sf2Sample>& used, size_t n_shdrs, std::vector<Region>& regions,
                const BankConfig& cfg, Bank& b) {
    uint32_t pool_rate = cfg.resample_pool ? cfg.sample_rate : 0;
    if (pool_rate != 0) {
        for (;;) {
            uint64_t est = 0;
            for (const auto& [sid, s] : used) {
                const double n = (double)s.data.size() * (double)pool_rate / (double)std::max<uint32_t>(s.rate, 1);
                est += sat_cast<uint64_t>(n) + POOL_GUARD;
            }
            if (est * 2 <= cfg.sample_pool_budget || pool_rate <= 8000) break;
            pool_rate /= 2;
        }
    }
    std::vector<uint32_t> remap(n_shdrs, UINT32_MAX);
    // With a batch resampler installed, every sample that needs converting
    // goes to it in one call (one sinc table per distinct ratio).
    std::unordered_map<uint32_t, std::vector<int16_t>> converted;
    if (const ResampleHook hook = resample_hook(); hook.fn && pool_rate != 0) {
        std::vector<uint32_t> ids, src_len, dst_len;
        std::vector<const int16_t*> src;
        std::vector<double> ratios;
        std::vector<const float*> tabs;
        std::vector<int16_t*> dst;
        std::unordered_map<uint64_t, std::vector<float>> tables;  // by the ratio's bits
        for (const auto& [sid, sh] : used) {
            const uint32_t src_rate = std::max<uint32_t>(sh.rate, 1);
            if (pool_rate == src_rate || sh.data.empty()) continue;
            const double ratio = (double)pool_rate / (double)src_rate;
            if (std::fabs(ratio - 1.0) < 1e-12) continue;
            uint64_t key;
            std::memcpy(&key, &ratio, 8);
            auto it = tables.find(key);
            if (it == tables.end()) it = tables.emplace(key, sinc_table(ratio)).first;
            const size_t out_len = std::max<size_t>(sat_cast<size_t>(std::round((double)sh.data.size() * ratio)), 1);
            auto& out = converted[sid];
            out.resize(out_len);
            ids.push_back(sid);
            src.push_back(sh.data.data());
            src_len.push_back((uint32_t)sh.data.size());
            ratios.push_back(ratio);
            tabs.push_back(it->second.data());
            dst.push_back(out.data());
            dst_len.push_back((uint32_t)out_len);
        }
        if (!ids.empty() && hook.fn(hook.user, (uint32_t)ids.size(), src.data(), src_len.data(), ratios.data(),
                                    tabs.data(), dst.data(), dst_len.data()) != 0)
            converted.clear();  // the host loop below converts them instead
    }
    for (const auto& [sid, sh] : used) {
        const uint32_t src_rate = std::max<uint32_t>(sh.rate, 1);
        uint32_t loop_start = sh.loop_start, loop_end = sh.loop_end;
        std::vector<int16_t> data;
        if (pool_rate != 0 && pool_rate != src_rate) {
            const double ratio = (double)pool_rate / (double)src_rate;
            if (auto it = converted.find(sid); it != converted.end()) data = std::move(it->second);
            else data = resample_i16(sh.data, ratio);
            loop_start = sat_cast<uint32_t>(std::round((double)loop_start * ratio));
            loop_end = sat_cast<uint32_t>(std::round((double)loop_end * ratio));
        } else {
            data = sh.data;
        }
        const uint32_t len = (uint32_t)data.size();
        loop_start = std::min(loop_start, len > 0 ? len - 1 : 0);
        loop_end = std::min(loop_end, len);
        SampleInfo si;
        si.start = (uint32_t)b.pool.size();
        b.pool.insert(b.pool.end(), data.begin(), data.end());
        b.pool.insert(b.pool.end(), POOL_GUARD, 0);
        si.len = len;
        si.loop_start = loop_start;
        si.loop_end = loop_end;
        si.rate = pool_rate != 0 ? pool_rate : src_rate;
        si.root_key = std::min<uint8_t>(sh.root, 127);
        si.correction_cents = (float)sh.correction;
        si.resample_ratio = pool_rate != 0 ? (float)pool_rate / (float)src_rate : 1.0f;
        remap[sid] = (uint32_t)b.samples.size();
        b.samples.push_back(si);
    }
    for (auto& r : regions) r.sample = r.sample < remap.size() ? remap[r.sample] : UINT32_MAX;
    b.pool_rate = pool_rate;
}

// sf2::load, src/sf2.rs:221-505.
bool load_source(Source& s, const BankConfig& cfg, Bank* bank, std::string* err) {
    std::vector<Chunk> sdta, pdta;
    if (!scan_chunks(s, sdta, pdta, err)) {
        *err = "scanning RIFF structure: " + *err;
        return false;
    }
    const Chunk* smpl = find_chunk(sdta, "smpl");
    if (!smpl) {
        *err = "soundfont has no smpl chunk";
        return false;
    }
    const uint64_t smpl_offset = smpl->offset;
    const uint32_t smpl_frames = (uint32_t)(smpl->size / 2);

    std::vector<Phdr> phdrs;
    std::vector<Bag> pbags, ibags;
    std::vector<Gen> pgens, igens;
    std::vector<uint16_t> insts;  // bag_ndx
    std::vector<Shdr> shdrs;
    auto bag = [](const uint8_t* c) { return Bag{le16(c)}; };
    auto gen = [](const uint8_t* c) { return Gen{le16(c), (int16_t)le16(c + 2)}; };
    if (!load_records<Phdr, 38>(s, pdta, "phdr", [](const uint8_t* c) { return Phdr{le16(c + 20), le16(c + 22), le16(c + 24)}; },
                                phdrs, err) ||
        !load_records<Bag, 4>(s, pdta, "pbag", bag, pbags, err) ||
        !load_records<Gen, 4>(s, pdta, "pgen", gen, pgens, err) ||
        !load_records<uint16_t, 22>(s, pdta, "inst", [](const uint8_t* c) { return le16(c + 20); }, insts, err) ||
        !load_records<Bag, 4>(s, pdta, "ibag", bag, ibags, err) ||
        !load_records<Gen, 4>(s, pdta, "igen", gen, igens, err) ||
        !load_records<Shdr, 46>(s, pdta, "shdr",
                                [](const uint8_t* c) {
                                    return Shdr{le32(c + 20), le32(c + 24), le32(c + 28), le32(c + 32), le32(c + 36),
                                                c[40], (int8_t)c[41], le16(c + 44)};
                                },
                                shdrs, err))
        return false;
    if (phdrs.size() < 2) {
        *err = "soundfont has no presets";
        return false;
    }

    // ---- flatten every preset into regions (src/sf2.rs:309-467) ----
    // phdr, pbag, inst and ibag each end in a terminal record whose index
    // bounds the one before it.
    std::vector<Region> regions;
    std::vector<Preset> presets;
    std::set<uint32_t> used;
    for (size_t pi = 0; pi + 1 < phdrs.size(); ++pi) {
        const Phdr& ph = phdrs[pi];
        const size_t bag_lo = ph.bag_ndx, bag_hi = phdrs[pi + 1].bag_ndx;
        if (bag_lo >= bag_hi || bag_hi > pbags.size()) continue;
        GenArray preset_global{};
        std::array<bool, GEN_COUNT> preset_global_set{};
        bool first_zone = true;
        std::vector<uint32_t> region_ids;
        for (size_t bi = bag_lo; bi < bag_hi; ++bi) {
            const size_t g_lo = pbags[bi].gen_ndx;
            const size_t g_hi = bi + 1 < pbags.size() ? pbags[bi + 1].gen_ndx : pgens.size();
            if (g_lo > g_hi || g_hi > pgens.size()) continue;
            GenArray zone{};
            std::array<bool, GEN_COUNT> zone_set{};
            bool has_inst = false;
            uint16_t inst_idx = 0;
            for (size_t gi = g_lo; gi < g_hi; ++gi) {
                const Gen& g = pgens[gi];
                if (g.op == G_INSTRUMENT) {
                    has_inst = true;
                    inst_idx = (uint16_t)g.amount;
                } else if (g.op < GEN_COUNT) {
                    zone[g.op] = g.amount;
                    zone_set[g.op] = true;
                }
            }
            if (!has_inst) {
                // only the first zone may be the global one
                if (first_zone) {
                    preset_global = zone;
                    preset_global_set = zone_set;
                }
                first_zone = false;
                continue;
            }
            first_zone = false;
            GenArray p_gen = preset_global;
            std::array<bool, GEN_COUNT> p_set = preset_global_set;
            for (int i = 0; i < GEN_COUNT; ++i)
                if (zone_set[i]) {
                    p_gen[i] = zone[i];
                    p_set[i] = true;
                }
            const auto p_key = range_of(p_gen, p_set[G_KEY_RANGE], G_KEY_RANGE);
            const auto p_vel = range_of(p_gen, p_set[G_VEL_RANGE], G_VEL_RANGE);
            if (inst_idx >= insts.size()) continue;
            const size_t ib_lo = insts[inst_idx];
            const size_t ib_hi = (size_t)inst_idx + 1 < insts.size() ? insts[inst_idx + 1] : ibags.size();
            if (ib_lo >= ib_hi || ib_hi > ibags.size()) continue;
            GenArray inst_global = default_generators();
            bool first_izone = true;
            for (size_t ibi = ib_lo; ibi < ib_hi; ++ibi) {
                const size_t ig_lo = ibags[ibi].gen_ndx;
                const size_t ig_hi = ibi + 1 < ibags.size() ? ibags[ibi + 1].gen_ndx : igens.size();
                if (ig_lo > ig_hi || ig_hi > igens.size()) continue;
                GenArray i_gen = inst_global;
                bool has_sample = false;
                uint16_t sid = 0;
                for (size_t gi = ig_lo; gi < ig_hi; ++gi) {
                    const Gen& g = igens[gi];
                    if (g.op == G_SAMPLE_ID) {
                        has_sample = true;
                        sid = (uint16_t)g.amount;
                    } else if (g.op < GEN_COUNT) {
                        i_gen[g.op] = g.amount;
                    }
                }
                if (!has_sample) {
                    if (first_izone) inst_global = i_gen;
                    first_izone = false;
                    continue;
                }
                first_izone = false;
                if (sid >= shdrs.size()) continue;
                const Shdr& sh = shdrs[sid];
                if (sh.sample_type & 0x8000) continue;  // a ROM sample: there is no ROM
                if (sh.end <= sh.start || sh.end > smpl_frames) continue;
                const auto i_key = range_of(i_gen, true, G_KEY_RANGE);
                const auto i_vel = range_of(i_gen, true, G_VEL_RANGE);
                const uint8_t klo = std::max(p_key.first, i_key.first), khi = std::min(p_key.second, i_key.second);
                const uint8_t vlo = std::max(p_vel.first, i_vel.first), vhi = std::min(p_vel.second, i_vel.second);
                if (klo > khi || vlo > vhi) continue;
                // preset generators offset the instrument's, except those the
                // format reserves to instruments
                GenArray f = i_gen;
                for (int op = 0; op < GEN_COUNT; ++op)
                    if (p_set[op] && !is_absolute_only((uint16_t)op)) f[op] = sat_add16(f[op], p_gen[op]);
                used.insert(sid);
                region_ids.push_back((uint32_t)regions.size());
                regions.push_back(build_region(f, sid, {klo, khi}, {vlo, vhi}));
            }
        }
        if (!region_ids.empty()) {
            Preset p;
            p.bank = ph.bank;
            p.program = ph.preset;
            p.regions = std::move(region_ids);
            presets.push_back(std::move(p));
        }
    }
    if (presets.empty()) {
        *err = "no usable presets";
        return false;
    }

    // ---- the referenced sample data, in sample-id order ----
    std::map<uint32_t, Sf2Sample> data;
    for (uint32_t sid : used) {
        const Shdr& sh = shdrs[sid];
        Sf2Sample& d = data[sid];
        d.data.resize(sh.end - sh.start);
        if (!s.read(smpl_offset + (uint64_t)sh.start * 2, d.data.data(), d.data.size() * 2)) {
            *err = "reading sample " + std::to_string(sid);
            return false;
        }
        d.rate = sh.rate;
        d.loop_start = sh.start_loop > sh.start ? sh.start_loop - sh.start : 0;
        d.loop_end = sh.end_loop > sh.start ? sh.end_loop - sh.start : 0;
        d.root = sh.original_pitch;
        d.correction = sh.pitch_correction;
    }
    Bank& b = *bank;
    b = Bank{};
    build_pool(data, shdrs.size(), regions, cfg, b);
    b.regions = std::move(regions);
    b.presets = std::move(presets);
    b.build_params(cfg);
    b.finish();
    return true;
}

// ---- the test kit's writer (src/testkit.rs:136-318) ----------------------------

void put16(std::vector<uint8_t>& v, uint16_t x) {
    v.push_back((uint8_t)x);
    v.push_back((uint8_t)(x >> 8));
}
void put32(std::vector<uint8_t>& v, uint32_t x) {
    put16(v, (uint16_t)x);
    put16(v, (uint16_t)(x >> 16));
}
void put_name(std::vector<uint8_t>& v, const std::string& s) {
    uint8_t b[20] = {};
    std::memcpy(b, s.data(), std::min<size_t>(s.size(), 19));
    v.insert(v.end(), b, b + 20);
}
// A chunk: id, size, payload, and a pad byte after an odd payload.
void put_chunk(std::vector<uint8_t>& v, const char* id, const std::vector<uint8_t>& payload) {
    v.insert(v.end(), id, id + 4);
    put32(v, (uint32_t)payload.size());
    v.insert(v.end(), payload.begin(), payload.end());
    if (payload.size() & 1) v.push_back(0);
}
// A ZSTR: the string and one or two zero bytes, making the length even.
std::vector<uint8_t> zstr(const std::string& s) {
    std::vector<uint8_t> v(s.begin(), s.end());
    v.push_back(0);
    if (v.size() & 1) v.push_back(0);
    return v;
}
}  // namespace

bool write_sf2(const Sf2& sf, std::vector<uint8_t>* out, std::string* err) {
    constexpr size_t SAMPLE_GAP = 46;  // zero frames after each sample in smpl
    // the format's record indexes are 16 bits
    size_t n_pgen = 1, n_igen = 1, n_ibag = 1, frames_total = 0;
    for (const auto& p : sf.presets) n_pgen += p.gens.size() + 1;
    for (const auto& i : sf.instruments) {
        n_ibag += i.size();
        for (const auto& z : i) n_igen += z.gens.size() + 3;
    }
    for (const auto& s : sf.samples) frames_total += s.data.size() + SAMPLE_GAP;
    if (sf.presets.size() + 1 > 65536 || sf.instruments.size() + 1 > 65536 || sf.samples.size() > 65536 ||
        n_pgen > 65536 || n_igen > 65536 || n_ibag > 65536 || frames_total > 0xFFFFFFFFull) {
        *err = "soundfont exceeds the SF2 format's 16-bit record indexes or 32-bit sample offsets";
        return false;
    }
    std::vector<uint8_t> smpl;
    std::vector<std::pair<uint32_t, uint32_t>> ranges;
    uint32_t frames = 0;
    for (const auto& s : sf.samples) {
        const uint32_t start = frames;
        for (int16_t x : s.data) put16(smpl, (uint16_t)x);
        frames += (uint32_t)s.data.size();
        ranges.push_back({start, frames});
        smpl.insert(smpl.end(), SAMPLE_GAP * 2, 0);
        frames += SAMPLE_GAP;
    }
    std::vector<uint8_t> phdr, pbag, pgen, inst, ibag, igen, shdr;
    auto gen = [](std::vector<uint8_t>& v, uint16_t op, uint16_t amount) {
        put16(v, op);
        put16(v, amount);
    };
    for (size_t i = 0; i < sf.presets.size(); ++i) {
        const Sf2Preset& p = sf.presets[i];
        put_name(phdr, "preset " + std::to_string(i));
        put16(phdr, p.program);
        put16(phdr, p.bank);
        put16(phdr, (uint16_t)(pbag.size() / 4));
        put32(phdr, 0);
        put32(phdr, 0);
        put32(phdr, 0);
        put16(pbag, (uint16_t)(pgen.size() / 4));
        put16(pbag, 0);
        for (auto [op, amt] : p.gens) gen(pgen, op, (uint16_t)amt);
        gen(pgen, 41, p.instrument);  // instrument ends a preset zone
    }
    put_name(phdr, "EOP");
    put16(phdr, 0);
    put16(phdr, 0);
    put16(phdr, (uint16_t)(pbag.size() / 4));
    put32(phdr, 0);
    put32(phdr, 0);
    put32(phdr, 0);
    put16(pbag, (uint16_t)(pgen.size() / 4));
    put16(pbag, 0);
    gen(pgen, 0, 0);
    for (size_t i = 0; i < sf.instruments.size(); ++i) {
        put_name(inst, "instrument " + std::to_string(i));
        put16(inst, (uint16_t)(ibag.size() / 4));
        for (const Sf2Zone& z : sf.instruments[i]) {
            put16(ibag, (uint16_t)(igen.size() / 4));
            put16(ibag, 0);
            gen(igen, 43, (uint16_t)(z.key_hi << 8 | z.key_lo));
            gen(igen, 44, (uint16_t)(z.vel_hi << 8 | z.vel_lo));
            for (auto [op, amt] : z.gens) gen(igen, op, (uint16_t)amt);
            gen(igen, 53, z.sample);  // sampleID ends an instrument zone
        }
    }
    put_name(inst, "EOI");
    put16(inst, (uint16_t)(ibag.size() / 4));
    put16(ibag, (uint16_t)(igen.size() / 4));
    put16(ibag, 0);
    gen(igen, 0, 0);
    for (size_t i = 0; i < sf.samples.size(); ++i) {
        const Sf2Sample& s = sf.samples[i];
        const auto [start, end] = ranges[i];
        put_name(shdr, "sample " + std::to_string(i));
        put32(shdr, start);
        put32(shdr, end);
        put32(shdr, start + s.loop_start);
        put32(shdr, start + s.loop_end);
        put32(shdr, s.rate);
        shdr.push_back(s.root);
        shdr.push_back((uint8_t)s.correction);
        put16(shdr, 0);  // sampleLink
        put16(shdr, 1);  // monoSample
    }
    put_name(shdr, "EOS");
    shdr.insert(shdr.end(), 26, 0);

    std::vector<uint8_t> sdta = {'s', 'd', 't', 'a'};
    put_chunk(sdta, "smpl", smpl);
    std::vector<uint8_t> pdta = {'p', 'd', 't', 'a'};
    put_chunk(pdta, "phdr", phdr);
    put_chunk(pdta, "pbag", pbag);
    put_chunk(pdta, "pmod", std::vector<uint8_t>(10, 0));
    put_chunk(pdta, "pgen", pgen);
    put_chunk(pdta, "inst", inst);
    put_chunk(pdta, "ibag", ibag);
    put_chunk(pdta, "imod", std::vector<uint8_t>(10, 0));
    put_chunk(pdta, "igen", igen);
    put_chunk(pdta, "shdr", shdr);
    std::vector<uint8_t> info = {'I', 'N', 'F', 'O'};
    put_chunk(info, "ifil", {2, 0, 1, 0});
    put_chunk(info, "isng", zstr("EMU8000"));
    put_chunk(info, "INAM", zstr("kestrel synthetic"));
    std::vector<uint8_t> body = {'s', 'f', 'b', 'k'};
    put_chunk(body, "LIST", info);
    put_chunk(body, "LIST", sdta);
    put_chunk(body, "LIST", pdta);
    std::vector<uint8_t>& file = *out;
    file = {'R', 'I', 'F', 'F'};
    put32(file, (uint32_t)body.size());
    file.insert(file.end(), body.begin(), body.end());
    return true;
}

bool load_sf2(const Sf2& sf, const BankConfig& cfg, Bank* out, std::string* err) {
    std::vector<uint8_t> bytes;
    if (!write_sf2(sf, &bytes, err)) return false;
    MemSource m(bytes);
    return load_source(m, cfg, out, err);
}

bool load_sf2_file(const std::string& path, const BankConfig& cfg, Bank* out, std::string* err) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) {
        *err = "opening " + path + ": " + std::strerror(errno);
        return false;
    }
    FileSource s(f);
    if (!load_source(s, cfg, out, err)) {
        *err = path + ": " + *err;
        return false;
    }
    return true;
}

}  // namespace kh
