// driver.cpp -- Driver::next_block (src/driver.rs:434-642) and its event,
// admission and controller machinery, restated in C++17, plus the C ABI of
// include/kestrel_host.h.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../../include/kestrel_host.h"
#include "bank.h"
#include "midi.h"
#include "voice.h"

namespace kh {

namespace {
thread_local std::string g_err;

constexpr size_t ADMIT_STRATA = 64;           // src/driver.rs:17-22
constexpr uint16_t RPN_NONE = 0x4000;         // src/driver.rs:24-27
constexpr uint32_t SOUND_CC_SHIFT = 1;        // src/driver.rs:29-37
constexpr double MAX_TAIL_SECONDS = 60.0;     // src/driver.rs:139-140
constexpr uint32_t DEFERRED = UINT32_MAX;     // src/driver.rs:240-241
constexpr float FRAC_PI_2_F = 1.57079632679489661923f;
constexpr float SQRT_2_F = 1.41421356237309504880f;

// note_pack / note_unpack, src/driver.rs:185-206.
inline uint64_t note_pack(uint8_t ch, uint8_t key, uint8_t vel, uint32_t variant, uint32_t rel) {
    return (uint64_t)(ch & 0xF) | ((uint64_t)(key & 0x7F) << 4) | ((uint64_t)(vel & 0x7F) << 11) |
           ((uint64_t)(variant & 0x3F) << 18) | ((uint64_t)(rel & 0xFFFF) << 24);
}

// Cand, src/driver.rs:208-238.
struct Cand {
    uint64_t key;
    uint32_t note, region, id_off;
};

// rank_key, src/driver.rs:243-247.
inline uint64_t rank_key(float gl, float gr, size_t index) {
    return (rank_gain_q(gl, gr) << 48) | mix48((uint64_t)index);
}

inline double rfract(double x) { return x - std::trunc(x); }
}  // namespace

std::string& last_error() { return g_err; }


struct Driver {
    kc_config cfg{};
    kh_options opt{};
    BankConfig bcfg;
    const Bank* bank = nullptr;
    std::unique_ptr<EventSource> stream;
    TempoClock clock;
    GateTable gates;
    ChannelTable chan;

    uint8_t bank_msb[16] = {}, bank_lsb[16] = {};
    uint32_t preset[16] = {};
    int16_t bend_val[16] = {};
    double bend_range[16];
    uint16_t rpn_sel[16] = {};
    uint8_t cc_volume[16], cc_expression[16], cc_pan[16];
    uint8_t cc_sound[16][5];
    uint8_t cc_mod[16] = {}, cc_vib_rate[16], cc_vib_depth[16], cc_tremolo[16] = {}, cc_soft[16] = {};
    uint8_t lsb_mod[16] = {}, lsb_volume[16] = {}, lsb_pan[16] = {}, lsb_expression[16] = {};
    double lfo_phase[16] = {};
    std::vector<std::array<uint8_t, 5>> variants, seen_states;
    uint32_t cur_variant[16] = {};
    uint64_t variant_used = 1;
    std::vector<uint64_t> variant_seen;
    uint64_t variant_clock = 0;
    std::vector<std::pair<uint32_t, ParamMod>> pending_variants;
    bool spawn_variants = false;

    uint64_t next_note_id = 1, block_index = 0;
    bool have_pending = false;
    uint64_t pending_tick = 0;
    Event pending_ev;
    bool stream_done = false, end_sent = false;
    uint64_t tail_blocks_left = 0;

    std::vector<kc_spawn_cmd> spawn_buf;
    std::vector<uint64_t> notes;
    std::vector<uint32_t> note_ordinal;
    std::vector<Cand> cands;
    std::vector<kc_spawn_cmd> deferred_now;
    std::vector<PreviewLayer> preview_buf;
    uint64_t block_first_id = 0;
    std::vector<std::pair<uint64_t, kc_spawn_cmd>> deferred;

    // variants built this block, for kh_driver_variant
    std::vector<std::pair<uint32_t, std::vector<kc_region_params>>> built;
    uint64_t notes_total = 0;
    uint32_t last_want = 0, last_take = 0, last_live = 0;
    uint64_t last_want_energy = 0, last_take_energy = 0;
    // What finish() decides the next block by, as each admitted block left
    // it, by block parity: a pipelined caller may admit block n + 1 before
    // asking about block n.
    bool done_after_admit[2] = {false, false};

    // Driver::open, src/driver.rs:343-413.
    // The event source is the synthetic stream of `m`, or `file` when given.
    Driver(const kc_config& c, const kh_options& o, const Bank& b, const kh_midi_spec& m,
           std::unique_ptr<EventSource> file = nullptr)
        : cfg(c), opt(o), bank(&b) {
        bcfg.sample_rate = c.sample_rate;
        bcfg.env_floor = c.env_floor;
        bcfg.exp_decay = c.decay_curve == KC_CURVE_EXPONENTIAL;
        bcfg.exp_release = c.release_curve == KC_CURVE_EXPONENTIAL;
        bcfg.filter_enabled = o.filter_enabled != 0;
        bcfg.master_volume = o.master_volume;
        if (file) stream = std::move(file);
        else stream = std::make_unique<SynthMidi>(m);
        if (o.read_ahead) stream = std::make_unique<AheadSource>(std::move(stream));
        clock = TempoClock(stream->division(), c.sample_rate);
        gates.init(c.block_frames, c.gate_frames);
        chan.init(c.block_frames, c.gate_frames);
        for (int i = 0; i < 16; ++i) {
            bend_range[i] = 2.0;
            cc_volume[i] = (uint8_t)std::min<uint32_t>(o.default_channel_volume, 127);
            cc_expression[i] = 127;
            cc_pan[i] = 64;
            for (int w = 0; w < 5; ++w) cc_sound[i][w] = 64;
            cc_vib_rate[i] = 64;
            cc_vib_depth[i] = 64;
        }
        std::array<uint8_t, 5> neutral;
        neutral.fill((uint8_t)(64 >> SOUND_CC_SHIFT));
        variants.push_back(neutral);
        seen_states.push_back(neutral);
        variant_seen.push_back(0);
        tail_blocks_left = (uint64_t)(MAX_TAIL_SECONDS * (double)c.sample_rate / (double)c.block_frames);
        for (int ch = 0; ch < 16; ++ch) refresh_preset(ch, 0);
    }

    // Config::max_steal / admit_take, src/config.rs:120-131, 549-552.
    uint32_t max_steal() const {
        const uint64_t n = (uint64_t)cfg.max_voices * cfg.max_steal_percent / 100;
        return std::max<uint32_t>((uint32_t)n, 1);
    }
    uint32_t admit_take(uint32_t live, uint32_t queued) const {
        const uint32_t cap = cfg.max_voices;
        const uint32_t want = std::min(queued, cap);
        if ((uint64_t)live + want <= cap) return want;
        const uint32_t need = cfg.steal_rule == KC_STEAL_DROP_NEW
                                  ? 0
                                  : std::min(std::min(live + want - cap, live), max_steal());
        return std::min(want, cap - (live - need));
    }

    void refresh_preset(int ch, uint8_t program) {
        const uint16_t bank_num = ch == 9 ? 128 : bank_msb[ch];
        uint32_t p = 0;
        if (!bank->find_preset(bank_num, program, &p)) p = 0;
        preset[ch] = p;
    }

    static kc_spawn_cmd make_cmd(const VoiceSpawn& v, uint32_t variant, uint32_t gate_slot, uint32_t ordinal,
                                 uint32_t start_rel, uint64_t id) {
        kc_spawn_cmd c{};
        c.phase_lo = (uint32_t)v.phase;
        c.phase_hi = (uint32_t)(v.phase >> 32);
        c.step_lo = (uint32_t)v.step;
        c.step_hi = (uint32_t)(v.step >> 32);
        c.smp_base = v.smp_base;
        c.smp_len = v.smp_len;
        c.loop_start = v.loop_start;
        c.loop_end = v.loop_end;
        c.flags = v.flags;
        c.params = v.params;
        c.variant = variant;
        c.region = v.region;
        c.gate_slot = gate_slot;
        c.ordinal = ordinal;
        c.start_rel = start_rel;
        c.note_id_lo = (uint32_t)id;
        c.note_id_hi = (uint32_t)(id >> 32);
        c.gain_l = v.gain_l;
        c.gain_r = v.gain_r;
        return c;
    }

    // next_block up to backend.spawn (src/driver.rs:434-588).
    // Driver::next_block up to the backend's spawn is two halves: collect()
    // drains the block's events (gate and controller rows, candidates,
    // variants) and needs nothing from the backend; admit(live) runs
    // admission against the backend's live count and materialises the
    // admitted voices. Collecting block n + 1 while the device renders
    // block n changes nothing, since collect reads only state that admit(n)
    // has finished with.
    void prepare(uint32_t live) {
        collect();
        admit(live);
    }

    void collect() {
        const uint64_t block_frames = cfg.block_frames;
        const uint64_t block_start = block_index * block_frames;
        const uint64_t block_end = block_start + block_frames;
        gates.begin_block();
        chan.begin_block();
        variant_used = 1;
        for (uint32_t v : cur_variant) variant_used |= 1ull << v;
        spawn_buf.clear();
        notes.clear();
        note_ordinal.clear();
        cands.clear();
        deferred_now.clear();
        built.clear();
        block_first_id = next_note_id;
        spawn_variants = false;

        for (size_t i = 0; i < deferred.size();) {
            if (deferred[i].first < block_end) {
                auto [frame, cmd] = deferred[i];
                deferred[i] = deferred.back();  // Vec::swap_remove
                deferred.pop_back();
                cmd.start_rel = (uint32_t)(frame > block_start ? frame - block_start : 0);
                if (cmd.variant != 0) {
                    variant_used |= 1ull << cmd.variant;
                    spawn_variants = true;
                }
                cands.push_back(Cand{rank_key(cmd.gain_l, cmd.gain_r, cands.size()), DEFERRED,
                                     (uint32_t)deferred_now.size(), 0});
                deferred_now.push_back(cmd);
            } else {
                ++i;
            }
        }

        for (;;) {
            uint64_t tick;
            Event ev;
            if (have_pending) {
                tick = pending_tick;
                ev = pending_ev;
                have_pending = false;
            } else if (!stream->next(&tick, &ev)) {
                stream_done = true;
                break;
            }
            if (ev.type == EvType::Tempo) {
                clock.set_tempo(tick, ev.tempo);
                continue;
            }
            const double fr = clock.frame_at(tick);
            const uint64_t frame = fr < 0.0 ? 0 : sat_cast<uint64_t>(fr);
            if (frame >= block_end) {
                have_pending = true;
                pending_tick = tick;
                pending_ev = ev;
                break;
            }
            uint32_t rel = (uint32_t)(frame > block_start ? frame - block_start : 0);
            rel = std::min<uint32_t>(rel, cfg.block_frames - 1);
            handle_event(ev, rel, block_start);
        }

        if (stream_done && !end_sent) {
            for (uint8_t ch = 0; ch < 16; ++ch) gates.all_sound_off(ch, 0);
            end_sent = true;
        }
        for (auto& [i, m] : pending_variants) built.push_back({i, bank->build_variant(bcfg, m)});
        pending_variants.clear();

        gates.end_block();
        chan.end_block();
        apply_modulation();
        chan.refresh_active();
    }

    // Whether this block's admission is the same for every live count: all
    // queued layers are admitted, however full the pool, when they fit in
    // what one block may steal (and the rule may steal at all).
    bool admit_ready() const {
        const uint32_t want = std::min<uint32_t>((uint32_t)cands.size(), cfg.max_voices);
        return cfg.steal_rule != KC_STEAL_DROP_NEW ? want <= max_steal() : want == 0;
    }

    void admit(uint32_t live) {
        const uint32_t want = (uint32_t)cands.size();
        const uint32_t take = admit_take(live, want);
        last_live = live;
        last_want = want;
        last_take = take;
        if (take < want && take > 0) {
            if (cfg.admit_rule == KC_ADMIT_EVEN) {
                for (size_t i = 0; i < take; ++i) cands[i] = cands[spawn_pick(i, want, take)];
            } else {
                rank_candidates(want, take);
            }
        }
        // Summed opening amplitude of the queued and of the admitted layers,
        // after the rule has reordered (src/driver.rs:581-585).
        last_want_energy = last_take_energy = 0;
        for (size_t i = 0; i < cands.size(); ++i) {
            const uint64_t e = (cands[i].key >> 48) & 0x7FFF;
            last_want_energy += e;
            if (i < take) last_take_energy += e;
        }
        materialise(take);
        // What finish() decides the next block by, as of this block.
        done_after_admit[block_index & 1] = stream_done && deferred.empty();
    }

    // rank_candidates, src/driver.rs:701-742. select_nth_unstable is a
    // partition; the admitted *set* per stratum is unique because keys are a
    // total order, while the order inside the prefix is this partition's.
    void rank_candidates(size_t want, size_t take) {
        const size_t strata = std::min(take, ADMIT_STRATA);
        for (size_t s = 0; s < strata; ++s) {
            const size_t lo = (size_t)((uint64_t)s * want / strata);
            const size_t hi = (size_t)((uint64_t)(s + 1) * want / strata);
            const size_t olo = (size_t)((uint64_t)s * take / strata);
            const size_t ohi = (size_t)((uint64_t)(s + 1) * take / strata);
            const size_t q = ohi - olo;
            if (q == 0) continue;
            const size_t n = hi - lo;
            if (q < n)
                std::nth_element(cands.begin() + lo, cands.begin() + lo + q, cands.begin() + hi,
                                 [](const Cand& a, const Cand& b) { return a.key > b.key; });
            for (size_t j = 0; j < q; ++j) std::swap(cands[olo + j], cands[lo + j]);
        }
    }

    // materialise, src/driver.rs:751-783.
    void materialise(size_t take) {
        const size_t n = std::min(take, cands.size());
        spawn_buf.reserve(n);
        for (size_t i = 0; i < n; ++i) {
            const Cand& c = cands[i];
            if (c.note == DEFERRED) {
                spawn_buf.push_back(deferred_now[c.region]);
                continue;
            }
            const uint64_t w = notes[c.note];
            const uint8_t ch = w & 0xF, key = (w >> 4) & 0x7F, vel = (w >> 11) & 0x7F;
            const uint32_t variant = (w >> 18) & 0x3F, rel = (w >> 24) & 0xFFFF;
            VoiceSpawn v;
            if (!bank->build_layer(c.region, key, vel, bcfg, &v)) continue;
            const uint32_t start_rel = v.delay_frames == 0 ? rel : rel + v.delay_frames;
            spawn_buf.push_back(make_cmd(v, variant, (uint32_t)GateTable::slot(ch, key), note_ordinal[c.note],
                                         start_rel, block_first_id + c.id_off));
        }
    }

    // handle_event, src/driver.rs:785-967.
    void handle_event(const Event& ev, uint32_t rel, uint64_t block_start) {
        const uint8_t ch = ev.ch;
        const int c = ch & 15;
        switch (ev.type) {
            case EvType::NoteOn: {
                const uint8_t key = ev.a, vel = ev.b;
                const uint32_t ordinal = gates.note_on(ch, key, rel);
                ++notes_total;
                const uint32_t variant = cur_variant[c];
                preview_buf.clear();
                bank->preview_note_on(preset[c], key, vel, opt.max_layers, preview_buf);
                const uint32_t note = (uint32_t)notes.size();
                bool recorded = false;
                for (const PreviewLayer& p : preview_buf) {
                    const uint64_t id = next_note_id++;
                    if (p.delay_frames != 0) {
                        const uint64_t start = block_start + rel + p.delay_frames;
                        if (start >= block_start + cfg.block_frames) {
                            VoiceSpawn v;
                            if (bank->build_layer(p.region, key, vel, bcfg, &v))
                                deferred.push_back({start, make_cmd(v, variant, (uint32_t)GateTable::slot(ch, key),
                                                                    ordinal, rel, id)});
                            continue;
                        }
                    }
                    if (!recorded) {
                        notes.push_back(note_pack(ch, key, vel, variant, rel));
                        note_ordinal.push_back(ordinal);
                        recorded = true;
                    }
                    cands.push_back(Cand{rank_key(p.gain_l, p.gain_r, cands.size()), note, p.region,
                                         (uint32_t)(id - block_first_id)});
                    if (variant != 0) {
                        variant_used |= 1ull << variant;
                        spawn_variants = true;
                    }
                }
                break;
            }
            case EvType::NoteOff:
                gates.note_off(ch, ev.a, rel);
                break;
            case EvType::Cc: {
                const uint8_t num = ev.a, val = ev.b;
                switch (num) {
                    case 0: bank_msb[c] = val; break;
                    case 1: cc_mod[c] = val; lsb_mod[c] = 0; break;
                    case 33: lsb_mod[c] = val; break;
                    case 39: lsb_volume[c] = val; refresh_gain(c, rel); break;
                    case 42: lsb_pan[c] = val; refresh_gain(c, rel); break;
                    case 43: lsb_expression[c] = val; refresh_gain(c, rel); break;
                    case 32: bank_lsb[c] = val; break;
                    case 6:
                        if (rpn_sel[c] == 0) { bend_range[c] = (double)val; refresh_bend(c, rel); }
                        break;
                    case 38:
                        if (rpn_sel[c] == 0) {
                            bend_range[c] = std::trunc(bend_range[c]) + (double)val / 100.0;
                            refresh_bend(c, rel);
                        }
                        break;
                    case 96:
                        if (rpn_sel[c] == 0) { bend_range[c] = rmind(bend_range[c] + 1.0, 127.0); refresh_bend(c, rel); }
                        break;
                    case 97:
                        if (rpn_sel[c] == 0) { bend_range[c] = rmaxd(bend_range[c] - 1.0, 0.0); refresh_bend(c, rel); }
                        break;
                    case 98: case 99: rpn_sel[c] = RPN_NONE; break;
                    case 100: {
                        const uint16_t keep = rpn_sel[c] == RPN_NONE ? 0 : rpn_sel[c];
                        rpn_sel[c] = (uint16_t)((keep & 0x3F80) | val);
                        break;
                    }
                    case 101: {
                        const uint16_t keep = rpn_sel[c] == RPN_NONE ? 0 : rpn_sel[c];
                        rpn_sel[c] = (uint16_t)((keep & 0x7F) | ((uint16_t)val << 7));
                        break;
                    }
                    case 7: cc_volume[c] = val; lsb_volume[c] = 0; refresh_gain(c, rel); break;
                    case 10: cc_pan[c] = val; lsb_pan[c] = 0; refresh_gain(c, rel); break;
                    case 11: cc_expression[c] = val; lsb_expression[c] = 0; refresh_gain(c, rel); break;
                    case 64: gates.set_sustain(ch, val >= 64, rel); break;
                    case 66: gates.set_sostenuto(ch, val >= 64, rel); break;
                    case 67: cc_soft[c] = val; refresh_gain(c, rel); break;
                    case 71: set_sound_cc(ch, 0, val, rel); break;
                    case 72: set_sound_cc(ch, 1, val, rel); break;
                    case 73: set_sound_cc(ch, 2, val, rel); break;
                    case 74: set_sound_cc(ch, 3, val, rel); break;
                    case 75: set_sound_cc(ch, 4, val, rel); break;
                    case 76: cc_vib_rate[c] = val; break;
                    case 77: cc_vib_depth[c] = val; break;
                    case 92: cc_tremolo[c] = val; break;
                    case 120: gates.all_sound_off(ch, rel); break;
                    case 121: reset_controllers(ch, rel); break;
                    case 123: case 124: case 125: case 126: case 127: gates.all_notes_off(ch, rel); break;
                    default: break;
                }
                break;
            }
            case EvType::Program:
                refresh_preset(c, ev.a);
                break;
            case EvType::PitchBend:
                bend_val[c] = ev.bend;
                refresh_bend(c, rel);
                break;
            default:
                break;
        }
    }

    // set_sound_cc, src/driver.rs:982-1061.
    void set_sound_cc(uint8_t ch, int which, uint8_t val, uint32_t rel) {
        const int c = ch & 15;
        if (cc_sound[c][which] == val) return;
        cc_sound[c][which] = val;
        std::array<uint8_t, 5> want;
        for (int i = 0; i < 5; ++i) want[i] = (uint8_t)(cc_sound[c][i] >> SOUND_CC_SHIFT);
        if (std::find(seen_states.begin(), seen_states.end(), want) == seen_states.end()) seen_states.push_back(want);
        const uint32_t cap = std::clamp<uint32_t>(cfg.max_param_variants, 1, 63);
        uint32_t idx;
        auto it = std::find(variants.begin(), variants.end(), want);
        if (it != variants.end()) {
            idx = (uint32_t)(it - variants.begin());
        } else if ((uint32_t)variants.size() < cap) {
            idx = (uint32_t)variants.size();
            variants.push_back(want);
            variant_seen.push_back(0);
            build_variant_at(idx, c);
        } else {
            int64_t victim = -1;
            for (size_t i = 1; i < variants.size(); ++i)
                if (!(variant_used & (1ull << i)) && (victim < 0 || variant_seen[i] < variant_seen[victim]))
                    victim = (int64_t)i;
            if (victim >= 0) {
                variants[victim] = want;
                build_variant_at((uint32_t)victim, c);
                idx = (uint32_t)victim;
            } else {
                uint32_t best = 0, best_d = UINT32_MAX;
                for (size_t i = 0; i < variants.size(); ++i) {
                    uint32_t d = 0;
                    for (int k = 0; k < 5; ++k) d += (uint32_t)std::abs((int)variants[i][k] - (int)want[k]);
                    if (d < best_d) {
                        best_d = d;
                        best = (uint32_t)i;
                    }
                }
                idx = best;
            }
        }
        variant_clock += 1;
        variant_seen[idx] = variant_clock;
        variant_used |= 1ull << idx;
        cur_variant[c] = idx;
        chan.set_variant(ch, idx, rel);
    }

    void build_variant_at(uint32_t i, int c) {
        const ParamMod m = ParamMod::from_controllers(cc_sound[c][0], cc_sound[c][1], cc_sound[c][2], cc_sound[c][3],
                                                      cc_sound[c][4]);
        pending_variants.erase(std::remove_if(pending_variants.begin(), pending_variants.end(),
                                              [i](const auto& p) { return p.first == i; }),
                               pending_variants.end());
        pending_variants.push_back({i, m});
    }

    // reset_controllers, src/driver.rs:1078-1102.
    void reset_controllers(uint8_t ch, uint32_t rel) {
        const int c = ch & 15;
        bank_msb[c] = 0;
        bank_lsb[c] = 0;
        bend_range[c] = 2.0;
        bend_val[c] = 0;
        rpn_sel[c] = RPN_NONE;
        cc_volume[c] = (uint8_t)std::min<uint32_t>(opt.default_channel_volume, 127);
        cc_expression[c] = 127;
        cc_pan[c] = 64;
        cc_soft[c] = 0;
        cc_mod[c] = 0;
        lsb_mod[c] = lsb_volume[c] = lsb_pan[c] = lsb_expression[c] = 0;
        cc_tremolo[c] = 0;
        cc_vib_rate[c] = 64;
        cc_vib_depth[c] = 64;
        for (int w = 0; w < 5; ++w) set_sound_cc(ch, w, 64, rel);
        refresh_bend(c, rel);
        refresh_gain(c, rel);
        gates.reset_controllers(ch, rel);
    }

    // apply_modulation, src/driver.rs:1110-1141.
    void apply_modulation() {
        const size_t tiles = chan.tiles;
        const double tile_seconds = (double)cfg.gate_frames / (double)cfg.sample_rate;
        for (int c = 0; c < 16; ++c) {
            const double vib = ((double)cc_mod[c] * 128.0 + (double)lsb_mod[c]) / 16383.0 *
                               ((double)cc_vib_depth[c] / 64.0) * 50.0;
            const double trem = (double)cc_tremolo[c] / 127.0 * 0.25;
            const double rate = 5.0 * std::pow(2.0, ((double)cc_vib_rate[c] - 64.0) / 32.0);
            if (vib <= 0.0 && trem <= 0.0) {
                lfo_phase[c] = rfract(lfo_phase[c] + rate * tile_seconds * (double)tiles);
                continue;
            }
            double phase = lfo_phase[c];
            for (size_t t = 0; t < tiles; ++t) {
                const double s = std::sin(phase * 2.0 * M_PI);
                if (vib > 0.0) chan.modulate_bend((uint8_t)c, t, bend_factor(vib * s / 100.0));
                if (trem > 0.0) chan.modulate_gain((uint8_t)c, t, (float)(1.0 - trem + trem * s));
                phase = rfract(phase + rate * tile_seconds);
            }
            lfo_phase[c] = phase;
        }
    }

    // refresh_bend, src/driver.rs:1146-1149.
    void refresh_bend(int c, uint32_t rel) {
        const double semitones = ((double)bend_val[c] / 8192.0) * bend_range[c];
        chan.set_bend((uint8_t)c, bend_factor(semitones), rel);
    }

    // refresh_gain, src/driver.rs:1161-1188.
    void refresh_gain(int c, uint32_t rel) {
        auto fine = [](uint8_t msb, uint8_t lsb) {
            return lsb == 0 ? (float)msb / 127.0f : ((float)msb * 128.0f + (float)lsb) / 16383.0f;
        };
        const float v = fine(cc_volume[c], lsb_volume[c]);
        const float e = fine(cc_expression[c], lsb_expression[c]);
        const float soft = 1.0f - 0.5f * ((float)cc_soft[c] / 127.0f);
        const float amp = (v * v) * (e * e) * soft;
        const float theta = fine(cc_pan[c], lsb_pan[c]) * FRAC_PI_2_F;
        float l = 1.0f, r = 1.0f;
        if (!(cc_pan[c] == 64 && lsb_pan[c] == 0)) {
            l = std::cos(theta) * SQRT_2_F;
            r = std::sin(theta) * SQRT_2_F;
        }
        chan.set_gain((uint8_t)c, amp * l, amp * r, rel);
    }

    // The rest of next_block (src/driver.rs:619-642).
    bool finish(uint64_t active_voices) {
        advance();
        return more(active_voices);
    }
    void advance() { block_index += 1; }
    // Driver::next_block's continuation test (src/driver.rs:625-642), on the
    // state the last admitted block left.
    bool more(uint64_t active_voices) {
        if (!done_after_admit[(block_index - 1) & 1]) return true;
        if (active_voices > 0) {
            tail_blocks_left = tail_blocks_left > 0 ? tail_blocks_left - 1 : 0;
            return tail_blocks_left != 0;
        }
        return false;
    }
};

// ---- synthetic soundfonts -----------------------------------------------------

namespace {
// The seeded synthetic bank: per preset, one instrument of 128 zones, zone k
// playing sample k (root k) on key k. Generators as an SF2 instrument zone
// holds them (src/testkit.rs:83-124 builds the same records).
Sf2 synth_sf2(const kh_synth_bank_spec& s) {
    Sf2 sf;
    std::mt19937_64 rng(s.seed);
    std::uniform_real_distribution<double> u(0.0, 1.0);
    for (int k = 0; k < 128; ++k) {
        Sf2Sample smp;
        smp.rate = s.sample_rate;
        smp.root = (uint8_t)k;
        const double freq = 440.0 * std::pow(2.0, (k - 69) / 12.0);
        const std::vector<int16_t> nz = noise(s.sample_frames, s.seed * 131 + (uint64_t)k + 1);
        smp.data.resize(s.sample_frames);
        for (uint32_t i = 0; i < s.sample_frames; ++i) {
            const double ph = (double)i * freq / (double)s.sample_rate * 2.0 * M_PI;
            // noise() spans about +-8192/32767; scale it to `noise` of full scale
            const double x = std::sin(ph) * s.amplitude + (double)nz[i] / 8192.0 * s.noise;
            smp.data[i] = (int16_t)std::clamp(std::round(x * 32767.0), -32767.0, 32767.0);
        }
        const uint32_t loop = std::min(s.loop_frames, s.sample_frames);
        smp.loop_start = s.sample_frames - loop;
        smp.loop_end = s.sample_frames;
        sf.samples.push_back(std::move(smp));
    }
    // One instrument of 128 zones on the base generators. A preset with its
    // own (random) generators states them as preset-level offsets, which the
    // loader adds to the instrument's (src/sf2.rs:449-455): the flattened
    // region holds the preset's values exactly, and the file's generator
    // lists stay within the format's 16-bit indexes at 128 presets. An
    // offset that would not fit 16 bits gets its own instrument instead.
    auto instrument = [&](int16_t attack, int16_t decay, int16_t sustain, int16_t release, int16_t fc, int16_t q) {
        std::vector<Sf2Zone> inst;
        for (int k = 0; k < 128; ++k) {
            Sf2Zone z;
            z.sample = (uint16_t)k;
            z.key_lo = z.key_hi = (uint8_t)k;
            z.gens = {{54, 1}, {34, attack}, {36, decay}, {37, sustain}, {38, release}, {8, fc}, {9, q}};
            inst.push_back(std::move(z));
        }
        sf.instruments.push_back(std::move(inst));
        return (uint16_t)(sf.instruments.size() - 1);
    };
    const uint16_t base = instrument(s.attack_tc, s.decay_tc, s.sustain_cb, s.release_tc, s.filter_fc_cents,
                                     s.filter_q_cb);
    for (uint32_t p = 0; p < std::max<uint32_t>(s.presets, 1); ++p) {
        Sf2Preset pr;
        pr.program = (uint16_t)(p % 128);
        pr.bank = (uint16_t)(p / 128);
        pr.instrument = base;
        if (s.random_generators && p > 0) {
            const int16_t attack = (int16_t)std::lround(-12000.0 + u(rng) * (1200.0 * std::log2(0.05) + 12000.0));
            const int16_t decay = (int16_t)std::lround(1200.0 * std::log2(0.05 + u(rng) * 1.95));
            const int16_t sustain = (int16_t)std::lround(u(rng) * 200.0);
            const int16_t release = (int16_t)std::lround(1200.0 * std::log2(0.05 + u(rng) * 0.95));
            const int16_t fc = (int16_t)std::lround(1200.0 * std::log2((1000.0 + u(rng) * 11000.0) / 8.176));
            const int16_t q = (int16_t)std::lround(u(rng) * 120.0);
            const std::pair<uint16_t, int32_t> offs[] = {
                {34, attack - s.attack_tc}, {36, decay - s.decay_tc},     {37, sustain - s.sustain_cb},
                {38, release - s.release_tc}, {8, fc - s.filter_fc_cents}, {9, q - s.filter_q_cb}};
            bool fits = true;
            for (auto [op, d] : offs) fits = fits && d >= -32768 && d <= 32767;
            if (fits) {
                for (auto [op, d] : offs) pr.gens.push_back({op, (int16_t)d});
            } else {
                pr.instrument = instrument(attack, decay, sustain, release, fc, q);
            }
        }
        sf.presets.push_back(pr);
    }
    return sf;
}
}  // namespace

}  // namespace kh

using namespace kh;

struct kh_bank {
    Bank bank;
    BankConfig cfg;
    std::string report;  // the loader's warnings, one per line
};
struct kh_driver {
    std::unique_ptr<Driver> d;
};

extern "C" {

const char* kh_last_error(void) { return g_err.c_str(); }

void kh_options_default(kh_options* o) {
    o->master_volume = 1.0f;
    o->filter_enabled = 1;
    o->max_layers = 16;
    o->default_channel_volume = 127;
    o->resample_pool = 1;
    o->read_ahead = 1;
    o->sample_pool_budget = 2ull << 30;
}

void kh_synth_bank_spec_default(kh_synth_bank_spec* s) {
    std::memset(s, 0, sizeof(*s));
    s->presets = 1;
    s->sample_frames = 32768;
    s->sample_rate = 44100;
    s->loop_frames = 8192;
    s->amplitude = 0.5f;
    s->noise = 0.01f;
    s->attack_tc = -9172;
    s->decay_tc = -2786;
    s->sustain_cb = 60;
    s->release_tc = -2084;
    s->filter_fc_cents = 11913;
    s->filter_q_cb = 30;
    s->random_generators = 0;
    s->seed = 0x5EED;
}

namespace {
BankConfig bank_config(const kc_config* cfg, const kh_options* opt) {
    kh_options o;
    kh_options_default(&o);
    if (opt) o = *opt;
    BankConfig b;
    b.sample_rate = cfg->sample_rate;
    b.env_floor = cfg->env_floor;
    b.exp_decay = cfg->decay_curve == KC_CURVE_EXPONENTIAL;
    b.exp_release = cfg->release_curve == KC_CURVE_EXPONENTIAL;
    b.filter_enabled = o.filter_enabled != 0;
    b.master_volume = o.master_volume;
    b.resample_pool = o.resample_pool != 0;
    b.sample_pool_budget = o.sample_pool_budget;
    return b;
}
}  // namespace

kh_bank* kh_bank_open_sf2(const char* path, const kc_config* cfg, const kh_options* opt) {
    if (!path || !cfg) {
        g_err = "null argument";
        return nullptr;
    }
    auto* kb = new kh_bank();
    kb->cfg = bank_config(cfg, opt);
    if (!load_sf2_file(path, kb->cfg, &kb->bank, &g_err)) {
        delete kb;
        return nullptr;
    }
    return kb;
}

kh_bank* kh_bank_open_sfz(const char* path, const kc_config* cfg, const kh_options* opt) {
    if (!path || !cfg) {
        g_err = "null argument";
        return nullptr;
    }
    auto* kb = new kh_bank();
    kb->cfg = bank_config(cfg, opt);
    std::vector<std::string> report;
    if (!load_sfz_file(path, kb->cfg, &kb->bank, &g_err, &report)) {
        delete kb;
        return nullptr;
    }
    for (const auto& line : report) kb->report += line + "\n";
    return kb;
}

kh_bank* kh_bank_open(const char* path, const kc_config* cfg, const kh_options* opt) {
    if (!path) {
        g_err = "null argument";
        return nullptr;
    }
    // load_bank (src/lib.rs:32-48): by the file's extension
    std::string p = path;
    const size_t dot = p.rfind('.');
    const size_t slash = p.rfind('/');
    std::string ext = dot == std::string::npos || (slash != std::string::npos && dot < slash) ? "" : p.substr(dot + 1);
    for (auto& c : ext) c = (char)std::tolower((unsigned char)c);
    if (ext == "sf2" || ext == "sf3" || ext == "sfbk") return kh_bank_open_sf2(path, cfg, opt);
    if (ext == "sfz") return kh_bank_open_sfz(path, cfg, opt);
    g_err = p + ": unrecognised soundfont extension \"" + ext + "\"; expected .sf2 or .sfz";
    return nullptr;
}

const char* kh_bank_report(const kh_bank* b) { return b ? b->report.c_str() : ""; }

int kh_sfz_note_name(const char* s, int32_t* out) { return s && out && sfz_note_name(s, out) ? 0 : 1; }
size_t kh_sfz_value_end(const char* s) { return s ? sfz_value_end(s) : 0; }

int kh_sf2_write_synthetic(const kh_synth_bank_spec* spec, const char* path) {
    if (!spec || !path) {
        g_err = "null argument";
        return 1;
    }
    std::vector<uint8_t> bytes;
    if (!write_sf2(synth_sf2(*spec), &bytes, &g_err)) return 1;
    FILE* f = std::fopen(path, "wb");
    if (!f) {
        g_err = std::string("creating ") + path;
        return 1;
    }
    const bool ok = std::fwrite(bytes.data(), 1, bytes.size(), f) == bytes.size();
    if (std::fclose(f) != 0 || !ok) {
        g_err = std::string("writing ") + path;
        return 1;
    }
    return 0;
}

uint32_t kh_bank_samples(const kh_bank* b) { return (uint32_t)b->bank.samples.size(); }

int kh_bank_region_info(const kh_bank* b, uint32_t i, kh_region_info* out) {
    if (!b || !out || i >= b->bank.regions.size()) {
        g_err = "region index out of range";
        return 1;
    }
    const Region& r = b->bank.regions[i];
    *out = kh_region_info{};
    out->sample = r.sample;
    out->key_lo = r.key_lo;
    out->key_hi = r.key_hi;
    out->vel_lo = r.vel_lo;
    out->vel_hi = r.vel_hi;
    out->root_key_override = r.root_key_override;
    out->fixed_key = r.fixed_key;
    out->fixed_vel = r.fixed_vel;
    out->coarse_tune = r.coarse_tune;
    out->fine_tune = r.fine_tune;
    out->scale_tuning = r.scale_tuning;
    out->keynum_to_hold = r.keynum_to_hold;
    out->keynum_to_decay = r.keynum_to_decay;
    out->loop_mode = r.loop_mode == LoopMode::Continuous ? 1 : r.loop_mode == LoopMode::UntilRelease ? 2 : 0;
    out->exclusive_class = r.exclusive_class;
    out->attenuation_cb = r.attenuation_cb;
    out->pan = r.pan;
    out->addr_start = r.addr_start;
    out->addr_end = r.addr_end;
    out->addr_loop_start = r.addr_loop_start;
    out->addr_loop_end = r.addr_loop_end;
    out->delay = r.delay;
    out->attack = r.attack;
    out->hold = r.hold;
    out->decay = r.decay;
    out->sustain = r.sustain;
    out->release = r.release;
    out->filter_fc_cents = r.filter_fc_cents;
    out->filter_q_cb = r.filter_q_cb;
    return 0;
}

int kh_bank_sample_info(const kh_bank* b, uint32_t i, kh_sample_info* out) {
    if (!b || !out || i >= b->bank.samples.size()) {
        g_err = "sample index out of range";
        return 1;
    }
    const SampleInfo& s = b->bank.samples[i];
    out->start = s.start;
    out->len = s.len;
    out->loop_start = s.loop_start;
    out->loop_end = s.loop_end;
    out->rate = s.rate;
    out->root_key = s.root_key;
    out->correction_cents = s.correction_cents;
    out->resample_ratio = s.resample_ratio;
    return 0;
}

int kh_bank_preset_info(const kh_bank* b, uint32_t i, uint16_t* bank, uint16_t* program, uint32_t* n_regions,
                        uint32_t* regions, uint32_t cap) {
    if (!b || i >= b->bank.presets.size()) {
        g_err = "preset index out of range";
        return 1;
    }
    const Preset& p = b->bank.presets[i];
    if (bank) *bank = p.bank;
    if (program) *program = p.program;
    if (n_regions) *n_regions = (uint32_t)p.regions.size();
    if (regions)
        for (uint32_t j = 0; j < std::min<uint32_t>(cap, (uint32_t)p.regions.size()); ++j) regions[j] = p.regions[j];
    return 0;
}

kh_bank* kh_bank_synthetic(const kh_synth_bank_spec* spec, const kc_config* cfg, const kh_options* opt) {
    if (!spec || !cfg) {
        g_err = "null argument";
        return nullptr;
    }
    auto* kb = new kh_bank();
    kb->cfg = bank_config(cfg, opt);
    if (!load_sf2(synth_sf2(*spec), kb->cfg, &kb->bank, &g_err)) {
        delete kb;
        return nullptr;
    }
    return kb;
}

void kh_bank_destroy(kh_bank* b) { delete b; }

int kh_bank_pool(const kh_bank* b, const int16_t** pool, uint64_t* len) {
    *pool = b->bank.pool.data();
    *len = b->bank.pool.size();
    return 0;
}
int kh_bank_params(const kh_bank* b, const kc_region_params** params, uint32_t* len) {
    *params = b->bank.params.data();
    *len = (uint32_t)b->bank.params.size();
    return 0;
}
uint32_t kh_bank_regions(const kh_bank* b) { return (uint32_t)b->bank.regions.size(); }
uint32_t kh_bank_presets(const kh_bank* b) { return (uint32_t)b->bank.presets.size(); }
uint32_t kh_bank_max_sample_len(const kh_bank* b) { return b->bank.max_sample_len(); }
uint32_t kh_bank_pool_rate(const kh_bank* b) { return b->bank.pool_rate; }

int kh_bank_filter_inputs(const kh_bank* b, float* fc_hz, float* q_cb, uint8_t* on, uint32_t n) {
    std::vector<float> f, q;
    std::vector<uint8_t> o;
    b->bank.filter_inputs(b->cfg, ParamMod{}, f, q, o);
    if (n != f.size()) {
        g_err = "filter inputs: expected one slot per params entry";
        return 1;
    }
    std::memcpy(fc_hz, f.data(), n * 4);
    std::memcpy(q_cb, q.data(), n * 4);
    std::memcpy(on, o.data(), n);
    return 0;
}

void kh_midi_spec_default(kh_midi_spec* s) {
    std::memset(s, 0, sizeof(*s));
    s->notes = 100000;
    s->seconds = 30.0;
    s->channels = 16;
    s->key_lo = 21;
    s->key_hi = 108;
    s->vel_lo = 1;
    s->vel_hi = 127;
    s->dur_median_s = 0.150;
    s->dur_sigma = 1.0;
    s->cluster_share = 0.0;
    s->cluster_lo = 1000;
    s->cluster_hi = 50000;
    s->cc_period_ms = 0.0;
    s->program_period_s = 0.0;
    s->programs = 1;
    s->ppq = 9600;
    s->seed = 1;
}

kh_driver* kh_driver_open(const kc_config* cfg, const kh_options* opt, const kh_bank* bank, const kh_midi_spec* midi) {
    if (!cfg || !bank || !midi) {
        g_err = "null argument";
        return nullptr;
    }
    if (cfg->gate_frames == 0 || cfg->block_frames % cfg->gate_frames) {
        g_err = "gate_frames must divide block_frames";
        return nullptr;
    }
    kh_options o;
    kh_options_default(&o);
    if (opt) o = *opt;
    auto* d = new kh_driver();
    d->d = std::make_unique<Driver>(*cfg, o, bank->bank, *midi);
    return d;
}

kh_driver* kh_driver_open_smf(const kc_config* cfg, const kh_options* opt, const kh_bank* bank, const char* path) {
    if (!cfg || !bank || !path) {
        g_err = "null argument";
        return nullptr;
    }
    if (cfg->gate_frames == 0 || cfg->block_frames % cfg->gate_frames) {
        g_err = "gate_frames must divide block_frames";
        return nullptr;
    }
    std::string err;
    std::unique_ptr<SmfStream> file = SmfStream::open(path, &err);
    if (!file) {
        g_err = err;
        return nullptr;
    }
    kh_options o;
    kh_options_default(&o);
    if (opt) o = *opt;
    kh_midi_spec unused;
    kh_midi_spec_default(&unused);
    auto* d = new kh_driver();
    d->d = std::make_unique<Driver>(*cfg, o, bank->bank, unused, std::move(file));
    return d;
}

void kh_driver_destroy(kh_driver* d) { delete d; }

int kh_driver_prepare(kh_driver* h, uint32_t live, kh_block* out) {
    Driver& d = *h->d;
    d.prepare(live);
    out->gates = d.gates.rows.data();
    out->n_gates = d.gates.rows.size();
    out->chan = d.chan.rows.data();
    out->n_chan = d.chan.rows.size();
    out->bend = d.chan.bend_active;
    out->gain = d.chan.gain_active;
    out->variant = d.chan.variant_active || d.spawn_variants;
    out->cmds = d.spawn_buf.data();
    out->n_cmds = d.spawn_buf.size();
    out->n_variants = (uint32_t)d.built.size();
    out->live = d.last_live;
    out->want = d.last_want;
    out->take = d.last_take;
    out->block_index = d.block_index;
    out->notes = d.notes_total;
    out->want_energy = d.last_want_energy;
    out->take_energy = d.last_take_energy;
    return 0;
}

int kh_driver_variant(kh_driver* h, uint32_t i, uint32_t* index, const kc_region_params** data, size_t* n) {
    Driver& d = *h->d;
    if (i >= d.built.size()) {
        g_err = "variant index out of range";
        return 1;
    }
    *index = d.built[i].first;
    *data = d.built[i].second.data();
    *n = d.built[i].second.size();
    return 0;
}

int kh_driver_collect(kh_driver* h) {
    h->d->collect();
    return 0;
}

int kh_driver_admit(kh_driver* h, uint32_t live, kh_block* out) {
    Driver& d = *h->d;
    d.admit(live);
    out->gates = d.gates.rows.data();
    out->n_gates = d.gates.rows.size();
    out->chan = d.chan.rows.data();
    out->n_chan = d.chan.rows.size();
    out->bend = d.chan.bend_active;
    out->gain = d.chan.gain_active;
    out->variant = d.chan.variant_active || d.spawn_variants;
    out->cmds = d.spawn_buf.data();
    out->n_cmds = d.spawn_buf.size();
    out->n_variants = (uint32_t)d.built.size();
    out->live = d.last_live;
    out->want = d.last_want;
    out->take = d.last_take;
    out->block_index = d.block_index;
    out->notes = d.notes_total;
    out->want_energy = d.last_want_energy;
    out->take_energy = d.last_take_energy;
    return 0;
}

int kh_driver_admit_ready(const kh_driver* h) { return h->d->admit_ready() ? 1 : 0; }

int kh_driver_advance(kh_driver* h) {
    h->d->advance();
    return 0;
}

int kh_driver_more(kh_driver* h, uint64_t active_voices, int* more) {
    *more = h->d->more(active_voices) ? 1 : 0;
    return 0;
}

int kh_driver_finish(kh_driver* h, uint64_t active_voices, int* more) {
    *more = h->d->finish(active_voices) ? 1 : 0;
    return 0;
}

struct kh_gates {
    GateTable t;
};
kh_gates* kh_gates_new(uint32_t block_frames, uint32_t gate_frames) {
    if (gate_frames == 0 || block_frames % gate_frames) return nullptr;
    auto* g = new kh_gates();
    g->t.init(block_frames, gate_frames);
    return g;
}
void kh_gates_destroy(kh_gates* g) { delete g; }
void kh_gates_begin_block(kh_gates* g) { g->t.begin_block(); }
void kh_gates_end_block(kh_gates* g) { g->t.end_block(); }
uint32_t kh_gates_note_on(kh_gates* g, uint8_t ch, uint8_t key, uint32_t frame) { return g->t.note_on(ch, key, frame); }
void kh_gates_note_off(kh_gates* g, uint8_t ch, uint8_t key, uint32_t frame) { g->t.note_off(ch, key, frame); }
void kh_gates_set_sustain(kh_gates* g, uint8_t ch, int down, uint32_t frame) { g->t.set_sustain(ch, down != 0, frame); }
void kh_gates_set_sostenuto(kh_gates* g, uint8_t ch, int down, uint32_t frame) {
    g->t.set_sostenuto(ch, down != 0, frame);
}
uint32_t kh_gates_row(const kh_gates* g, uint32_t tile, uint32_t slot) {
    return g->t.rows[(size_t)tile * GATE_SLOTS + (slot % GATE_SLOTS)];
}
uint32_t kh_gates_tiles(const kh_gates* g) { return (uint32_t)g->t.tiles; }
uint64_t kh_gates_sounding(const kh_gates* g) { return g->t.sounding(); }

float kh_velocity_atten_cb(uint8_t vel, float veltrack) { return velocity_atten_cb(vel, veltrack); }
void kh_biquad_lowpass(float fc, float q_cb, float sr, float* b0, float* b1, float* a1, float* a2) {
    biquad_lowpass(fc, q_cb, sr, b0, b1, a1, a2);
}
float kh_timecents_to_secs(float tc) { return timecents_to_secs(tc); }
size_t kh_resample_i16(const int16_t* src, size_t n, double ratio, int16_t* out, size_t cap) {
    std::vector<int16_t> v(src, src + n);
    std::vector<int16_t> r = resample_i16(v, ratio);
    const size_t m = std::min(cap, r.size());
    std::memcpy(out, r.data(), m * 2);
    return r.size();
}
void kh_set_resampler(kh_resample_fn fn, void* user) { set_resample_hook(fn, user); }
int kh_sinc_table(double ratio, float* out, size_t cap) {
    const std::vector<float> t = sinc_table(ratio);
    if (!out || cap < t.size()) {
        g_err = "sinc table: need 512 * 32 floats";
        return 1;
    }
    std::memcpy(out, t.data(), t.size() * 4);
    return 0;
}
uint64_t kh_mix48(uint64_t index) { return mix48(index); }
uint64_t kh_rank_gain_q(float gain_l, float gain_r) { return rank_gain_q(gain_l, gain_r); }

}  // extern "C"

// ---- standard MIDI files ------------------------------------------------------

struct kh_smf {
    std::unique_ptr<kh::SmfStream> s;
};

namespace {
void write_varlen(std::vector<uint8_t>& buf, uint64_t v) {
    uint8_t stack[10];
    int n = 0;
    stack[n++] = (uint8_t)(v & 0x7F);
    v >>= 7;
    while (v > 0) {
        stack[n++] = (uint8_t)((v & 0x7F) | 0x80);
        v >>= 7;
    }
    for (int i = n - 1; i >= 0; --i) buf.push_back(stack[i]);
}
void put_be32(std::vector<uint8_t>& b, uint32_t v) {
    for (int s = 24; s >= 0; s -= 8) b.push_back((uint8_t)(v >> s));
}
}  // namespace

extern "C" {

kh_smf* kh_smf_open(const char* path) {
    if (!path) {
        g_err = "null path";
        return nullptr;
    }
    std::string err;
    auto s = kh::SmfStream::open(path, &err);
    if (!s) {
        g_err = err;
        return nullptr;
    }
    auto* m = new kh_smf();
    m->s = std::move(s);
    return m;
}

void kh_smf_close(kh_smf* m) { delete m; }

int kh_smf_info(const kh_smf* m, uint16_t* format, uint16_t* tracks, uint32_t* ppq, uint8_t* fps,
                uint8_t* ticks_per_frame) {
    if (!m) return 1;
    const kh::Division d = m->s->division();
    if (format) *format = m->s->format();
    if (tracks) *tracks = m->s->tracks();
    if (ppq) *ppq = d.smpte ? 0 : d.ppq;
    if (fps) *fps = d.fps;
    if (ticks_per_frame) *ticks_per_frame = d.ticks_per_frame;
    return 0;
}

int kh_smf_next(kh_smf* m, uint64_t* tick, uint32_t* type, uint8_t* ch, uint8_t* a, uint8_t* b, int16_t* bend,
                uint32_t* tempo) {
    kh::Event ev;
    uint64_t t = 0;
    if (!m || !m->s->next(&t, &ev)) return 0;
    if (tick) *tick = t;
    if (type) *type = (uint32_t)ev.type;
    if (ch) *ch = ev.ch;
    if (a) *a = ev.a;
    if (b) *b = ev.b;
    if (bend) *bend = ev.bend;
    if (tempo) *tempo = ev.tempo;
    return 1;
}

int kh_midi_write_synthetic(const kh_midi_spec* spec, const char* path, uint64_t max_events) {
    if (!spec || !path) {
        g_err = "null argument";
        return 1;
    }
    kh::SynthMidi src(*spec);
    std::vector<uint8_t> trk;
    uint64_t last = 0, t = 0, n = 0;
    kh::Event ev;
    while ((max_events == 0 || n < max_events) && src.next(&t, &ev)) {
        write_varlen(trk, t - last);
        last = t;
        const uint8_t c = ev.ch & 0x0F;
        switch (ev.type) {
            case kh::EvType::NoteOn: trk.insert(trk.end(), {(uint8_t)(0x90 | c), ev.a, ev.b}); break;
            case kh::EvType::NoteOff: trk.insert(trk.end(), {(uint8_t)(0x80 | c), ev.a, 0}); break;
            case kh::EvType::Cc: trk.insert(trk.end(), {(uint8_t)(0xB0 | c), ev.a, ev.b}); break;
            case kh::EvType::Program: trk.insert(trk.end(), {(uint8_t)(0xC0 | c), ev.a}); break;
            case kh::EvType::PitchBend: {
                const uint16_t raw = (uint16_t)(ev.bend + 8192);
                trk.insert(trk.end(), {(uint8_t)(0xE0 | c), (uint8_t)(raw & 0x7F), (uint8_t)((raw >> 7) & 0x7F)});
                break;
            }
            case kh::EvType::Tempo:
                trk.insert(trk.end(), {0xFF, 0x51, 0x03, (uint8_t)(ev.tempo >> 16), (uint8_t)(ev.tempo >> 8),
                                       (uint8_t)ev.tempo});
                break;
            default:
                trk.insert(trk.end(), {0xFF, 0x01, 0x00});  // an empty text event
                break;
        }
        ++n;
    }
    write_varlen(trk, 0);
    trk.insert(trk.end(), {0xFF, 0x2F, 0x00});
    std::vector<uint8_t> out = {'M', 'T', 'h', 'd', 0, 0, 0, 6, 0, 1, 0, 1};
    const uint16_t ppq = (uint16_t)std::min<uint32_t>(spec->ppq ? spec->ppq : 9600, 0x7FFF);
    out.push_back((uint8_t)(ppq >> 8));
    out.push_back((uint8_t)ppq);
    out.insert(out.end(), {'M', 'T', 'r', 'k'});
    put_be32(out, (uint32_t)trk.size());
    out.insert(out.end(), trk.begin(), trk.end());
    std::FILE* f = std::fopen(path, "wb");
    if (!f) {
        g_err = std::string("cannot create ") + path;
        return 1;
    }
    const bool ok = std::fwrite(out.data(), 1, out.size(), f) == out.size();
    return std::fclose(f) == 0 && ok ? 0 : 1;
}

}  // extern "C"
