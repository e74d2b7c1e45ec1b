// voice.h -- the host tables of src/voice.rs: the note-off gate table, the
// per-channel controller table, and the admission ranking keys.
#pragma once

#include <cstdint>
#include <cstring>
#include <vector>

#include "rust.h"

namespace kh {

constexpr size_t GATE_SLOTS = 2048;
constexpr size_t BEND_CHANNELS = 16, CHAN_FIELDS = 4;
constexpr size_t CHAN_BEND = 0, CHAN_GAIN_L = 1, CHAN_GAIN_R = 2, CHAN_VARIANT = 3;
constexpr uint32_t BEND_ONE = 1u << 24;

inline uint32_t f2b(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}
inline float b2f(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

// spawn_pick, src/voice.rs:71-75.
inline size_t spawn_pick(size_t i, size_t want, size_t take) {
    return (size_t)((uint64_t)i * (uint64_t)want / (uint64_t)take);
}

// mix48, src/voice.rs:167-177: an avalanche bijection on 48 bits.
inline uint64_t mix48(uint64_t index) {
    constexpr uint64_t M = 0x0000FFFFFFFFFFFFull;
    uint64_t z = index & M;
    z = (z ^ (z >> 24)) & M;
    z = (z * 0x9E3779B97F4Bull) & M;
    z = (z ^ (z >> 23)) & M;
    z = (z * 0xBF58476D1CE5ull) & M;
    z = (z ^ (z >> 25)) & M;
    return z;
}

// rank_gain_q, src/voice.rs:202-210.
inline uint64_t rank_gain_q(float gain_l, float gain_r) {
    const float g = std::fabs(gain_l) + std::fabs(gain_r);
    if (std::isnan(g) || g <= 0.0f) return 0;
    return (uint64_t)((f2b(g) >> 16) & 0x7FFF);
}

// GateTable, src/voice.rs:212-452.
struct GateTable {
    std::vector<uint32_t> rows;
    size_t tiles = 0;
    std::vector<uint32_t> on_count, off_count, pending_off, sost_held;
    uint16_t sustain = 0, sostenuto = 0;
    size_t cursor = 0;
    uint32_t tile_frames = 32;

    void init(uint32_t block_frames, uint32_t gate_frames) {
        tiles = block_frames / gate_frames;
        rows.assign(tiles * GATE_SLOTS, 0);
        on_count.assign(GATE_SLOTS, 0);
        off_count.assign(GATE_SLOTS, 0);
        pending_off.assign(GATE_SLOTS, 0);
        sost_held.assign(GATE_SLOTS, 0);
        tile_frames = gate_frames;
    }
    static size_t slot(uint8_t ch, uint8_t key) { return (size_t)(ch & 15) * 128 + (key & 127); }
    void begin_block() { cursor = 0; }
    void advance_to(uint32_t frame) {
        const size_t tile = frame / tile_frames;
        while (cursor <= tile && cursor < tiles) {
            std::memcpy(&rows[cursor * GATE_SLOTS], off_count.data(), GATE_SLOTS * 4);
            ++cursor;
        }
    }
    bool sustained(uint8_t ch) const { return sustain & (1u << (ch & 15)); }
    uint32_t note_on(uint8_t ch, uint8_t key, uint32_t frame) {
        advance_to(frame);
        const size_t s = slot(ch, key);
        on_count[s] += 1;
        return on_count[s];
    }
    void note_off(uint8_t ch, uint8_t key, uint32_t frame) {
        advance_to(frame);
        const size_t s = slot(ch, key);
        if ((sostenuto & (1u << (ch & 15))) && sost_held[s] > 0) {
            if (off_count[s] + pending_off[s] != on_count[s]) {
                pending_off[s] += 1;
                sost_held[s] -= 1;
            }
            return;
        }
        if (sustained(ch)) {
            if (off_count[s] + pending_off[s] != on_count[s]) pending_off[s] += 1;
        } else if (off_count[s] != on_count[s]) {
            off_count[s] += 1;
        }
    }
    void flush_pending(uint8_t ch) {
        const size_t base = (size_t)(ch & 15) * 128;
        for (size_t k = 0; k < 128; ++k) {
            const size_t s = base + k;
            if (pending_off[s] != 0) {
                off_count[s] += pending_off[s];
                pending_off[s] = 0;
            }
        }
    }
    void set_sustain(uint8_t ch, bool down, uint32_t frame) {
        if (down == sustained(ch)) return;
        advance_to(frame);
        const uint16_t bit = (uint16_t)(1u << (ch & 15));
        if (down) {
            sustain |= bit;
            return;
        }
        sustain &= (uint16_t)~bit;
        if (sostenuto & bit) return;
        flush_pending(ch);
    }
    void set_sostenuto(uint8_t ch, bool down, uint32_t frame) {
        const uint16_t bit = (uint16_t)(1u << (ch & 15));
        if (down == ((sostenuto & bit) != 0)) return;
        advance_to(frame);
        const size_t base = (size_t)(ch & 15) * 128;
        if (down) {
            sostenuto |= bit;
            for (size_t k = 0; k < 128; ++k)
                sost_held[base + k] = on_count[base + k] - off_count[base + k] - pending_off[base + k];
            return;
        }
        sostenuto &= (uint16_t)~bit;
        for (size_t k = 0; k < 128; ++k) sost_held[base + k] = 0;
        if (sustained(ch)) return;
        flush_pending(ch);
    }
    void all_notes_off(uint8_t ch, uint32_t frame) {
        advance_to(frame);
        const size_t base = (size_t)(ch & 15) * 128;
        if (sustained(ch)) {
            for (size_t k = 0; k < 128; ++k) pending_off[base + k] = on_count[base + k] - off_count[base + k];
            return;
        }
        for (size_t k = 0; k < 128; ++k) off_count[base + k] = on_count[base + k];
    }
    void all_sound_off(uint8_t ch, uint32_t frame) {
        advance_to(frame);
        const size_t base = (size_t)(ch & 15) * 128;
        for (size_t k = 0; k < 128; ++k) {
            off_count[base + k] = on_count[base + k];
            pending_off[base + k] = 0;
            sost_held[base + k] = 0;
        }
    }
    void reset_controllers(uint8_t ch, uint32_t frame) {
        set_sostenuto(ch, false, frame);
        set_sustain(ch, false, frame);
    }
    void end_block() {
        while (cursor < tiles) {
            std::memcpy(&rows[cursor * GATE_SLOTS], off_count.data(), GATE_SLOTS * 4);
            ++cursor;
        }
    }
    uint64_t sounding() const {
        uint64_t n = 0;
        for (size_t s = 0; s < GATE_SLOTS; ++s) n += (uint32_t)(on_count[s] - off_count[s]);
        return n;
    }
};

// ChannelTable, src/voice.rs:465-658.
struct ChannelTable {
    std::vector<uint32_t> rows;
    size_t tiles = 0;
    uint32_t now[BEND_CHANNELS * CHAN_FIELDS];
    size_t cursor = 0;
    uint32_t tile_frames = 32;
    bool bend_active = false, gain_active = false, variant_active = false;

    void init(uint32_t block_frames, uint32_t gate_frames) {
        tiles = block_frames / gate_frames;
        tile_frames = gate_frames;
        for (size_t c = 0; c < BEND_CHANNELS; ++c) {
            now[c * CHAN_FIELDS + CHAN_BEND] = BEND_ONE;
            now[c * CHAN_FIELDS + CHAN_GAIN_L] = f2b(1.0f);
            now[c * CHAN_FIELDS + CHAN_GAIN_R] = f2b(1.0f);
            now[c * CHAN_FIELDS + CHAN_VARIANT] = 0;
        }
        rows.assign(tiles * BEND_CHANNELS * CHAN_FIELDS, 0);
        for (size_t t = 0; t < tiles; ++t) std::memcpy(&rows[t * 64], now, sizeof(now));
        cursor = 0;
    }
    void begin_block() { cursor = 0; }
    void advance_to(uint32_t frame) {
        const size_t tile = frame / tile_frames;
        while (cursor <= tile && cursor < tiles) {
            std::memcpy(&rows[cursor * 64], now, sizeof(now));
            ++cursor;
        }
    }
    void set_bend(uint8_t ch, uint32_t factor, uint32_t frame) {
        const size_t i = (size_t)(ch & 15) * CHAN_FIELDS + CHAN_BEND;
        if (now[i] == factor) return;
        advance_to(frame);
        now[i] = factor;
    }
    void set_gain(uint8_t ch, float l, float r, uint32_t frame) {
        const size_t base = (size_t)(ch & 15) * CHAN_FIELDS;
        const uint32_t lb = f2b(l), rb = f2b(r);
        if (now[base + CHAN_GAIN_L] == lb && now[base + CHAN_GAIN_R] == rb) return;
        advance_to(frame);
        now[base + CHAN_GAIN_L] = lb;
        now[base + CHAN_GAIN_R] = rb;
    }
    void set_variant(uint8_t ch, uint32_t variant, uint32_t frame) {
        const size_t i = (size_t)(ch & 15) * CHAN_FIELDS + CHAN_VARIANT;
        if (now[i] == variant) return;
        advance_to(frame);
        now[i] = variant;
    }
    void end_block() {
        while (cursor < tiles) {
            std::memcpy(&rows[cursor * 64], now, sizeof(now));
            ++cursor;
        }
    }
    void modulate_bend(uint8_t ch, size_t tile, uint32_t factor) {
        const size_t i = (tile * BEND_CHANNELS + (ch & 15)) * CHAN_FIELDS + CHAN_BEND;
        const uint32_t scaled = (uint32_t)(((uint64_t)rows[i] * factor) >> 24);
        rows[i] = scaled > 1 ? scaled : 1;
    }
    void modulate_gain(uint8_t ch, size_t tile, float factor) {
        const size_t base = (tile * BEND_CHANNELS + (ch & 15)) * CHAN_FIELDS;
        for (size_t f : {CHAN_GAIN_L, CHAN_GAIN_R}) rows[base + f] = f2b(b2f(rows[base + f]) * factor);
    }
    void refresh_active() {
        const uint32_t one = f2b(1.0f);
        bend_active = gain_active = variant_active = false;
        for (size_t e = 0; e + CHAN_FIELDS <= rows.size(); e += CHAN_FIELDS) {
            if (rows[e + CHAN_BEND] != BEND_ONE) bend_active = true;
            if (rows[e + CHAN_GAIN_L] != one || rows[e + CHAN_GAIN_R] != one) gain_active = true;
            if (rows[e + CHAN_VARIANT] != 0) variant_active = true;
        }
    }
};

}  // namespace kh
