// common.cuh -- device-side layout shared by every kernel of the backend.
//
// The voice pool is structure-of-arrays in HBM: field f of voice i is the u32
// at pool[f * cap + i]. The field numbering is the reference's
// (shaders/common.wgsl:15-43) so the pool reads back in the same order the CPU
// restatement writes it; `cap` is padded to a multiple of 32 so every field
// row starts 128-byte aligned and a warp's 32 voices are one coalesced line.
#pragma once

#include <cstdint>

#include "../../include/kestrel_cuda.h"

namespace kc {

enum Field : uint32_t {
    F_PHASE_LO = 0,
    F_PHASE_HI = 1,
    F_STEP_LO = 2,
    F_STEP_HI = 3,
    F_SMP_BASE = 4,
    F_SMP_LEN = 5,
    F_LOOP_START = 6,
    F_LOOP_END = 7,
    F_FLAGS = 8,
    F_ENV_STAGE = 9,
    F_ENV_LEVEL = 10,
    F_GAIN_L = 11,
    F_GAIN_R = 12,
    F_FILT_Z1 = 13,
    F_FILT_Z2 = 14,
    F_PARAMS = 15,
    F_REGION = 16,
    F_GATE_SLOT = 17,
    F_ORDINAL = 18,
    F_START_REL = 19,
    F_NOTE_LO = 20,
    F_NOTE_HI = 21,
    F_BORN_VARIANT = 22,
    F_STOP_REL = 23,
    VOICE_FIELDS = 24,
};

constexpr uint32_t ENV_ATTACK = KC_ENV_ATTACK;
constexpr uint32_t ENV_DECAY = KC_ENV_DECAY;
constexpr uint32_t ENV_SUSTAIN = KC_ENV_SUSTAIN;
constexpr uint32_t ENV_RELEASE = KC_ENV_RELEASE;
constexpr uint32_t ENV_DEAD = KC_ENV_DEAD;

// Frames reduced per mix tile: 16 frames x 2 channels = 32 lanes' worth of
// output slots, so one warp's transpose-reduce gives each lane one slot.
constexpr uint32_t MIX_TILE = 16;
constexpr uint32_t SEL_ROUNDS = 8;  // 64-bit key, 8-bit digits

// Error bits a kernel may raise in DevState::error (never a trap).
constexpr uint32_t ERR_PARAMS_RANGE = 1u << 0;
constexpr uint32_t ERR_SELECT = 1u << 1;
constexpr uint32_t ERR_COMPACT = 1u << 2;
constexpr uint32_t ERR_SLOT_RANGE = 1u << 3;

// Per-block control words, written by the host (or by a staging kernel for the
// device-resident form) before the block's kernels run.
struct BlockCtl {
    uint32_t want;         // spawn commands queued for this block
    uint32_t chan_active;  // bit 0 bend, bit 1 gain, bit 2 variant
    uint32_t pad[2];
};

// Device-resident state. The live count never leaves the device between
// blocks, so a whole block is a fixed sequence of launches with no host
// round trip (the reference's S_* slots, shaders/common.wgsl:70-83).
struct DevState {
    uint32_t live;         // voices in the current pool
    uint32_t live_old;     // live before this block's spawn (steal candidates)
    uint32_t need;         // voices to steal this block
    uint32_t take;         // commands admitted this block
    uint32_t live_render;  // live_old + take: what the render pass covers
    uint32_t live_new;     // survivors after compaction
    uint32_t sel_k;        // radix select: rank still to find inside the prefix
    uint32_t error;        // ERR_* bits
    uint64_t sel_prefix;   // radix select: digits pinned so far
    uint64_t stolen;       // cumulative
    uint64_t dropped;      // cumulative
    uint32_t peak_bits;    // max |out| of the block, as f32 bits
    uint32_t active_warps; // render warps that own at least one voice
    uint32_t hot_tiles;    // warp-tiles the render ran on a hot path (unit, integral or fractional step)
    uint32_t all_tiles;    // warp-tiles the render ran
    uint32_t pad[2];
};

// 64-bit step scaled by an 8.24 factor, truncating, saturating
// (Fixed::scale, src/fixed.rs:83-90; the device form of shaders/common.wgsl:198-216).
__device__ __forceinline__ uint64_t scale_step(uint64_t v, uint32_t factor) {
    const uint64_t lo = v * (uint64_t)factor;       // product bits 0..63
    const uint64_t hi = __umul64hi(v, (uint64_t)factor);  // bits 64..95
    if (hi >> 24) return ~0ull;
    return (hi << 40) | (lo >> 24);
}

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

}  // namespace kc
