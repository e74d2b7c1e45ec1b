// pool_ops.cuh -- the per-voice pool passes around the render: admission
// arithmetic, steal selection, spawn, stable compaction and the pool sort.
//
// Every pass reads its counts from DevState, so one block is a fixed launch
// sequence (capturable as one CUDA graph) with no host round trip. Passes that
// have nothing to do this block return at once.
#pragma once

#include <cstdint>

#include "common.cuh"

namespace kc {

struct PoolArgs {
    uint32_t* pool;        // current pool
    uint32_t* pool_out;    // the other buffer (compaction target)
    uint32_t cap;
    DevState* st;
    const BlockCtl* ctl;
    uint32_t max_voices;
    uint32_t max_steal;
    uint32_t steal_rule;
    uint32_t admit_rule;
    uint32_t steal_span;
    uint32_t render_warps; // total warps of the render grid
    uint32_t voices_per_lane;
};

// ---- admission ---------------------------------------------------------------
// The spawn arithmetic of CpuSynth::spawn (src/cpu.rs:330-390), on the device
// so the live count never has to come back to the host between blocks.
__device__ __forceinline__ void admit_state(PoolArgs a, BlockCtl* ctl, uint32_t want32, uint32_t chan_active) {
    ctl->want = want32;
    ctl->chan_active = chan_active;
    DevState* st = a.st;
    const uint64_t cap = a.max_voices;
    const uint64_t live = st->live;
    const uint64_t want = want32;
    uint64_t need = 0, take = want;
    if (live + want > cap) {
        if (a.steal_rule == KC_STEAL_DROP_NEW) {
            take = want < (cap > live ? cap - live : 0) ? want : (cap > live ? cap - live : 0);
        } else {
            need = live + want - cap;
            if (need > live) need = live;
            if (need > a.max_steal) need = a.max_steal;
            const uint64_t room = cap - (live - need);
            take = want < room ? want : room;
        }
    }
    st->live_old = (uint32_t)live;
    st->need = (uint32_t)need;
    st->take = (uint32_t)take;
    st->live_render = (uint32_t)(live + take);
    st->stolen += need;
    st->dropped += want - take;
    st->sel_prefix = 0;
    st->sel_k = (uint32_t)need;
    st->peak_bits = 0;
    st->hot_tiles = 0;
    st->all_tiles = 0;
    // Must match k_render's batching: 32 * voices-per-lane voices per warp.
    const uint64_t n = live + take;
    const uint32_t per = 32u * a.voices_per_lane;
    const uint32_t nb = (uint32_t)((n + per - 1u) / per);
    st->active_warps = nb < a.render_warps ? nb : a.render_warps;
}

// ---- steal selection --------------------------------------------------------
// The k = need smallest steal keys among the pre-spawn voices, by an MSB-first
// radix select: eight rounds, each a 256-bin histogram of one key byte among
// the keys that match the bytes pinned so far (shaders/select.wgsl:1-112 is
// the reference's form of the same algorithm). Keys are a total order
// (src/cpu.rs:345-350), so "key <= k-th key" names exactly the victim set
// select_nth_unstable picks on the CPU.

// CpuSynth::steal_key (src/cpu.rs:212-221).
__device__ __forceinline__ uint64_t steal_key(const uint32_t* pool, uint32_t cap, uint32_t i,
                                              uint32_t rule) {
    const uint64_t id = ((uint64_t)pool[F_NOTE_HI * cap + i] << 32) | pool[F_NOTE_LO * cap + i];
    if (rule != KC_STEAL_QUIETEST) return id;
    float level = __uint_as_float(pool[F_ENV_LEVEL * cap + i]);
    // clamp(0, 1) then `as u32`: NaN maps to 0 on both sides.
    level = fminf(fmaxf(level, 0.0f), 1.0f);
    const uint64_t q = (uint64_t)__float2uint_rz(__fmul_rn(level, 65535.0f));
    return (q << 48) | (id & 0x0000FFFFFFFFFFFFull);
}

__device__ __forceinline__ void select_hist_body(PoolArgs a, uint32_t* sel_hist, uint32_t round, uint32_t cta,
                                                 uint32_t ctas) {
    __shared__ uint32_t h[256];
    const DevState* st = a.st;
    if (st->need == 0) return;
    h[threadIdx.x] = 0u;
    __syncthreads();
    const uint32_t n = st->live_old;
    const uint32_t b = 7u - round;              // byte index, MSB first
    const uint64_t prefix = st->sel_prefix;
    const uint32_t hs = 8u * (b + 1u);          // bits above this byte
    for (uint32_t i = cta * blockDim.x + threadIdx.x; i < n; i += ctas * blockDim.x) {
        const uint64_t k = steal_key(a.pool, a.cap, i, a.steal_rule);
        if (hs >= 64u || (k >> hs) == (prefix >> hs)) atomicAdd(&h[(uint32_t)(k >> (8u * b)) & 255u], 1u);
    }
    __syncthreads();
    const uint32_t c = h[threadIdx.x];
    if (c) atomicAdd(&sel_hist[round * 256u + threadIdx.x], c);
}

// Pin one byte: the bin where the running count reaches k. One CTA of 256.
__device__ __forceinline__ void select_refine_body(PoolArgs a, const uint32_t* sel_hist, uint32_t round) {
    __shared__ uint32_t scan[256];
    DevState* st = a.st;
    if (st->need == 0) return;
    const uint32_t t = threadIdx.x;
    const uint32_t k = st->sel_k;
    const uint32_t hv = sel_hist[round * 256u + t];
    scan[t] = hv;
    __syncthreads();
    for (uint32_t o = 1; o < 256u; o <<= 1) {
        const uint32_t x = t >= o ? scan[t - o] : 0u;
        __syncthreads();
        scan[t] += x;
        __syncthreads();
    }
    const uint32_t incl = scan[t];
    const uint32_t excl = incl - hv;
    // Exactly one bin satisfies excl < k <= incl when 1 <= k <= total.
    if (excl < k && k <= incl) {
        const uint32_t b = 7u - round;
        st->sel_prefix |= (uint64_t)t << (8u * b);
        st->sel_k = k - excl;
    }
    if (t == 255u && incl < k) atomicOr(&st->error, ERR_SELECT);
}

// Schedule each victim's fade (src/cpu.rs:360-371; shaders/compact.wgsl:
// 148-179): stop_rel = (note id low word) % span + 1. Only the pre-spawn
// voices are candidates.
__device__ __forceinline__ void mark_stolen_body(PoolArgs a, uint32_t cta, uint32_t ctas) {
    const DevState* st = a.st;
    if (st->need == 0) return;
    const uint32_t n = st->live_old;
    const uint64_t thresh = st->sel_prefix;
    for (uint32_t i = cta * blockDim.x + threadIdx.x; i < n; i += ctas * blockDim.x) {
        if (steal_key(a.pool, a.cap, i, a.steal_rule) <= thresh) {
            const uint32_t lo = a.pool[F_NOTE_LO * a.cap + i];
            a.pool[F_STOP_REL * a.cap + i] = lo % a.steal_span + 1u;
        }
    }
}

// ---- spawn --------------------------------------------------------------------
// Append the admitted commands at slots live_old.. (Pool::push, src/cpu.rs:
// 59-82). The i-th admitted command is cmds[i] under AdmitRule::Loudest and
// cmds[spawn_pick(i, want, take)] under AdmitRule::Even (src/cpu.rs:200-206,
// src/voice.rs:71-75). One warp handles 32 commands: it stages their 76-byte
// records through shared memory so both the read of the command array and the
// 24 field rows of the pool are written with full coalescing.
__device__ __forceinline__ void spawn_body(PoolArgs a, const kc_spawn_cmd* __restrict__ cmds, uint32_t cta,
                                           uint32_t ctas) {
    __shared__ uint32_t stage[8][32 * 19 + 1];
    const DevState* st = a.st;
    const uint32_t take = st->take;
    if (take == 0) return;
    const uint32_t want = a.ctl->want;
    const uint32_t base = st->live_old;
    const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
    const uint32_t gw = cta * 8u + w, tw = ctas * 8u;
    uint32_t* s = stage[w];
    for (uint32_t g = gw; g * 32u < take; g += tw) {
        const uint32_t i0 = g * 32u;
        const uint32_t cnt = take - i0 < 32u ? take - i0 : 32u;
        if (a.admit_rule == KC_ADMIT_LOUDEST) {
            // Contiguous records: copy 19 * cnt words cooperatively.
            const uint32_t* src = reinterpret_cast<const uint32_t*>(cmds + i0);
            for (uint32_t k = lane; k < 19u * cnt; k += 32u) s[k] = __ldg(src + k);
        } else {
            for (uint32_t r = 0; r < cnt; ++r) {
                const uint64_t pick = (uint64_t)(i0 + r) * want / take;
                const uint32_t* src = reinterpret_cast<const uint32_t*>(cmds + pick);
                if (lane < 19u) s[r * 19u + lane] = __ldg(src + lane);
            }
        }
        __syncwarp();
        if (lane < cnt) {
            const uint32_t* c = s + lane * 19u;
            uint32_t* P = a.pool + base + i0 + lane;
            const uint32_t cap = a.cap;
            P[F_PHASE_LO * cap] = c[0];
            P[F_PHASE_HI * cap] = c[1];
            P[F_STEP_LO * cap] = c[2];
            P[F_STEP_HI * cap] = c[3];
            P[F_SMP_BASE * cap] = c[4];
            P[F_SMP_LEN * cap] = c[5];
            P[F_LOOP_START * cap] = c[6];
            P[F_LOOP_END * cap] = c[7];
            P[F_FLAGS * cap] = c[8];
            P[F_ENV_STAGE * cap] = ENV_ATTACK;
            P[F_ENV_LEVEL * cap] = 0u;
            P[F_GAIN_L * cap] = c[17];
            P[F_GAIN_R * cap] = c[18];
            P[F_FILT_Z1 * cap] = 0u;
            P[F_FILT_Z2 * cap] = 0u;
            P[F_PARAMS * cap] = c[9];
            P[F_REGION * cap] = c[11];
            P[F_GATE_SLOT * cap] = c[12];
            P[F_ORDINAL * cap] = c[13];
            P[F_START_REL * cap] = c[14];
            P[F_NOTE_LO * cap] = c[15];
            P[F_NOTE_HI * cap] = c[16];
            P[F_BORN_VARIANT * cap] = c[10] + 1u;
            P[F_STOP_REL * cap] = 0u;
        }
        __syncwarp();
    }
}

// ---- compaction ---------------------------------------------------------------
// Stable, order-preserving (Pool::swap_remove_compact, src/cpu.rs:84-117), as
// reduce-then-scan: each CTA owns a contiguous chunk; count, scan the counts,
// then each CTA scatters its survivors in order. No inter-CTA waiting.

__device__ __forceinline__ uint32_t compact_chunk(uint32_t n, uint32_t nblocks) {
    const uint32_t c = (n + nblocks - 1u) / nblocks;
    return (c + 255u) & ~255u;
}

__device__ __forceinline__ void compact_count_body(PoolArgs a, uint32_t* counts, uint32_t cta, uint32_t ctas) {
    __shared__ uint32_t wsum[8];
    const uint32_t n = a.st->live_render;
    const uint32_t chunk = compact_chunk(n, ctas);
    const uint32_t lo = cta * chunk;
    const uint32_t hi = min(n, lo + chunk);
    uint32_t c = 0;
    for (uint32_t i = lo + threadIdx.x; i < hi; i += 256u) c += a.pool[F_ENV_STAGE * a.cap + i] != ENV_DEAD;
    for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
    if (lane_id() == 0) wsum[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int k = 0; k < 8; ++k) t += wsum[k];
        counts[cta] = t;
    }
}

// Exclusive scan of the per-CTA counts (any count of CTAs), one CTA of 1024.
__device__ __forceinline__ void scan_counts_body(uint32_t* counts, uint32_t m, uint32_t* total) {
    __shared__ uint32_t wsum[32];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
    for (uint32_t base = 0; base < m; base += 1024u) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t v = i < m ? counts[i] : 0u;
        uint32_t x = v;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
            if (lane >= (uint32_t)o) x += y;
        }
        if (lane == 31) wsum[w] = x;
        __syncthreads();
        if (w == 0) {
            uint32_t z = wsum[lane];
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, z, o);
                if (lane >= (uint32_t)o) z += y;
            }
            wsum[lane] = z;
        }
        __syncthreads();
        const uint32_t incl = x + (w ? wsum[w - 1] : 0u) + carry;
        if (i < m) counts[i] = incl - v;
        __syncthreads();
        if (threadIdx.x == 1023) carry = incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

// The two pool buffers never overlap, so every field is loaded before any is
// stored: 21 loads in flight per thread instead of a load-store chain the
// compiler would have to keep in order for possibly aliasing pointers.
__device__ __forceinline__ void copy_voice(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst, uint32_t cap,
                                           uint32_t from, uint32_t to) {
    uint32_t w[VOICE_FIELDS];
#pragma unroll
    for (uint32_t f = 0; f < VOICE_FIELDS; ++f) {
        // Start offset, born-under variant and stop frame apply only to the
        // block a voice was born or stolen in (shaders/compact.wgsl:134-138).
        const bool cleared = f == F_START_REL || f == F_BORN_VARIANT || f == F_STOP_REL;
        w[f] = cleared ? 0u : __ldg(src + (size_t)f * cap + from);
    }
#pragma unroll
    for (uint32_t f = 0; f < VOICE_FIELDS; ++f) dst[(size_t)f * cap + to] = w[f];
}

__device__ __forceinline__ void compact_scatter_body(PoolArgs a, const uint32_t* offsets, uint32_t cta,
                                                     uint32_t ctas) {
    __shared__ uint32_t wsum[8];
    const uint32_t n = a.st->live_render;
    const uint32_t chunk = compact_chunk(n, ctas);
    const uint32_t lo = cta * chunk;
    const uint32_t hi = min(n, lo + chunk);
    const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
    uint32_t run = offsets[cta];
    for (uint32_t t0 = lo; t0 < hi; t0 += 256u) {
        const uint32_t i = t0 + threadIdx.x;
        const bool alive = i < hi && a.pool[F_ENV_STAGE * a.cap + i] != ENV_DEAD;
        const uint32_t m = __ballot_sync(0xFFFFFFFFu, alive);
        if (lane == 0) wsum[w] = __popc(m);
        __syncthreads();
        uint32_t before = 0, tot = 0;
        for (uint32_t k = 0; k < 8; ++k) {
            before += k < w ? wsum[k] : 0u;
            tot += wsum[k];
        }
        if (alive) {
            const uint32_t dst = run + before + __popc(m & ((1u << lane) - 1u));
            copy_voice(a.pool, a.pool_out, a.cap, i, dst);
        }
        run += tot;
        __syncthreads();
    }
}

__device__ __forceinline__ void commit_body(DevState* st, const uint32_t* total) {
    st->live_new = *total;
    st->live = *total;
}

// ---- pool sort ------------------------------------------------------------------
// Performance mode (Config::sort_voices, src/config.rs:243-247): survivors are
// reordered by (region, envelope stage, coarse phase) so a warp's voices share
// sample data and branch the same way (src/gpu/mod.rs:59-106, shaders/
// sort.wgsl:1-23). A stable LSD radix sort with 8-bit digits: per pass, count
// per (digit, CTA chunk), scan digit-major, then each CTA ranks its chunk in
// order (warp match + per-warp digit counts) and scatters. Dead voices carry
// the region one past the last, so they sort to the end and the gather stops
// before them: compaction and reordering are one copy of the pool.

// The phase field is the one the voice is predicted to reach halfway through
// the next block, phase + rate * half, where rate is the base step times the
// channel's bend at the last gate tile of this block (when bend rows are on),
// wrapped into the loop of a looping voice and clamped to the field for the
// rest. Voices at one rate keep the reference's order (shifted by the same
// amount); voices at different rates -- bends, detunes, transposed notes --
// drift apart in both directions from the middle of the block instead of all
// from its start, which halves the average spread of a warp's taps. The sort
// only orders the pool for the render's locality: the live set and every
// voice's state are the same under any key.
struct SortLayout {
    uint32_t bits, region_shift, stage_shift, phase_shift, phase_mask, dead_region;
    uint32_t half;               // frames to the middle of the next block (0: the current phase)
    const uint32_t* chan;        // this block's channel rows while bend rows are on, else null
    uint32_t last_tile;          // the row of `chan` the prediction reads
};

__device__ __forceinline__ uint32_t predicted_phase(const uint32_t* pool, uint32_t cap, uint32_t i,
                                                    const SortLayout& L) {
    const uint32_t ph = pool[F_PHASE_HI * cap + i];
    if (L.half == 0) return ph;
    const uint64_t step = ((uint64_t)pool[F_STEP_HI * cap + i] << 32) | pool[F_STEP_LO * cap + i];
    // Frames in 16.16, at most 2^20 (past any sample), so the bend product
    // below stays inside 64 bits.
    uint64_t adv = (step >> 16) * L.half;
    if (adv > (1ull << 36)) adv = 1ull << 36;
    if (L.chan) {
        const uint32_t ch = (pool[F_GATE_SLOT * cap + i] >> 7) & 15u;
        const uint32_t bend = L.chan[(L.last_tile * KC_BEND_CHANNELS + ch) * KC_CHAN_FIELDS];  // 8.24
        adv = (adv >> 8) * bend >> 16;  // still 16.16 (the shifts keep the product in 64 bits)
    }
    uint64_t p = (uint64_t)ph + (adv >> 16);
    const uint32_t ls = pool[F_LOOP_START * cap + i], le = pool[F_LOOP_END * cap + i];
    if ((pool[F_FLAGS * cap + i] & KC_VF_LOOP) && le > ls + 1u && p >= le) {
        // Half a block rarely crosses more than one loop: one subtraction,
        // the remainder (a long division) only when it does.
        p -= le - ls;
        if (p >= le) p = ls + (p - ls) % (le - ls);
    }
    const uint64_t top = (uint64_t)L.phase_mask << L.phase_shift | ((1ull << L.phase_shift) - 1u);
    return (uint32_t)(p < top ? p : top);
}

__device__ __forceinline__ uint32_t sort_key(const uint32_t* pool, uint32_t cap, uint32_t i,
                                             const SortLayout& L) {
    const uint32_t stage = pool[F_ENV_STAGE * cap + i];
    uint32_t region = L.dead_region;
    if (stage != ENV_DEAD) region = min(pool[F_REGION * cap + i], L.dead_region - 1u);
    const uint32_t ph = (predicted_phase(pool, cap, i, L) >> L.phase_shift) & L.phase_mask;
    return (region << L.region_shift) | (min(stage, 7u) << L.stage_shift) | ph;
}

__device__ __forceinline__ uint32_t sort_chunk(uint32_t n, uint32_t nblocks) {
    const uint32_t c = (n + nblocks - 1u) / nblocks;
    return (c + 255u) & ~255u;
}

// Digit widths the pool sort can run with (kc_config::sort_radix_bits): a
// pass handles RB key bits with 2^RB bins per CTA.
constexpr uint32_t SORT_RADIX_MIN = 4, SORT_RADIX_MAX = 10, SORT_RADIX_DEFAULT = 8;

// Pass `shift`: count digit occurrences per CTA chunk into counts[d * G + cta].
// Pass 0 computes keys from the pool (and stores them in `keys_save`, when
// given, for that pass's scatter); later passes read the key array.
// `totals` (when given) also receives each digit's count over all CTAs, for
// sort_offsets_body; it must be zero when the pass starts.
template <uint32_t RB>
__device__ __forceinline__ void sort_count_body(PoolArgs a, SortLayout L, const uint32_t* keys, uint32_t shift,
                                                uint32_t* counts, uint32_t cta, uint32_t ctas,
                                                uint32_t* totals = nullptr, uint32_t* keys_save = nullptr) {
    constexpr uint32_t BINS = 1u << RB;
    __shared__ uint32_t h[BINS];
    const uint32_t n = a.st->live_render;
    for (uint32_t d = threadIdx.x; d < BINS; d += blockDim.x) h[d] = 0u;
    __syncthreads();
    const uint32_t chunk = sort_chunk(n, ctas);
    const uint32_t lo = cta * chunk, hi = min(n, lo + chunk);
    for (uint32_t i = lo + threadIdx.x; i < hi; i += 256u) {
        uint32_t k;
        if (keys) {
            k = keys[i];
        } else {
            k = sort_key(a.pool, a.cap, i, L);
            if (keys_save) keys_save[i] = k;
        }
        atomicAdd(&h[(k >> shift) & (BINS - 1u)], 1u);
    }
    __syncthreads();
    for (uint32_t d = threadIdx.x; d < BINS; d += blockDim.x) {
        counts[d * ctas + cta] = h[d];
        if (totals && h[d]) atomicAdd(&totals[d], h[d]);
    }
}

// The digit-major exclusive scan of counts[d * ctas + c] for one pass, one
// warp per digit d (any number of CTAs of any width): the digit's base is the
// sum of the totals of the digits below it, and the warp scans its digit's
// per-CTA counts in place on top of that base (each lane a contiguous run of
// CTAs, lane sums scanned with shuffles). The last digit writes the grand
// total. Replaces a single-CTA scan of all 2^RB * ctas words.
__device__ __forceinline__ void sort_offsets_body(uint32_t* counts, uint32_t ctas, uint32_t bins,
                                                  const uint32_t* totals, uint32_t* total, uint32_t d) {
    if (d >= bins) return;
    const uint32_t lane = lane_id();
    uint32_t base = 0;
    for (uint32_t k = lane; k < d; k += 32u) base += totals[k];
#pragma unroll
    for (int o = 16; o; o >>= 1) base += __shfl_xor_sync(0xFFFFFFFFu, base, o);
    uint32_t* row = counts + (size_t)d * ctas;
    const uint32_t per = (ctas + 31u) / 32u;
    const uint32_t c0 = min(ctas, lane * per), c1 = min(ctas, c0 + per);
    uint32_t local = 0;
    for (uint32_t c = c0; c < c1; ++c) local += row[c];
    uint32_t x = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    uint32_t run = base + x - local;
    for (uint32_t c = c0; c < c1; ++c) {
        const uint32_t v = row[c];
        row[c] = run;
        run += v;
    }
    if (d == bins - 1u && lane == 31u) *total = run;
}

// Stable scatter of one pass. keys_in == nullptr on the first pass (keys and
// indices come from the pool order). Each 256-key step ranks equal digits
// inside a warp with __match_any_sync and across the CTA's 8 warps with
// per-warp digit counts, so keys keep their input order within a digit.
template <uint32_t RB>
__device__ __forceinline__ void sort_scatter_body(PoolArgs a, SortLayout L, const uint32_t* keys_in,
                                                      const uint32_t* idx_in, uint32_t* keys_out,
                                                      uint32_t* idx_out, uint32_t shift,
                                                      const uint32_t* offsets, uint32_t cta, uint32_t ctas) {
    constexpr uint32_t BINS = 1u << RB;
    __shared__ uint32_t run[BINS];
    __shared__ uint32_t wcnt[8][BINS];
    const uint32_t n = a.st->live_render;
    const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
    for (uint32_t d = threadIdx.x; d < BINS; d += blockDim.x) run[d] = offsets[d * ctas + cta];
    const uint32_t chunk = sort_chunk(n, ctas);
    const uint32_t lo = cta * chunk, hi = min(n, lo + chunk);
    for (uint32_t t0 = lo; t0 < hi; t0 += 256u) {
        for (uint32_t d = threadIdx.x; d < BINS; d += blockDim.x)
            for (uint32_t k = 0; k < 8; ++k) wcnt[k][d] = 0u;
        __syncthreads();
        const uint32_t i = t0 + threadIdx.x;
        const bool valid = i < hi;
        uint32_t key = 0, id = 0, d = BINS + lane;  // invalid lanes get unique dummy digits
        if (valid) {
            key = keys_in ? keys_in[i] : sort_key(a.pool, a.cap, i, L);
            id = idx_in ? idx_in[i] : i;
            d = (key >> shift) & (BINS - 1u);
        }
        const uint32_t peers = __match_any_sync(0xFFFFFFFFu, d);
        const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
        if (valid && rank == 0) wcnt[w][d] = __popc(peers);
        __syncthreads();
        if (valid) {
            uint32_t before = run[d];
            for (uint32_t k = 0; k < w; ++k) before += wcnt[k][d];
            const uint32_t dst = before + rank;
            keys_out[dst] = key;
            idx_out[dst] = id;
        }
        __syncthreads();
        for (uint32_t dd = threadIdx.x; dd < BINS; dd += blockDim.x) {
            uint32_t tot = 0;
            for (uint32_t k = 0; k < 8; ++k) tot += wcnt[k][dd];
            run[dd] += tot;
        }
        __syncthreads();
    }
}

// Scan counts[2^RB * G] digit-major (one CTA).
// (k_scan_counts handles it: it is a plain exclusive scan of m words.)

// Copy the sorted survivors into the other pool buffer.
__device__ __forceinline__ void sort_gather_body(PoolArgs a, const uint32_t* idx, uint32_t cta, uint32_t ctas) {
    const uint32_t n = a.st->live_new;
    for (uint32_t j = cta * blockDim.x + threadIdx.x; j < n; j += ctas * blockDim.x)
        copy_voice(a.pool, a.pool_out, a.cap, idx[j], j);
}

}  // namespace kc
