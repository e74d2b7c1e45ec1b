// synth.cu -- host orchestrator and C ABI of the B200 synthesis backend.
//
// One kc_synth is one Backend (src/backend.rs:22-58): it owns the device copy
// of the sample pool and params tables, a double-buffered structure-of-arrays
// voice pool in HBM, one CUDA stream, and pinned staging for the per-block
// inputs. A block is a fixed sequence of kernel launches whose counts all live
// on the device (DevState), so nothing comes back to the host between the
// steal, spawn, render, mix and compaction passes; kc_render then reads the
// stereo block and the state words back in one copy.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"
#include "pool_ops.cuh"
#include "render.cuh"
#include "synth_impl.cuh"

// The single-context kernels: each runs one pass body (pool_ops.cuh) over
// this launch's own grid.
namespace kc {

__global__ void k_admit(PoolArgs a, uint32_t* sel_hist, BlockCtl* ctl, uint32_t want32, uint32_t chan_active) {
    for (uint32_t i = threadIdx.x; i < SEL_ROUNDS * 256u; i += blockDim.x) sel_hist[i] = 0u;
    if (threadIdx.x == 0) admit_state(a, ctl, want32, chan_active);
}

__global__ void __launch_bounds__(256) k_select_hist(PoolArgs a, uint32_t* sel_hist, uint32_t round) {
    select_hist_body(a, sel_hist, round, blockIdx.x, gridDim.x);
}

__global__ void __launch_bounds__(256) k_select_refine(PoolArgs a, const uint32_t* sel_hist, uint32_t round) { select_refine_body(a, sel_hist, round); }

__global__ void __launch_bounds__(256) k_mark_stolen(PoolArgs a) { mark_stolen_body(a, blockIdx.x, gridDim.x); }

__global__ void __launch_bounds__(256) k_spawn(PoolArgs a, const kc_spawn_cmd* __restrict__ cmds) {
    spawn_body(a, cmds, blockIdx.x, gridDim.x);
}

__global__ void __launch_bounds__(256) k_compact_count(PoolArgs a, uint32_t* counts) {
    compact_count_body(a, counts, blockIdx.x, gridDim.x);
}

__global__ void __launch_bounds__(1024) k_scan_counts(uint32_t* counts, uint32_t m, uint32_t* total) { scan_counts_body(counts, m, total); }

__global__ void __launch_bounds__(256) k_compact_scatter(PoolArgs a, const uint32_t* offsets) {
    compact_scatter_body(a, offsets, blockIdx.x, gridDim.x);
}

__global__ void k_commit(DevState* st, const uint32_t* total) { commit_body(st, total); }

template <uint32_t RB>
__global__ void __launch_bounds__(256) k_sort_count(PoolArgs a, SortLayout L, const uint32_t* keys,
                                                    uint32_t shift, uint32_t* counts, uint32_t* totals,
                                                    uint32_t* keys_save) {
    sort_count_body<RB>(a, L, keys, shift, counts, blockIdx.x, gridDim.x, totals, keys_save);
}

// One warp per digit: 8 digits per CTA.
__global__ void __launch_bounds__(256) k_sort_offsets(uint32_t* counts, uint32_t ctas, uint32_t bins,
                                                      const uint32_t* totals, uint32_t* total) {
    sort_offsets_body(counts, ctas, bins, totals, total, blockIdx.x * 8u + (threadIdx.x >> 5));
}

// The scatter also clears the digit totals for the next pass (nothing reads
// them once the offsets are formed).
template <uint32_t RB>
__global__ void __launch_bounds__(256) k_sort_scatter(PoolArgs a, SortLayout L, const uint32_t* keys_in,
                                                      const uint32_t* idx_in, uint32_t* keys_out,
                                                      uint32_t* idx_out, uint32_t shift,
                                                      const uint32_t* offsets, uint32_t* totals) {
    if (blockIdx.x == 0)
        for (uint32_t d = threadIdx.x; d < (1u << RB); d += blockDim.x) totals[d] = 0u;
    sort_scatter_body<RB>(a, L, keys_in, idx_in, keys_out, idx_out, shift, offsets, blockIdx.x, gridDim.x);
}

// One LSD pass of the pool sort at digit width RB: count (with the digit
// totals), the digit-major offsets, scatter. `totals` is zero on entry and on
// return. Pass 0 (kin null) computes the keys once, in the count, into
// `ksave`, and its scatter reads them from there.
template <uint32_t RB>
void sort_pass(cudaStream_t q, uint32_t G, const PoolArgs& pa, const SortLayout& L, const uint32_t* kin,
               const uint32_t* iin, uint32_t* kout, uint32_t* iout, uint32_t shift, uint32_t* counts,
               uint32_t* totals, uint32_t* total, uint32_t* ksave) {
    constexpr uint32_t BINS = 1u << RB;
    k_sort_count<RB><<<G, 256, 0, q>>>(pa, L, kin, shift, counts, totals, kin ? nullptr : ksave);
    k_sort_offsets<<<(BINS + 7u) / 8u, 256, 0, q>>>(counts, G, BINS, totals, total);
    k_sort_scatter<RB><<<G, 256, 0, q>>>(pa, L, kin ? kin : ksave, iin, kout, iout, shift, counts, totals);
}

void sort_pass_rb(uint32_t rb, cudaStream_t q, uint32_t G, const PoolArgs& pa, const SortLayout& L,
                  const uint32_t* kin, const uint32_t* iin, uint32_t* kout, uint32_t* iout, uint32_t shift,
                  uint32_t* counts, uint32_t* totals, uint32_t* total, uint32_t* ksave) {
    switch (rb) {
        case 4: sort_pass<4>(q, G, pa, L, kin, iin, kout, iout, shift, counts, totals, total, ksave); break;
        case 5: sort_pass<5>(q, G, pa, L, kin, iin, kout, iout, shift, counts, totals, total, ksave); break;
        case 6: sort_pass<6>(q, G, pa, L, kin, iin, kout, iout, shift, counts, totals, total, ksave); break;
        case 7: sort_pass<7>(q, G, pa, L, kin, iin, kout, iout, shift, counts, totals, total, ksave); break;
        case 9: sort_pass<9>(q, G, pa, L, kin, iin, kout, iout, shift, counts, totals, total, ksave); break;
        case 10: sort_pass<10>(q, G, pa, L, kin, iin, kout, iout, shift, counts, totals, total, ksave); break;
        default: sort_pass<8>(q, G, pa, L, kin, iin, kout, iout, shift, counts, totals, total, ksave); break;
    }
}

__global__ void __launch_bounds__(256) k_sort_gather(PoolArgs a, const uint32_t* idx) { sort_gather_body(a, idx, blockIdx.x, gridDim.x); }

// The f32 copy of the sample pool: one conversion per sample, at creation.
__global__ void __launch_bounds__(256) k_convert_pool(const int16_t* __restrict__ pcm, float* __restrict__ pcmf,
                                                      uint64_t n) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        pcmf[i] = fmaxf(__fmul_rn((float)pcm[i], 1.0f / 32767.0f), -1.0f);
}

// The fractional path's tap pairs, from the f32 copy (and its zero pad):
// entry i = (s_i, (s_{i+1} - s_i) * 2^-32). The difference is rounded once,
// as the reference rounds `s1 - s0`, and the power-of-two scale is exact, so
// (d * 2^-32) * f32(lo) is the reference's (s1 - s0) * (lo as f32 * 2^-32)
// bit for bit (render.cuh, hot_tile). Entries past the pool pair zeros.
__global__ void __launch_bounds__(256) k_pair_pool(const float* __restrict__ pcmf, float2* __restrict__ pcmp,
                                                   uint64_t n, uint64_t n_pad) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_pad; i += (uint64_t)gridDim.x * blockDim.x) {
        const float s0 = i < n ? pcmf[i] : 0.0f;
        const float s1 = i + 1 < n ? pcmf[i + 1] : 0.0f;
        pcmp[i] = make_float2(s0, __fmul_rn(__fsub_rn(s1, s0), 2.3283064365386963e-10f));
    }
}

}  // namespace kc

using namespace kc;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

#define KC_CUDA(call)                                                                   \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return fail(KC_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

const char* kPassNames[kc::N_TIMERS] = {"steal", "spawn", "render", "reduce", "compact"};

uint32_t max_steal_of(const kc_config& c) {
    const uint64_t n = (uint64_t)c.max_voices * c.max_steal_percent / 100;
    const uint32_t v = (uint32_t)n;
    return v > 1 ? v : 1;
}

uint32_t clz32(uint32_t v) { return v ? (uint32_t)__builtin_clz(v) : 32u; }

uint32_t radix_of(const kc_config& c) { return c.sort_radix_bits ? c.sort_radix_bits : SORT_RADIX_DEFAULT; }

// SortKeyLayout::plan, src/gpu/mod.rs:77-105.
SortLayout plan_sort(uint32_t n_regions, uint32_t max_len, uint32_t block_frames) {
    SortLayout L{};
    L.half = block_frames / 2;
    L.dead_region = std::max<uint32_t>(n_regions, 1);
    const uint32_t region_bits = 32 - clz32(L.dead_region);
    const uint32_t stage_bits = 3;
    const uint32_t len_bits = 32 - clz32(std::max<uint32_t>(max_len, 1));
    const uint32_t room = region_bits + stage_bits >= 32 ? 0 : 32 - (region_bits + stage_bits);
    const uint32_t phase_bits = std::min(room, len_bits);
    L.phase_shift = len_bits > phase_bits ? len_bits - phase_bits : 0;
    L.phase_mask = phase_bits >= 32 ? 0xFFFFFFFFu : ((1u << phase_bits) - 1u);
    L.bits = region_bits + stage_bits + phase_bits;
    L.region_shift = phase_bits + stage_bits;
    L.stage_shift = phase_bits;
    return L;
}

template <int I, bool C, bool S, int M, int V, bool D = false>
void* render_fn() {
    return reinterpret_cast<void*>(&k_render<I, C, S, M, V, D>);
}

// Two voices per lane is instantiated for the linear interpolator and the
// f32 mix only (the combinations the autotuner chooses between); so are the
// 32-frame unit tiles (`dbl`), for one voice per lane.
template <int I, bool C, bool S, int M>
void* render_v(uint32_t v, bool dbl) {
    if constexpr (I == KC_INTERP_LINEAR && M == KC_MIX_F32_TREE) {
        if (v == 2) return render_fn<I, C, S, M, 2>();
        if (dbl) return render_fn<I, C, S, M, 1, true>();
    }
    return render_fn<I, C, S, M, 1>();
}

template <int I, bool C, bool S>
void* render_m(uint32_t mix, uint32_t v, bool dbl) {
    if (mix == KC_MIX_TWO_SUM) return render_v<I, C, S, KC_MIX_TWO_SUM>(v, dbl);
    if (mix == KC_MIX_F64) return render_v<I, C, S, KC_MIX_F64>(v, dbl);
    return render_v<I, C, S, KC_MIX_F32_TREE>(v, dbl);
}

template <int I, bool C>
void* render_sm(bool strict, uint32_t mix, uint32_t v, bool dbl) {
    return strict ? render_m<I, C, true>(mix, v, dbl) : render_m<I, C, false>(mix, v, dbl);
}

// The render instantiation for [interp][chan][strict][mix][voices per
// lane][32-frame unit tiles]. Both tile lengths give the same output bits.
void* render_table(uint32_t interp, bool chan, bool strict, uint32_t mix, uint32_t v, bool dbl = false) {
    switch (interp) {
        case KC_INTERP_NEAREST:
            return chan ? render_sm<0, true>(strict, mix, v, dbl) : render_sm<0, false>(strict, mix, v, dbl);
        case KC_INTERP_LINEAR:
            return chan ? render_sm<1, true>(strict, mix, v, dbl) : render_sm<1, false>(strict, mix, v, dbl);
        default:
            return chan ? render_sm<2, true>(strict, mix, v, dbl) : render_sm<2, false>(strict, mix, v, dbl);
    }
}

}  // namespace

namespace kc {
// The error text of the last failing call on this thread, for entry points
// defined in other files of this library.
__attribute__((visibility("hidden"))) int set_last_error(int code, const std::string& msg) {
    return fail(code, msg);
}
}  // namespace kc



namespace {

void free_all(kc_synth* s) {
    if (!s) return;
    cudaFree(s->pool[0]);
    cudaFree(s->pool[1]);
    cudaFree(s->pcm);
    cudaFree(s->pcmf);
    cudaFree(s->pcmp);
    cudaFree(s->params);
    cudaFree(s->gates);
    cudaFree(s->chan);
    cudaFree(s->cmds);
    cudaFree(s->out);
    cudaFree(s->partial);
    cudaFree(s->partial_c);
    cudaFree(s->st);
    cudaFree(s->ctl);
    cudaFree(s->sel_hist);
    cudaFree(s->counts);
    cudaFree(s->total);
    cudaFree(s->sort_totals);
    for (int i = 0; i < 2; ++i) {
        cudaFree(s->keys[i]);
        cudaFree(s->idx[i]);
    }
    cudaFreeHost(s->h_gates);
    cudaFreeHost(s->h_chan);
    cudaFreeHost(s->h_cmds);
    cudaFreeHost(s->h_out);
    cudaFreeHost(s->h_st);
    for (auto& e : s->ev)
        if (e) cudaEventDestroy(e);
    if (s->ev_inputs) cudaEventDestroy(s->ev_inputs);
    for (auto& set : s->ring)
        for (auto& e : set) cudaEventDestroy(e);
    if (s->stream) cudaStreamDestroy(s->stream);
    if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
}

// Config::validate (src/config.rs:412-525), the part the backend reads, plus
// this backend's own tiling constraints.
int validate(const kc_config& c) {
    if (c.sample_rate < 8000 || c.sample_rate > 768000) return fail(KC_ERR_INVALID, "sample_rate out of range");
    if (c.block_frames == 0 || c.block_frames % MIX_TILE != 0 || c.block_frames > 65535)
        return fail(KC_ERR_INVALID, "block_frames must be a non-zero multiple of 16, at most 65535");
    if (c.gate_frames == 0 || c.gate_frames % MIX_TILE != 0 || c.block_frames % c.gate_frames != 0)
        return fail(KC_ERR_INVALID, "gate_frames must be a multiple of 16 that divides block_frames");
    if (c.max_voices == 0) return fail(KC_ERR_INVALID, "max_voices must be non-zero");
    if (c.steal_fade_frames == 0 || c.steal_fade_frames >= c.block_frames)
        return fail(KC_ERR_INVALID, "steal_fade_frames must be in 1..block_frames-1");
    if (c.max_steal_percent == 0 || c.max_steal_percent > 100)
        return fail(KC_ERR_INVALID, "max_steal_percent must be in 1..=100");
    if (c.steal_rule > 2 || c.admit_rule > 1 || c.interpolation > 2 || c.decay_curve > 1 ||
        c.release_curve > 1 || c.mix_mode > 2)
        return fail(KC_ERR_INVALID, "unknown enum value in config");
    if (c.voices_per_lane > 2) return fail(KC_ERR_INVALID, "voices_per_lane must be 0, 1 or 2");
    if (c.sort_radix_bits && (c.sort_radix_bits < SORT_RADIX_MIN || c.sort_radix_bits > SORT_RADIX_MAX))
        return fail(KC_ERR_INVALID, "sort_radix_bits must be 0 or in 4..=10");
    if (c.unit_tile_frames != 0 && c.unit_tile_frames != 16 && c.unit_tile_frames != 32)
        return fail(KC_ERR_INVALID, "unit_tile_frames must be 0, 16 or 32");
    if (c.max_param_variants == 0 || c.max_param_variants > 64)
        return fail(KC_ERR_INVALID, "max_param_variants must be in 1..=64");
    return KC_OK;
}

// Enqueue one block on the stream. All inputs are device pointers.
uint32_t launches_for(const kc_synth* s, bool sort_now);

// `inputs_ready` (optional): an event the spawn pass waits for, recorded
// after the block's inputs were copied up on another stream.
int enqueue_block(kc_synth* s, const uint32_t* d_gates, const uint32_t* d_chan, bool bend, bool gain,
                  bool variant, const kc_spawn_cmd* d_cmds, uint32_t n_cmds, float* d_out,
                  cudaEvent_t inputs_ready = nullptr) {
    cudaStream_t q = s->stream;
    const kc_config& c = s->cfg;
    const uint32_t chan_active = (bend ? 1u : 0u) | (gain ? 2u : 0u) | (variant ? 4u : 0u);

    PoolArgs pa{};
    pa.pool = s->pool[s->parity];
    pa.pool_out = s->pool[s->parity ^ 1];
    pa.cap = s->cap;
    pa.st = s->st;
    pa.ctl = s->ctl;
    pa.max_voices = c.max_voices;
    pa.max_steal = max_steal_of(c);
    pa.steal_rule = c.steal_rule;
    pa.admit_rule = c.admit_rule;
    const uint32_t span = c.block_frames > c.steal_fade_frames ? c.block_frames - c.steal_fade_frames : 1;
    pa.steal_span = std::max<uint32_t>(span, 1);
    pa.render_warps = s->render_warps;
    pa.voices_per_lane = s->vpl;

    cudaEvent_t* ev = s->ev;
    if (s->profile) {
        if (s->ring_pending == s->ring.size()) {
            std::vector<cudaEvent_t> set(kc::N_TIMERS + 1);
            for (auto& e : set) KC_CUDA(cudaEventCreate(&e));
            s->ring.push_back(std::move(set));
        }
        ev = s->ring[s->ring_pending++].data();
    }
    if (s->profile) cudaEventRecord(ev[0], q);
    k_admit<<<1, 256, 0, q>>>(pa, s->sel_hist, s->ctl, n_cmds, chan_active);
    // ---- 1. steal ----
    if (c.steal_rule != KC_STEAL_DROP_NEW) {
        for (uint32_t r = 0; r < SEL_ROUNDS; ++r) {
            k_select_hist<<<s->pool_ctas, 256, 0, q>>>(pa, s->sel_hist, r);
            k_select_refine<<<1, 256, 0, q>>>(pa, s->sel_hist, r);
        }
        k_mark_stolen<<<s->pool_ctas, 256, 0, q>>>(pa);
    }
    if (s->profile) cudaEventRecord(ev[1], q);
    // ---- 2. spawn ----
    if (inputs_ready) KC_CUDA(cudaStreamWaitEvent(q, inputs_ready, 0));
    k_spawn<<<s->pool_ctas, 256, 0, q>>>(pa, d_cmds);
    if (s->profile) cudaEventRecord(ev[2], q);
    // ---- 3. render ----
    RenderArgs ra{};
    ra.pool = pa.pool;
    ra.cap = s->cap;
    ra.pcm = s->pcm;
    ra.pcmf = s->pcmf;
    ra.pcmp = s->pcmp;
    ra.pcm_len = (uint32_t)std::min<uint64_t>(s->pcm_len, 0xFFFFFFFFull);
    ra.params = s->params;
    ra.params_per = s->params_per;
    ra.n_slots = s->n_slots;
    ra.gates = d_gates;
    ra.chan = d_chan;
    ra.ctl = s->ctl;
    ra.st = s->st;
    ra.partial = s->partial;
    ra.partial_c = s->partial_c;
    ra.block_frames = c.block_frames;
    ra.gate_frames = c.gate_frames;
    ra.fade = c.steal_fade_frames;
    ra.env_floor = c.env_floor;
    ra.exp_decay = c.decay_curve == KC_CURVE_EXPONENTIAL;
    ra.exp_release = c.release_curve == KC_CURVE_EXPONENTIAL;
    const bool dbl = c.unit_tile_frames == 32 || (c.unit_tile_frames == 0 && s->hot_tiles);
    void* fn = render_table(c.interpolation, chan_active != 0, c.strict_fp != 0, c.mix_mode, s->vpl, dbl);
    void* args[] = {&ra};
    KC_CUDA(cudaLaunchKernel(fn, dim3(s->render_ctas), dim3(RENDER_WARPS * 32), args, s->render_smem, q));
    if (s->profile) cudaEventRecord(ev[3], q);
    // ---- 4. reduce ----
    const uint32_t samples = c.block_frames * 2;
    if (c.mix_mode == KC_MIX_F32_TREE)
        k_reduce<KC_MIX_F32_TREE><<<(samples + 31) / 32, 256, 0, q>>>(s->partial, s->partial_c, d_out, s->st, samples);
    else if (c.mix_mode == KC_MIX_TWO_SUM)
        k_reduce<KC_MIX_TWO_SUM><<<(samples + 31) / 32, 256, 0, q>>>(s->partial, s->partial_c, d_out, s->st, samples);
    else
        k_reduce<KC_MIX_F64><<<(samples + 31) / 32, 256, 0, q>>>(s->partial, s->partial_c, d_out, s->st, samples);
    if (s->profile) cudaEventRecord(ev[4], q);
    // ---- 5. compact (and sort) ----
    k_compact_count<<<s->compact_ctas, 256, 0, q>>>(pa, s->counts);
    k_scan_counts<<<1, 1024, 0, q>>>(s->counts, s->compact_ctas, s->total);
    k_commit<<<1, 1, 0, q>>>(s->st, s->total);
    const bool sort_now = sort_this_block(s);
    if (!sort_now) {
        k_compact_scatter<<<s->compact_ctas, 256, 0, q>>>(pa, s->counts);
    } else {
        const uint32_t passes = (s->sort.bits + s->radix - 1) / s->radix;
        const uint32_t G = s->compact_ctas;
        const SortLayout L = block_sort_layout(s, bend ? d_chan : nullptr);
        int cur = 0;
        for (uint32_t p = 0; p < passes; ++p) {
            const uint32_t shift = s->radix * p;
            const uint32_t* kin = p == 0 ? nullptr : s->keys[cur];
            const uint32_t* iin = p == 0 ? nullptr : s->idx[cur];
            // Pass 0 writes keys[1] and idx[1]: idx[0] holds its computed keys.
            sort_pass_rb(s->radix, q, G, pa, L, kin, iin, s->keys[cur ^ 1], s->idx[cur ^ 1], shift, s->counts,
                         s->sort_totals, s->total + 1, s->idx[0]);
            cur ^= 1;
        }
        k_sort_gather<<<s->pool_ctas, 256, 0, q>>>(pa, s->idx[cur]);
    }
    if (s->profile) cudaEventRecord(ev[5], q);
    KC_CUDA(cudaGetLastError());
    s->parity ^= 1;
    s->launches += launches_for(s, sort_now);
    ++s->blocks;
    return KC_OK;
}

// After a synchronisation: fold every profiled block's pass times into the
// totals and keep the last block's as `last_ms`.
void drain_timings(kc_synth* s) {
    for (size_t b = 0; b < s->ring_pending; ++b) {
        for (int i = 0; i < kc::N_TIMERS; ++i) {
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, s->ring[b][i], s->ring[b][i + 1]);
            s->total_ms[i] += ms;
            s->last_ms[i] = ms;
        }
        s->total_blocks += 1;
        s->have_timings = true;
    }
    s->ring_pending = 0;
}

}  // namespace

namespace {
uint32_t launches_for(const kc_synth* s, bool sort_now) {
    uint32_t n = 1;                                                       // admit
    if (s->cfg.steal_rule != KC_STEAL_DROP_NEW) n += 2 * SEL_ROUNDS + 1;  // select + mark
    n += 1 + 1 + 1;                                                       // spawn, render, reduce
    n += 3;                                                               // count, scan, commit
    if (!sort_now) n += 1;
    else n += 3 * ((s->sort.bits + s->radix - 1) / s->radix) + 1;
    return n;
}

// Device bytes a context holds, from its geometry (kc_synth_create's
// allocations, in the same order).
uint64_t footprint(const kc_config& c, uint64_t cap, uint64_t pcm_len, uint64_t params_per, uint32_t n_slots,
                   uint32_t tiles, uint32_t cmds_cap, uint32_t partial_slices, uint32_t compact_ctas) {
    const uint64_t samples = (uint64_t)c.block_frames * 2;
    uint64_t n = 2ull * VOICE_FIELDS * cap * 4;                                 // pool, double-buffered
    n += std::max<uint64_t>(pcm_len, 1) * 2 + 64;                               // sample pool (i16)
    n += (pcm_len + ZERO_PAD) * 12;                                              // its f32 copy and tap pairs
    n += params_per * sizeof(kc_region_params) * n_slots;                       // params variants
    n += (uint64_t)tiles * (KC_GATE_SLOTS + KC_BEND_CHANNELS * KC_CHAN_FIELDS) * 4;
    n += (uint64_t)cmds_cap * sizeof(kc_spawn_cmd) + samples * 4;               // spawn buffer, block
    n += (uint64_t)partial_slices * samples * (c.mix_mode == KC_MIX_F64 ? 8 : 4);
    if (c.mix_mode == KC_MIX_TWO_SUM) n += (uint64_t)partial_slices * samples * 4;
    n += sizeof(DevState) + sizeof(BlockCtl) + SEL_ROUNDS * 256 * 4 + 16;
    n += (uint64_t)std::max<uint32_t>(256u, 1u << radix_of(c)) * compact_ctas * 4;  // digit counts
    n += (1u << SORT_RADIX_MAX) * 4;                                            // digit totals
    if (c.sort_voices) n += 4ull * cap * 4;                                     // keys, indices
    return n;
}

uint32_t partial_slices_of(uint64_t cap, uint32_t vpl, uint32_t render_warps) {
    const uint64_t batches = (cap + 32ull * vpl - 1) / (32ull * vpl);
    return (uint32_t)std::min<uint64_t>(render_warps, std::max<uint64_t>(batches, 1));
}

// Render CTAs per SM for a config (the occupancy the grid is sized by).
int render_occupancy(const kc_config& c, uint32_t vpl, size_t smem, int* per_sm) {
    void* fn = render_table(c.interpolation, true, c.strict_fp != 0, c.mix_mode, vpl);
    for (int ch = 0; ch < 2; ++ch) {
        void* f2 = render_table(c.interpolation, ch != 0, c.strict_fp != 0, c.mix_mode, vpl);
        KC_CUDA(cudaFuncSetAttribute(f2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    }
    KC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, fn, RENDER_WARPS * 32, smem));
    *per_sm = std::max(*per_sm, 1);
    return KC_OK;
}

}  // namespace

extern "C" {

const char* kc_last_error(void) { return g_err.c_str(); }

int kc_config_default(kc_config* c) {
    if (!c) return fail(KC_ERR_INVALID, "null config");
    std::memset(c, 0, sizeof(*c));
    c->sample_rate = 48000;
    c->block_frames = 4096;
    c->gate_frames = 32;
    c->max_voices = 1u << 20;
    c->max_steal_percent = 25;
    c->steal_fade_frames = 96;
    c->steal_rule = KC_STEAL_QUIETEST;
    c->admit_rule = KC_ADMIT_LOUDEST;
    c->interpolation = KC_INTERP_LINEAR;
    c->decay_curve = KC_CURVE_EXPONENTIAL;
    c->release_curve = KC_CURVE_EXPONENTIAL;
    c->env_floor = 1.0e-5f;
    c->sort_voices = 1;
    c->max_param_variants = 32;
    c->mix_mode = KC_MIX_F32_TREE;
    c->strict_fp = 1;
    c->device = 0;
    return KC_OK;
}

uint32_t kc_pool_slots(const kc_config* c) {
    const uint64_t s = (uint64_t)c->max_voices + max_steal_of(*c);
    return s > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)s;
}

int kc_synth_create(const kc_config* cfg, const int16_t* pool, uint64_t pool_len,
                    const kc_region_params* params, uint32_t params_len, uint32_t n_regions,
                    uint32_t max_sample_len, kc_synth** out) {
    if (!cfg || !out) return fail(KC_ERR_INVALID, "null argument");
    *out = nullptr;
    if (int rc = validate(*cfg)) return rc;
    if (params_len == 0 || !params) return fail(KC_ERR_INVALID, "params table is empty");
    if (pool_len && !pool) return fail(KC_ERR_INVALID, "null sample pool");
    const uint64_t slots = kc_pool_slots(cfg);
    if (slots > 0x7FFFFFE0ull) return fail(KC_ERR_INVALID, "pool slots exceed 2^31");

    kc_synth* s = new kc_synth();
    s->cfg = *cfg;
    s->device = (int)cfg->device;
    auto bail = [&](int rc) {
        free_all(s);
        delete s;
        return rc;
    };
#define KC_TRY(call)                                                                      \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return bail(fail(e_ == cudaErrorMemoryAllocation ? KC_ERR_OOM : KC_ERR_CUDA,  \
                             std::string(#call) + ": " + cudaGetErrorString(e_)));        \
    } while (0)

    KC_TRY(cudaSetDevice(s->device));
    KC_TRY(cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, s->device));
    KC_TRY(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    KC_TRY(cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking));

    s->cap = (uint32_t)((slots + 31) & ~31ull);
    s->vpl = cfg->voices_per_lane == 2 ? 2u : 1u;
    s->radix = radix_of(*cfg);
    s->tiles = cfg->block_frames / cfg->gate_frames;
    s->params_per = params_len;
    s->n_slots = cfg->max_param_variants;
    s->pcm_len = pool_len;
    s->sort = plan_sort(n_regions, max_sample_len, cfg->block_frames);
    s->n_regions = n_regions;
    s->max_sample_len = max_sample_len;

    // Launch geometry: the render grid is every resident CTA of the device,
    // and the partial buffer has one slice per render warp.
    s->render_smem = (size_t)RENDER_WARPS * SM_WARP * sizeof(float);
    int per_sm = 0;
    if (int rc = render_occupancy(*cfg, s->vpl, s->render_smem, &per_sm)) return bail(rc);
    s->render_ctas = (uint32_t)(s->sms * per_sm);
    s->render_warps = s->render_ctas * RENDER_WARPS;
    s->pool_ctas = (uint32_t)s->sms * 4;
    s->compact_ctas = (uint32_t)s->sms * 2;

    const size_t pool_words = (size_t)VOICE_FIELDS * s->cap;
    KC_TRY(cudaMalloc(&s->pool[0], pool_words * 4));
    KC_TRY(cudaMalloc(&s->pool[1], pool_words * 4));
    KC_TRY(cudaMalloc(&s->pcm, std::max<uint64_t>(pool_len, 1) * 2 + 64));
    if (pool_len) KC_TRY(cudaMemcpy(s->pcm, pool, pool_len * 2, cudaMemcpyDefault));
    // The f32 copy, then ZERO_PAD zero frames (neutral lanes' taps).
    KC_TRY(cudaMalloc(&s->pcmf, (pool_len + ZERO_PAD) * 4));
    KC_TRY(cudaMemsetAsync(s->pcmf + pool_len, 0, ZERO_PAD * 4, s->stream));
    if (pool_len) {
        k_convert_pool<<<(unsigned)std::min<uint64_t>((pool_len + 255) / 256, (uint64_t)s->sms * 16), 256, 0,
                         s->stream>>>(s->pcm, s->pcmf, pool_len);
        KC_TRY(cudaGetLastError());
    }
    KC_TRY(cudaMalloc(&s->pcmp, (pool_len + ZERO_PAD) * sizeof(float2)));
    k_pair_pool<<<(unsigned)std::min<uint64_t>((pool_len + ZERO_PAD + 255) / 256, (uint64_t)s->sms * 16), 256, 0,
                  s->stream>>>(s->pcmf, s->pcmp, pool_len, pool_len + ZERO_PAD);
    KC_TRY(cudaGetLastError());
    const size_t per_bytes = (size_t)params_len * sizeof(kc_region_params);
    KC_TRY(cudaMalloc(&s->params, per_bytes * s->n_slots));
    // Every slot starts as a copy of the bank's table, which is what
    // CpuSynth::params_of falls back to for a variant never uploaded.
    for (uint32_t v = 0; v < s->n_slots; ++v)
        KC_TRY(cudaMemcpy((char*)s->params + v * per_bytes, params, per_bytes, cudaMemcpyDefault));
    const size_t gate_words = (size_t)s->tiles * KC_GATE_SLOTS;
    const size_t chan_words = (size_t)s->tiles * KC_BEND_CHANNELS * KC_CHAN_FIELDS;
    KC_TRY(cudaMalloc(&s->gates, gate_words * 4));
    KC_TRY(cudaMalloc(&s->chan, chan_words * 4));
    KC_TRY(cudaMemset(s->gates, 0, gate_words * 4));
    KC_TRY(cudaMemset(s->chan, 0, chan_words * 4));
    s->cmds_cap = 4096;
    KC_TRY(cudaMalloc(&s->cmds, (size_t)s->cmds_cap * sizeof(kc_spawn_cmd)));
    const size_t samples = (size_t)cfg->block_frames * 2;
    KC_TRY(cudaMalloc(&s->out, samples * 4));
    // One partial slice per render warp that can own a voice: at most one
    // batch of 32 * voices-per-lane voices per slice, and never more slices
    // than the grid has warps (live + admitted <= cap).
    s->partial_slices = partial_slices_of(s->cap, s->vpl, s->render_warps);
    const size_t slice_bytes = cfg->mix_mode == KC_MIX_F64 ? 8 : 4;
    KC_TRY(cudaMalloc(&s->partial, (size_t)s->partial_slices * samples * slice_bytes));
    if (cfg->mix_mode == KC_MIX_TWO_SUM)
        KC_TRY(cudaMalloc(&s->partial_c, (size_t)s->partial_slices * samples * 4));
    KC_TRY(cudaMalloc(&s->st, sizeof(DevState)));
    KC_TRY(cudaMemset(s->st, 0, sizeof(DevState)));
    KC_TRY(cudaMalloc(&s->ctl, sizeof(BlockCtl)));
    KC_TRY(cudaMalloc(&s->sel_hist, SEL_ROUNDS * 256 * 4));
    KC_TRY(cudaMalloc(&s->counts, (size_t)std::max<uint32_t>(256u, 1u << s->radix) * s->compact_ctas * 4));
    KC_TRY(cudaMalloc(&s->total, 16));
    KC_TRY(cudaMalloc(&s->sort_totals, (1u << SORT_RADIX_MAX) * 4));
    KC_TRY(cudaMemset(s->sort_totals, 0, (1u << SORT_RADIX_MAX) * 4));
    if (cfg->sort_voices) {
        for (int i = 0; i < 2; ++i) {
            KC_TRY(cudaMalloc(&s->keys[i], (size_t)s->cap * 4));
            KC_TRY(cudaMalloc(&s->idx[i], (size_t)s->cap * 4));
        }
    }
    KC_TRY(cudaMallocHost(&s->h_gates, gate_words * 4));
    KC_TRY(cudaMallocHost(&s->h_chan, chan_words * 4));
    std::memset(s->h_gates, 0, gate_words * 4);
    std::memset(s->h_chan, 0, chan_words * 4);
    s->h_cmds_cap = 4096;
    KC_TRY(cudaMallocHost(&s->h_cmds, (size_t)s->h_cmds_cap * sizeof(kc_spawn_cmd)));
    KC_TRY(cudaMallocHost(&s->h_out, samples * 4));
    KC_TRY(cudaMallocHost(&s->h_st, sizeof(DevState)));
    for (auto& e : s->ev) KC_TRY(cudaEventCreate(&e));
    KC_TRY(cudaEventCreateWithFlags(&s->ev_inputs, cudaEventDisableTiming));
    KC_TRY(cudaDeviceSynchronize());
#undef KC_TRY
    *out = s;
    return KC_OK;
}

int kc_synth_clone(kc_synth* src, kc_synth** out) {
    if (!src) return fail(KC_ERR_INVALID, "null argument");
    return kc_synth_clone_config(src, &src->cfg, out);
}

int kc_synth_clone_config(kc_synth* src, const kc_config* cfg, kc_synth** out) {
    if (!src || !cfg || !out) return fail(KC_ERR_INVALID, "null argument");
    *out = nullptr;
    // Only the tunables that change how a block is computed may differ.
    kc_config a = src->cfg, b = *cfg;
    a.voices_per_lane = b.voices_per_lane = 0;
    a.sort_radix_bits = b.sort_radix_bits = 0;
    a.unit_tile_frames = b.unit_tile_frames = 0;
    if (std::memcmp(&a, &b, sizeof(a)) != 0)
        return fail(KC_ERR_INVALID, "clone config may differ from the source only in voices_per_lane, "
                                    "sort_radix_bits and unit_tile_frames");
    if (src->pending) return fail(KC_ERR_INVALID, "clone: the source has a block in flight");
    cudaSetDevice(src->device);
    KC_CUDA(cudaStreamSynchronize(src->stream));
    kc_synth* s = nullptr;
    // The bank and variant-0 table come straight from the source's device
    // copies (cudaMemcpyDefault resolves device pointers under UVA).
    if (int rc = kc_synth_create(cfg, src->pcm, src->pcm_len, src->params, src->params_per,
                                 src->n_regions, src->max_sample_len, &s))
        return rc;
    auto bail = [&](cudaError_t e) {
        kc_synth_destroy(s);
        return fail(KC_ERR_CUDA, std::string("clone: ") + cudaGetErrorString(e));
    };
    const size_t per_bytes = (size_t)src->params_per * sizeof(kc_region_params);
    cudaError_t e = cudaMemcpy(s->params, src->params, per_bytes * src->n_slots, cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(s->pool[0], src->pool[src->parity], (size_t)VOICE_FIELDS * src->cap * 4,
                       cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(s->st, src->st, sizeof(DevState), cudaMemcpyDeviceToDevice);
    if (e != cudaSuccess) return bail(e);
    s->parity = 0;
    s->stats = src->stats;
    s->blocks = src->blocks;  // the pool-sort interval continues where the source's stands
    s->hot_tiles = src->hot_tiles;
    *out = s;
    return KC_OK;
}

void kc_synth_destroy(kc_synth* s) {
    if (!s) return;
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    free_all(s);
    delete s;
}

namespace {
// The pinned staging buffers feed the in-flight block's host-to-device
// copies until its `ev_inputs` fires; the next block's inputs overwrite them
// only after that.
int staging_free(kc_synth* s) {
    if (!s->pending) return KC_OK;
    cudaSetDevice(s->device);
    KC_CUDA(cudaEventSynchronize(s->ev_inputs));
    return KC_OK;
}
}  // namespace

int kc_set_gates(kc_synth* s, const uint32_t* rows, size_t n) {
    if (!s || (!rows && n)) return fail(KC_ERR_INVALID, "null argument");
    if (n != (size_t)s->tiles * KC_GATE_SLOTS)
        return fail(KC_ERR_INVALID, "gate rows: expected tiles * 2048 words");
    if (int rc = staging_free(s)) return rc;
    std::memcpy(s->h_gates, rows, n * 4);
    return KC_OK;
}

int kc_set_channels(kc_synth* s, const uint32_t* rows, size_t n, int bend, int gain, int variant) {
    if (!s || (!rows && n)) return fail(KC_ERR_INVALID, "null argument");
    if (n != (size_t)s->tiles * KC_BEND_CHANNELS * KC_CHAN_FIELDS)
        return fail(KC_ERR_INVALID, "channel rows: expected tiles * 64 words");
    if (int rc = staging_free(s)) return rc;
    std::memcpy(s->h_chan, rows, n * 4);
    s->bend = bend != 0;
    s->gain = gain != 0;
    s->variant = variant != 0;
    return KC_OK;
}

int kc_set_params_variant(kc_synth* s, uint32_t index, const kc_region_params* data, size_t n) {
    if (!s) return fail(KC_ERR_INVALID, "null synth");
    if (index == 0) return KC_OK;  // the bank's own table (src/cpu.rs:314-316)
    if (n != s->params_per)
        return fail(KC_ERR_INVALID, "params variant " + std::to_string(index) + " has " + std::to_string(n) +
                                        " entries, expected " + std::to_string(s->params_per));
    if (index >= s->n_slots) return fail(KC_ERR_INVALID, "params variant is past the configured maximum");
    cudaSetDevice(s->device);
    KC_CUDA(cudaStreamSynchronize(s->stream));
    KC_CUDA(cudaMemcpy((char*)s->params + (size_t)index * n * sizeof(kc_region_params), data,
                       n * sizeof(kc_region_params), cudaMemcpyHostToDevice));
    return KC_OK;
}

int kc_spawn(kc_synth* s, const kc_spawn_cmd* cmds, size_t n) {
    if (!s || (!cmds && n)) return fail(KC_ERR_INVALID, "null argument");
    if (n > 0x7FFFFFFFull) return fail(KC_ERR_INVALID, "too many spawn commands");
    if (int rc = staging_free(s)) return rc;
    if (n > s->h_cmds_cap) {
        cudaSetDevice(s->device);
        KC_CUDA(cudaStreamSynchronize(s->stream));
        uint32_t nc = std::max<uint32_t>(s->h_cmds_cap, 1);
        while (nc < n) nc *= 2;
        cudaFreeHost(s->h_cmds);
        s->h_cmds = nullptr;
        s->h_cmds_cap = 0;
        if (cudaMallocHost(&s->h_cmds, (size_t)nc * sizeof(kc_spawn_cmd)) != cudaSuccess)
            return fail(KC_ERR_OOM, "pinned spawn staging");
        s->h_cmds_cap = nc;
    }
    // The CPU backend indexes the params and gate tables directly and would
    // panic on a bad index; reject such commands here instead of reading out
    // of bounds on the device. Validation and the copy into pinned staging run
    // together, split over a few threads for large blocks (a saturated
    // block's commands are megabytes); a refused call leaves no commands
    // staged.
    s->want = 0;
    const size_t chunk = (size_t)1 << 15;
    const unsigned workers = n >= 2 * chunk ? (unsigned)std::min<size_t>(4, n / chunk) : 1u;
    std::vector<int> bad(workers, 0);
    auto part = [&](unsigned w) {
        const size_t lo = n * w / workers, hi = n * (w + 1) / workers;
        for (size_t i = lo; i < hi; ++i)
            if (cmds[i].params >= s->params_per || cmds[i].gate_slot >= KC_GATE_SLOTS) {
                bad[w] = cmds[i].params >= s->params_per ? 1 : 2;
                return;
            }
        std::memcpy(s->h_cmds + lo, cmds + lo, (hi - lo) * sizeof(kc_spawn_cmd));
    };
    if (workers == 1) {
        if (n) part(0);
    } else {
        std::vector<std::thread> th;
        for (unsigned w = 1; w < workers; ++w) th.emplace_back(part, w);
        part(0);
        for (auto& t : th) t.join();
    }
    for (int b : bad) {
        if (b == 1) return fail(KC_ERR_INVALID, "spawn command params index out of range");
        if (b == 2) return fail(KC_ERR_INVALID, "spawn command gate_slot out of range");
    }
    s->want = (uint32_t)n;
    return KC_OK;
}

// Backend::render split at the device boundary: begin enqueues the block
// (input copies, every pass, the copies back) and returns; end waits for it.
int kc_render_begin(kc_synth* s) {
    if (!s) return fail(KC_ERR_INVALID, "null synth");
    if (s->pending) return fail(KC_ERR_INVALID, "a block is already in flight; end it first");
    cudaSetDevice(s->device);
    cudaStream_t q = s->stream;
    if (s->want > s->cmds_cap) {
        KC_CUDA(cudaStreamSynchronize(q));
        uint32_t nc = std::max<uint32_t>(s->cmds_cap, 1);
        while (nc < s->want) nc *= 2;
        cudaFree(s->cmds);
        s->cmds = nullptr;
        s->cmds_cap = 0;
        if (cudaMalloc(&s->cmds, (size_t)nc * sizeof(kc_spawn_cmd)) != cudaSuccess)
            return fail(KC_ERR_OOM, "device spawn buffer");
        s->cmds_cap = nc;
    }
    const size_t samples = (size_t)s->cfg.block_frames * 2;
    const size_t gate_words = (size_t)s->tiles * KC_GATE_SLOTS;
    const size_t chan_words = (size_t)s->tiles * KC_BEND_CHANNELS * KC_CHAN_FIELDS;
    // The inputs go up on the copy stream while the block's admission and
    // steal select (which read none of them) run; the spawn pass waits for
    // them. Nothing of an earlier block reads these buffers any more: a block
    // begun here has been ended (synchronised) before the next begins.
    cudaStream_t cq = s->copy_stream;
    KC_CUDA(cudaMemcpyAsync(s->gates, s->h_gates, gate_words * 4, cudaMemcpyHostToDevice, cq));
    KC_CUDA(cudaMemcpyAsync(s->chan, s->h_chan, chan_words * 4, cudaMemcpyHostToDevice, cq));
    if (s->want)
        KC_CUDA(cudaMemcpyAsync(s->cmds, s->h_cmds, (size_t)s->want * sizeof(kc_spawn_cmd),
                                cudaMemcpyHostToDevice, cq));
    KC_CUDA(cudaEventRecord(s->ev_inputs, cq));
    if (int rc = enqueue_block(s, s->gates, s->chan, s->bend, s->gain, s->variant, s->cmds, s->want, s->out,
                               s->ev_inputs))
        return rc;
    KC_CUDA(cudaMemcpyAsync(s->h_out, s->out, samples * 4, cudaMemcpyDeviceToHost, q));
    KC_CUDA(cudaMemcpyAsync(s->h_st, s->st, sizeof(DevState), cudaMemcpyDeviceToHost, q));
    s->want = 0;
    s->pending = true;
    return KC_OK;
}

int kc_render_end(kc_synth* s, float* out, size_t n) {
    if (!s || !out) return fail(KC_ERR_INVALID, "null argument");
    const size_t samples = (size_t)s->cfg.block_frames * 2;
    if (n != samples) return fail(KC_ERR_INVALID, "output must be block_frames * 2 samples");
    if (!s->pending) return fail(KC_ERR_INVALID, "no block in flight");
    cudaSetDevice(s->device);
    KC_CUDA(cudaStreamSynchronize(s->stream));
    s->pending = false;
    std::memcpy(out, s->h_out, samples * 4);
    s->stats.active_voices = s->h_st->live;
    if (s->h_st->all_tiles) s->hot_tiles = (uint64_t)s->h_st->hot_tiles * 2u >= s->h_st->all_tiles;
    s->stats.stolen = s->h_st->stolen;
    s->stats.dropped = s->h_st->dropped;
    uint32_t pb = s->h_st->peak_bits;
    std::memcpy(&s->stats.peak, &pb, 4);
    drain_timings(s);
    if (s->h_st->error)
        return fail(KC_ERR_DEVICE, "device error word " + std::to_string(s->h_st->error));
    return KC_OK;
}

int kc_render_pending(const kc_synth* s) { return s && s->pending ? 1 : 0; }

int kc_render(kc_synth* s, float* out, size_t n) {
    if (!s || !out) return fail(KC_ERR_INVALID, "null argument");
    const size_t samples = (size_t)s->cfg.block_frames * 2;
    if (n != samples) return fail(KC_ERR_INVALID, "output must be block_frames * 2 samples");
    if (int rc = kc_render_begin(s)) return rc;
    return kc_render_end(s, out, n);
}

int kc_stats(kc_synth* s, kc_block_stats* out) {
    if (!s || !out) return fail(KC_ERR_INVALID, "null argument");
    *out = s->stats;
    return KC_OK;
}

const char* kc_name(const kc_synth*) { return "cuda-sm100a"; }

int kc_set_profile(kc_synth* s, int on) {
    if (!s) return fail(KC_ERR_INVALID, "null synth");
    cudaSetDevice(s->device);
    KC_CUDA(cudaStreamSynchronize(s->stream));
    drain_timings(s);
    s->profile = on != 0;
    s->have_timings = false;
    for (auto& t : s->total_ms) t = 0.0;
    s->total_blocks = 0;
    return KC_OK;
}

int kc_timings_total(kc_synth* s, double* ms, size_t cap, uint64_t* blocks) {
    if (!s || !blocks) return fail(KC_ERR_INVALID, "null argument");
    for (size_t i = 0; i < std::min<size_t>(cap, kc::N_TIMERS); ++i) ms[i] = s->total_ms[i];
    *blocks = s->total_blocks;
    return KC_OK;
}

int kc_timings(kc_synth* s, const char** names, double* ms, size_t cap, size_t* n) {
    if (!s || !n) return fail(KC_ERR_INVALID, "null argument");
    *n = 0;
    if (!s->have_timings) return KC_OK;
    const size_t k = std::min<size_t>(cap, kc::N_TIMERS);
    for (size_t i = 0; i < k; ++i) {
        if (names) names[i] = kPassNames[i];
        if (ms) ms[i] = s->last_ms[i];
    }
    *n = k;
    return KC_OK;
}

int kc_enqueue_block_device(kc_synth* s, const uint32_t* d_gates, const uint32_t* d_chan, int bend, int gain,
                            int variant, const kc_spawn_cmd* d_cmds, uint32_t n_cmds, float* d_out) {
    if (!s || !d_gates || !d_chan || !d_out || (n_cmds && !d_cmds)) return fail(KC_ERR_INVALID, "null argument");
    cudaSetDevice(s->device);
    return enqueue_block(s, d_gates, d_chan, bend != 0, gain != 0, variant != 0, d_cmds, n_cmds, d_out);
}

int kc_synchronize(kc_synth* s) {
    if (!s) return fail(KC_ERR_INVALID, "null synth");
    cudaSetDevice(s->device);
    KC_CUDA(cudaMemcpyAsync(s->h_st, s->st, sizeof(DevState), cudaMemcpyDeviceToHost, s->stream));
    KC_CUDA(cudaStreamSynchronize(s->stream));
    drain_timings(s);
    s->stats.active_voices = s->h_st->live;
    if (s->h_st->all_tiles) s->hot_tiles = (uint64_t)s->h_st->hot_tiles * 2u >= s->h_st->all_tiles;
    s->stats.stolen = s->h_st->stolen;
    s->stats.dropped = s->h_st->dropped;
    uint32_t pb = s->h_st->peak_bits;
    std::memcpy(&s->stats.peak, &pb, 4);
    if (s->h_st->error) return fail(KC_ERR_DEVICE, "device error word " + std::to_string(s->h_st->error));
    return KC_OK;
}

void* kc_stream(kc_synth* s) { return s ? (void*)s->stream : nullptr; }

int kc_block_launches(kc_synth* s, uint32_t* out) {
    if (!s || !out) return fail(KC_ERR_INVALID, "null argument");
    *out = launches_for(s, true);
    return KC_OK;
}

int kc_device_memory(int device, uint64_t* free_bytes, uint64_t* total_bytes) {
    if (!free_bytes || !total_bytes) return fail(KC_ERR_INVALID, "null argument");
    size_t f = 0, t = 0;
    KC_CUDA(cudaSetDevice(device));
    KC_CUDA(cudaMemGetInfo(&f, &t));
    *free_bytes = f;
    *total_bytes = t;
    return KC_OK;
}

int kc_last_block_voices(kc_synth* s, uint32_t* rendered) {
    if (!s || !rendered) return fail(KC_ERR_INVALID, "null argument");
    *rendered = s->h_st->live_render;
    return KC_OK;
}

int kc_launches_total(kc_synth* s, uint64_t* out) {
    if (!s || !out) return fail(KC_ERR_INVALID, "null argument");
    *out = s->launches;
    return KC_OK;
}

int kc_last_block_tiles(kc_synth* s, uint32_t* hot_tiles, uint32_t* all_tiles) {
    if (!s || !hot_tiles || !all_tiles) return fail(KC_ERR_INVALID, "null argument");
    *hot_tiles = s->h_st->hot_tiles;
    *all_tiles = s->h_st->all_tiles;
    return KC_OK;
}

uint64_t kc_synth_device_bytes(const kc_synth* s) {
    if (!s) return 0;
    return footprint(s->cfg, s->cap, s->pcm_len, s->params_per, s->n_slots, s->tiles, s->cmds_cap,
                     s->partial_slices, s->compact_ctas);
}

int kc_estimate_device_bytes(const kc_config* cfg, uint64_t pool_len, uint32_t params_len, uint64_t* bytes) {
    if (!cfg || !bytes) return fail(KC_ERR_INVALID, "null argument");
    *bytes = 0;
    if (int rc = validate(*cfg)) return rc;
    const uint64_t slots = kc_pool_slots(cfg);
    if (slots > 0x7FFFFFE0ull) return fail(KC_ERR_INVALID, "pool slots exceed 2^31");
    int sms = 0, per_sm = 0;
    KC_CUDA(cudaSetDevice((int)cfg->device));
    KC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, (int)cfg->device));
    const uint32_t vpl = cfg->voices_per_lane == 2 ? 2u : 1u;
    if (int rc = render_occupancy(*cfg, vpl, (size_t)RENDER_WARPS * SM_WARP * sizeof(float), &per_sm)) return rc;
    const uint64_t cap = (slots + 31) & ~31ull;
    const uint32_t render_warps = (uint32_t)(sms * per_sm) * RENDER_WARPS;
    // The spawn buffer grows with the largest block; admission never hands a
    // block more commands than the pool has slots.
    *bytes = footprint(*cfg, cap, pool_len, params_len, cfg->max_param_variants,
                       cfg->block_frames / cfg->gate_frames, (uint32_t)std::max<uint64_t>(slots, 4096),
                       partial_slices_of(cap, vpl, render_warps), (uint32_t)sms * 2);
    return KC_OK;
}

int kc_read_pool(kc_synth* s, uint32_t* fields, size_t cap_words, uint32_t* live) {
    if (!s || !live) return fail(KC_ERR_INVALID, "null argument");
    cudaSetDevice(s->device);
    KC_CUDA(cudaStreamSynchronize(s->stream));
    DevState h{};
    KC_CUDA(cudaMemcpy(&h, s->st, sizeof(h), cudaMemcpyDeviceToHost));
    *live = h.live;
    if (cap_words < (size_t)h.live * VOICE_FIELDS) return fail(KC_ERR_INVALID, "buffer too small");
    if (!h.live) return KC_OK;
    KC_CUDA(cudaMemcpy2D(fields, (size_t)h.live * 4, s->pool[s->parity], (size_t)s->cap * 4, (size_t)h.live * 4,
                         VOICE_FIELDS, cudaMemcpyDeviceToHost));
    return KC_OK;
}

}  // extern "C"
