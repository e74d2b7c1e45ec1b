// synth_impl.cuh -- the context object behind kc_synth, shared by the files
// of this library that drive contexts (synth.cu, batch.cu). Not installed.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "common.cuh"
#include "pool_ops.cuh"
#include "render.cuh"

namespace kc {
constexpr int N_TIMERS = 5;
}  // namespace kc

struct kc_synth;
namespace kc {
// Does the next block re-sort the pool (Config::sort_voices every Nth block:
// 1 = every block, 0 = never) or only compact it? Both leave the same voices;
// the sort only orders them for the render's locality.
bool sort_this_block(const kc_synth* s);
}  // namespace kc

struct kc_synth {
    kc_config cfg{};
    int device = 0;
    int sms = 148;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr;  // the host-buffer inputs' uploads (kc_render_begin)

    uint32_t cap = 0;           // pool slots, padded to 32
    uint32_t tiles = 0;         // gate tiles per block
    uint32_t params_per = 0;    // entries per params variant
    uint32_t n_slots = 0;       // params variant slots
    uint64_t pcm_len = 0;
    uint32_t n_regions = 0, max_sample_len = 0;
    kc::SortLayout sort{};

    // device buffers
    uint32_t* pool[2] = {nullptr, nullptr};
    int parity = 0;
    int16_t* pcm = nullptr;
    float* pcmf = nullptr;      // the pool converted to f32 once (k_convert_pool)
    float2* pcmp = nullptr;     // per frame: (tap, (next tap - tap) * 2^-32), the fractional path's taps
    kc_region_params* params = nullptr;
    uint32_t* gates = nullptr;
    uint32_t* chan = nullptr;
    kc_spawn_cmd* cmds = nullptr;
    uint32_t cmds_cap = 0;
    float* out = nullptr;
    float* partial = nullptr;
    float* partial_c = nullptr;
    kc::DevState* st = nullptr;
    kc::BlockCtl* ctl = nullptr;
    uint32_t* sel_hist = nullptr;
    uint32_t* counts = nullptr;
    uint32_t* total = nullptr;
    uint32_t* sort_totals = nullptr;  // per-digit totals of the pool-sort pass in flight (zero between passes)
    uint32_t* keys[2] = {nullptr, nullptr};
    uint32_t* idx[2] = {nullptr, nullptr};

    // launch geometry
    uint32_t render_ctas = 0, render_warps = 0;
    uint32_t partial_slices = 0; // partial-mix slices allocated
    uint32_t vpl = 1;           // render voices per lane
    uint32_t radix = 8;         // pool-sort digit width (bits)
    size_t render_smem = 0;
    uint32_t pool_ctas = 0;     // grid-stride passes
    uint32_t compact_ctas = 0;  // chunked passes (compaction, sort)

    // pinned host staging
    uint32_t* h_gates = nullptr;
    uint32_t* h_chan = nullptr;
    kc_spawn_cmd* h_cmds = nullptr;
    uint32_t h_cmds_cap = 0;
    float* h_out = nullptr;
    kc::DevState* h_st = nullptr;

    uint32_t want = 0;
    bool bend = false, gain = false, variant = false;
    // A block begun with kc_render_begin and not yet ended. `ev_inputs` is
    // recorded once the block's staged inputs have been copied to the
    // device; the staging writers wait on it before overwriting them.
    bool pending = false;
    cudaEvent_t ev_inputs = nullptr;
    // Render with 32-frame hot tiles: set when most of the last block read
    // back ran on a hot path (unit, integral or fractional step).
    bool hot_tiles = false;

    // Blocks enqueued on this context (its own render or a batch's), which
    // times the pool sort's interval, and kernel launches its renders enqueued.
    uint64_t blocks = 0;
    uint64_t launches = 0;

    // host mirror of BlockStats
    kc_block_stats stats{};

    bool profile = false;
    cudaEvent_t ev[kc::N_TIMERS + 1] = {};
    double last_ms[kc::N_TIMERS] = {};
    bool have_timings = false;
    // Profiling over many blocks in flight: one event set per enqueued block,
    // read back at the next synchronisation.
    std::vector<std::vector<cudaEvent_t>> ring;
    size_t ring_pending = 0;
    double total_ms[kc::N_TIMERS] = {};
    uint64_t total_blocks = 0;
};

namespace kc {
inline bool sort_this_block(const kc_synth* s) {
    return s->cfg.sort_voices != 0 && s->blocks % s->cfg.sort_voices == 0;
}

// The pool sort's layout for the block being enqueued: `chan` is its channel
// rows when bend rows are on (the predicted phase reads the bend of their last
// tile), else null.
inline SortLayout block_sort_layout(const kc_synth* s, const uint32_t* chan) {
    SortLayout L = s->sort;
    L.chan = chan;
    L.last_tile = s->tiles - 1u;
    return L;
}
}  // namespace kc
