/*
 * kestrel_cuda.h -- C ABI of the B200 (sm_100a) synthesis backend.
 *
 * This is the drop-in boundary for Kestrel's `Backend` trait
 * (src/backend.rs:22-58). Every entry point below replaces one trait method
 * (cited per function), takes plain pointers and sizes, copies what it keeps
 * before returning, and reports failure as a non-zero status with a message
 * readable through kc_last_error(). A context is single-threaded, exactly like
 * the trait object it replaces (one driver thread, strictly sequential calls);
 * it owns one CUDA stream.
 *
 * Byte layouts of kc_spawn_cmd and kc_region_params match the reference's
 * repr(C) structs field for field, so the Rust side can pass its slices
 * straight through (bytemuck::cast_slice).
 */
#ifndef KESTREL_CUDA_H
#define KESTREL_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define KC_OK 0
#define KC_ERR_INVALID 1   /* bad argument: size, index, layout */
#define KC_ERR_CUDA 2      /* a CUDA call failed */
#define KC_ERR_OOM 3       /* device or pinned memory exhausted */
#define KC_ERR_DEVICE 4    /* a kernel reported an internal error word */

/* ---- layouts shared with the reference ---------------------------------- */

/* Envelope stages, src/voice.rs:11-15. Part of the host/device contract. */
#define KC_ENV_ATTACK 0u
#define KC_ENV_DECAY 1u
#define KC_ENV_SUSTAIN 2u
#define KC_ENV_RELEASE 3u
#define KC_ENV_DEAD 4u

/* Gate table width: 16 channels x 128 keys, src/voice.rs:18. */
#define KC_GATE_SLOTS 2048u
/* Channel controller rows, src/voice.rs:454-463. */
#define KC_BEND_CHANNELS 16u
#define KC_CHAN_FIELDS 4u
#define KC_CHAN_BEND 0u
#define KC_CHAN_GAIN_L 1u
#define KC_CHAN_GAIN_R 2u
#define KC_CHAN_VARIANT 3u

/* Voice flags, src/bank.rs:13-15; region-params flag, src/bank.rs:190. */
#define KC_VF_LOOP 1u
#define KC_VF_LOOP_UNTIL_RELEASE 2u
#define KC_RP_FILTER 1u

/* One voice's birth record. Mirrors voice::SpawnCmd (src/voice.rs:22-57):
 * 19 x 32-bit words, 76 bytes, tightly packed. */
typedef struct kc_spawn_cmd {
    uint32_t phase_lo;
    uint32_t phase_hi;
    uint32_t step_lo;
    uint32_t step_hi;
    uint32_t smp_base;
    uint32_t smp_len;
    uint32_t loop_start;
    uint32_t loop_end;
    uint32_t flags;
    uint32_t params;
    uint32_t variant;
    uint32_t region;
    uint32_t gate_slot;
    uint32_t ordinal;
    uint32_t start_rel;
    uint32_t note_id_lo;
    uint32_t note_id_hi;
    float gain_l;
    float gain_r;
} kc_spawn_cmd;

/* Per-(region, key, velocity) DSP constants. Mirrors bank::RegionParams
 * (src/bank.rs:166-188): 12 x 32-bit words, 48 bytes. */
typedef struct kc_region_params {
    float attack_rate;
    float attack_end;
    float decay_coef;
    float decay_target;
    float sustain;
    float release_coef;
    float b0;
    float b1;
    float a1;
    float a2;
    uint32_t flags;
    uint32_t pad;
} kc_region_params;

/* Mirrors backend::BlockStats (src/backend.rs:11-20). */
typedef struct kc_block_stats {
    uint64_t active_voices; /* live voices after the last compaction */
    uint64_t stolen;        /* cumulative */
    uint64_t dropped;       /* cumulative */
    float peak;             /* max |sample| of the last block */
    uint32_t pad;
} kc_block_stats;

/* Rules, src/config.rs:11-109 (the enum discriminants are the reference's). */
#define KC_INTERP_NEAREST 0u
#define KC_INTERP_LINEAR 1u
#define KC_INTERP_CUBIC 2u
#define KC_CURVE_EXPONENTIAL 0u
#define KC_CURVE_LINEAR 1u
#define KC_STEAL_OLDEST 0u
#define KC_STEAL_DROP_NEW 1u
#define KC_STEAL_QUIETEST 2u
#define KC_ADMIT_LOUDEST 0u
#define KC_ADMIT_EVEN 1u

/* Mixdown arithmetic of the stereo block. */
#define KC_MIX_F32_TREE 0u     /* fixed-order f32 tree (the reference's device form) */
#define KC_MIX_TWO_SUM 1u      /* fixed-order tree with compensated two-sum carries */
#define KC_MIX_F64 2u          /* the f32 voice terms accumulated in f64: an FP64 mix oracle on the device */

/* The subset of config::Config (src/config.rs:164-343) that the backend reads,
 * plus the backend's own tunables. Fill with kc_config_default() first. */
typedef struct kc_config {
    uint32_t sample_rate;        /* Hz, 48000 */
    uint32_t block_frames;       /* frames per render, 4096; a multiple of 16 */
    uint32_t gate_frames;        /* gate/controller tile, 32; a multiple of 16 or a divisor of 16 */
    uint32_t max_voices;         /* pool ceiling surviving a block */
    uint32_t max_steal_percent;  /* 1..=100, 25 */
    uint32_t steal_fade_frames;  /* 1..block_frames-1, 96 */
    uint32_t steal_rule;         /* KC_STEAL_*, Quietest */
    uint32_t admit_rule;         /* KC_ADMIT_*, Loudest */
    uint32_t interpolation;      /* KC_INTERP_*, Linear */
    uint32_t decay_curve;        /* KC_CURVE_*, Exponential */
    uint32_t release_curve;      /* KC_CURVE_*, Exponential */
    float env_floor;             /* 1e-5 */
    uint32_t sort_voices;        /* N > 0: re-sort the pool by (region, stage, phase) on every
                                    Nth block (1: every block, the default), compact it in
                                    place of the sort on the others; 0: never sort */
    uint32_t max_param_variants; /* params-table copies, 32 */
    uint32_t mix_mode;           /* KC_MIX_*, F32 tree */
    uint32_t strict_fp;          /* 1: no FMA contraction anywhere in the voice DSP */
    uint32_t device;             /* CUDA ordinal */
    uint32_t voices_per_lane;    /* render voices per GPU lane: 0 = default (1), 1 or 2 */
    uint32_t sort_radix_bits;    /* key bits per pool-sort pass, 4..=10; 0 = default (8). The
                                    sorted order is the same for every width. */
    uint32_t unit_tile_frames;   /* frames per render tile on the hot paths -- unit, integral
                                    and fractional steps with no envelope transition (one voice
                                    per lane, f32 tree mix): 16, 32, or 0 = chosen per block (32
                                    when the block before ran mostly on those paths). The
                                    output is the same for every choice. */
    uint32_t reserved[4];
} kc_config;

typedef struct kc_synth kc_synth;

/* Defaults of config.rs:345-409 for every field above. */
int kc_config_default(kc_config* cfg);

/* The pool size the backend allocates for a config: max_voices plus the
 * steal headroom, config.rs:542-552. */
uint32_t kc_pool_slots(const kc_config* cfg);

/* Replaces GpuSynth::new (src/gpu/mod.rs:276). Copies the i16 sample pool and
 * the variant-0 params table to the device. `n_regions` and `max_sample_len`
 * size the pool sort key exactly as SortKeyLayout::plan does
 * (src/gpu/mod.rs:77-105). */
int kc_synth_create(const kc_config* cfg, const int16_t* pool, uint64_t pool_len,
                    const kc_region_params* params, uint32_t params_len,
                    uint32_t n_regions, uint32_t max_sample_len, kc_synth** out);
void kc_synth_destroy(kc_synth* s);

/* A second context on the same device in the same state: bank, params
 * variants, voice pool and counters are copied device to device. No
 * counterpart in the reference trait; it is how a render is checkpointed or
 * forked (the benchmark forks one to replay recorded blocks from HBM). */
int kc_synth_clone(kc_synth* src, kc_synth** out);
/* The same, with other tunables: `cfg` must equal the source's config except
 * in voices_per_lane, sort_radix_bits and unit_tile_frames, which change how a block is
 * computed but not the voice state it leaves (voices per lane also changes
 * the summation order of the mix, within its tolerance). The autotuner times
 * its candidates on such clones of one pre-rolled context. */
int kc_synth_clone_config(kc_synth* src, const kc_config* cfg, kc_synth** out);

/* Backend::set_gates (src/backend.rs:23-25): tiles * KC_GATE_SLOTS words,
 * tile-major; tiles = block_frames / gate_frames. */
int kc_set_gates(kc_synth* s, const uint32_t* rows, size_t n);

/* Backend::set_channels (src/backend.rs:27-33): tiles * 16 * 4 words. */
int kc_set_channels(kc_synth* s, const uint32_t* rows, size_t n, int bend, int gain,
                    int variant);

/* Backend::set_params_variant (src/backend.rs:35-39). Index 0 is the bank's
 * own table and is left untouched, as CpuSynth does (src/cpu.rs:313-323). */
int kc_set_params_variant(kc_synth* s, uint32_t index, const kc_region_params* data,
                          size_t n);

/* Backend::spawn (src/backend.rs:41-43). The commands are validated and
 * copied; steal/drop/admit happen on the device inside the next render. A
 * refused call (a params index or gate slot out of range) leaves no commands
 * staged. */
int kc_spawn(kc_synth* s, const kc_spawn_cmd* cmds, size_t n);

/* Backend::render (src/backend.rs:45-47): `out` receives block_frames * 2
 * interleaved stereo floats. Blocks until the block is on the host. */
int kc_render(kc_synth* s, float* out, size_t n);

/* kc_render in two halves, so the caller can prepare the next block while
 * this one renders: kc_render_begin enqueues the block (the staged inputs'
 * copies, every pass, the copies back) and returns at once; kc_render_end
 * waits for it, writes `out` and updates kc_stats. kc_render is begin then
 * end. Between the two, kc_set_gates / kc_set_channels / kc_spawn may stage
 * the next block (they wait only until this block's inputs have reached the
 * device); a second begin, kc_synth_clone* and kc_batch_render are refused
 * until end. kc_stats reports the previous block until end. No counterpart
 * in the reference trait, whose render is synchronous. */
int kc_render_begin(kc_synth* s);
int kc_render_end(kc_synth* s, float* out, size_t n);
int kc_render_pending(const kc_synth* s);

/* Backend::stats (src/backend.rs:49). */
int kc_stats(kc_synth* s, kc_block_stats* out);

/* Backend::name (src/backend.rs:51). */
const char* kc_name(const kc_synth* s);

/* Backend::timings (src/backend.rs:53-57): per-pass device milliseconds of
 * the last render when timing is enabled (kc_set_profile). */
int kc_set_profile(kc_synth* s, int on);
int kc_timings(kc_synth* s, const char** names, double* ms, size_t cap, size_t* n);
/* The same passes summed over every block completed since profiling was
 * switched on (blocks enqueued back to back included), and the block count.
 * No counterpart in the reference trait. */
int kc_timings_total(kc_synth* s, double* ms, size_t cap, uint64_t* blocks);

/* Message of the last failing call on this thread ("" when none). */
const char* kc_last_error(void);

/* ---- device-resident form ---------------------------------------------- *
 * The same block with its inputs already in device memory: no host copies
 * and no synchronisation. A streaming caller (or the benchmark) stages the
 * inputs of many blocks in HBM and enqueues blocks back to back. Pointers
 * must stay valid until the block has executed (kc_synchronize). */
int kc_enqueue_block_device(kc_synth* s, const uint32_t* d_gates, const uint32_t* d_chan,
                            int bend, int gain, int variant, const kc_spawn_cmd* d_cmds,
                            uint32_t n_cmds, float* d_out);
int kc_synchronize(kc_synth* s);
/* The context's cudaStream_t, for event timing by the caller. */
void* kc_stream(kc_synth* s);
/* Number of kernel launches one block enqueues when it sorts the pool (the
 * captured graph's nodes), and the launches this context's blocks have
 * enqueued so far. */
int kc_block_launches(kc_synth* s, uint32_t* out);
int kc_launches_total(kc_synth* s, uint64_t* out);

/* ---- precision form ------------------------------------------------------ *
 * RBJ lowpass coefficients designed in FP64 on the device: `coefs` receives
 * n x (b0, b1, a1, a2) for the n (cutoff Hz, Q in centibels) pairs, with the
 * arithmetic of biquad_lowpass (src/bank.rs:956-979) carried out in double.
 * a1 and a2 are the exact design rounded once to f32; b0 is matched to them
 * (b0 = gain (1 + a1 + a2) / 4, b1 = 2 b0) so the stored filter keeps the
 * design's DC gain to within one f32 rounding. For regions with a low cutoff
 * or a high Q, where the reference's f32 design loses most of (1 - cos w0);
 * the caller patches the returned coefficients into the params table it
 * hands to kc_synth_create / kc_set_params_variant. Host buffers in and out. */
int kc_design_lowpass_f64(const float* fc_hz, const float* q_cb, uint32_t n, float sample_rate,
                          float* coefs, int device);

/* ---- load-time resampling -------------------------------------------------- *
 * SincBank::process (src/resample.rs:51-107) for a batch of samples in one
 * launch, bit-exact with the host loop: source i (src_len[i] frames) at
 * ratio[i] (output rate / input rate) goes to dst[i], which must hold
 * dst_len[i] = max(round(src_len[i] * ratio[i]), 1) frames; table[i] is that
 * ratio's 512 x 32 f32 sinc table (kh_sinc_table), built on the host so no
 * device transcendental enters the result. `device` points to the CUDA ordinal
 * (NULL: device 0). Host buffers in and out. The signature is the host
 * library's kh_resample_fn, so kh_set_resampler(kc_resample_i16_batch, &ord)
 * moves every bank's load-time conversion onto the GPU. */
int kc_resample_i16_batch(void* device, uint32_t n, const int16_t* const* src, const uint32_t* src_len,
                          const double* ratio, const float* const* table, int16_t* const* dst,
                          const uint32_t* dst_len);

/* ---- rendering without allocating --------------------------------------- *
 * No counterpart in the reference. For callers that cannot call cudaMalloc:
 * allocation can synchronise the whole device and take milliseconds, which a
 * real-time audio callback cannot wait for, and hosts that manage device
 * memory themselves (arenas, buffers fixed at start-up) hand every buffer in.
 * This renders one block of a voice pool the caller owns -- field-major, the
 * field order of kc_read_pool, `cap` words per field, `n_voices` live -- with
 * no steal, spawn or compaction, writing block_frames * 2 floats to `d_out`
 * and updating the voices' state in place. All pointers are device pointers;
 * `d_params` holds `n_slots` copies of `params_len` entries; `stream` is a
 * cudaStream_t (NULL: the legacy default stream). The call only enqueues work.
 * `d_params` and `d_chan` must be 16-byte aligned, `d_pool`, `d_gates` and
 * `d_out` 4-byte aligned (KC_ERR_INVALID otherwise). The mix is KC_MIX_F32_TREE
 * or KC_MIX_TWO_SUM; KC_MIX_F64 is refused.
 *
 * It renders from the i16 sample pool the caller passes, converting each tap,
 * and a voice that dies mid-block keeps its lane idle for the rest of the
 * block (kc_render instead renders from an f32 copy of the pool and turns
 * dead voices into silent lanes that keep their warp on the fast paths), so
 * it is slower per voice than kc_render; the output is the same within the
 * mix's tolerance. Device-side range errors are not reported: a voice whose
 * params index is past `params_len` or whose gate slot is past
 * KC_GATE_SLOTS renders with entry 0 or slot 0 (kc_render reports both as
 * KC_ERR_DEVICE; its kc_spawn refuses such commands up front).
 *
 * Its scratch (the partial-mix slices and control words) is a 32 MiB
 * file-scope device array that every GPU loading this library holds until the
 * process exits; it bounds a call to 32 voices per 2 * block_frames * 4-byte
 * slice: 32,736 voices at block_frames 4096 (16,352 with the two-sum mix).
 * Larger calls are rejected with KC_ERR_INVALID and a message naming the
 * limit. The first call on a device looks up the array's device address with
 * that device current; make that first call before any stream capture. Every
 * call on a device shares the array, so calls that overlap on the GPU race
 * and must be serialised by the caller. Nothing here calls cudaMalloc,
 * cudaFree or an allocating library routine. */
int kc_render_block_noalloc(const kc_config* cfg, uint32_t* d_pool, uint32_t cap, uint32_t n_voices,
                            const int16_t* d_pcm, uint64_t pcm_len, const kc_region_params* d_params,
                            uint32_t params_len, uint32_t n_slots, const uint32_t* d_gates,
                            const uint32_t* d_chan, int bend, int gain, int variant, float* d_out,
                            void* stream);

/* ---- batched form --------------------------------------------------------- *
 * No counterpart in the reference (it renders one file per process). One
 * kc_batch renders one block of each of up to max_jobs contexts with a single
 * launch sequence: persistent passes over every job's voices, the render one
 * persistent kernel over (job, slice) items, captured once as a CUDA graph and
 * replayed each block. Each job is an ordinary kc_synth whose inputs were set
 * with kc_set_gates / kc_set_channels / kc_spawn, exactly as before kc_render;
 * a job's output block, state and stats are byte-identical to rendering that
 * context alone with kc_render. All jobs must match the batch's device,
 * block_frames, interpolation, strict_fp, mix_mode, voices_per_lane and
 * sort_radix_bits; the steal and admit rules, pool sizes, banks and sort
 * setting are per job. */
typedef struct kc_batch_config {
    uint32_t device;
    uint32_t max_jobs;           /* 1..=1024 */
    uint32_t block_frames;
    uint32_t interpolation;      /* KC_INTERP_* */
    uint32_t strict_fp;
    uint32_t mix_mode;           /* KC_MIX_* */
    uint32_t voices_per_lane;    /* 0 or 1: one voice per lane; 2: two */
    uint32_t use_graph;          /* 1: replay a captured graph; 0: launch each pass */
    uint32_t sort_radix_bits;    /* 0 = 8, else 4..=10, as kc_config */
    uint32_t reserved[7];
} kc_batch_config;

typedef struct kc_batch kc_batch;

int kc_batch_config_default(kc_batch_config* cfg);
int kc_batch_create(const kc_batch_config* cfg, kc_batch** out);
void kc_batch_destroy(kc_batch* b);
/* One block of each listed job; outs[j] receives block_frames * 2 floats.
 * Blocks until every output is on the host. A job listed twice, a job of
 * another variant or more than max_jobs jobs is KC_ERR_INVALID. */
int kc_batch_render(kc_batch* b, kc_synth* const* jobs, uint32_t n_jobs, float* const* outs);
/* Device milliseconds of the last kc_batch_render's launch sequence. */
int kc_batch_last_ms(kc_batch* b, float* ms);
/* Device memory a context holds now, in bytes, and the most a context not yet
 * created can come to hold (its spawn buffer grown to one command per pool
 * slot, the largest block admission can produce). The serving loop admits
 * jobs by the second figure. */
uint64_t kc_synth_device_bytes(const kc_synth* s);
int kc_estimate_device_bytes(const kc_config* cfg, uint64_t pool_len, uint32_t params_len, uint64_t* bytes);
/* Free and total memory of a device, in bytes. */
int kc_device_memory(int device, uint64_t* free_bytes, uint64_t* total_bytes);
/* Voices the last completed block rendered: the live voices before its spawn
 * plus the admitted commands (the per-block term of the voice-samples
 * metric). */
int kc_last_block_voices(kc_synth* s, uint32_t* rendered);
/* How the last completed block's render ran: 16-frame warp-tiles classified
 * onto a hot path (every lane live and sounding with no envelope transition:
 * unit, integral or fractional step), and all warp-tiles. No counterpart in
 * the reference; the render picks 32-frame hot tiles when most tiles are. */
int kc_last_block_tiles(kc_synth* s, uint32_t* hot_tiles, uint32_t* all_tiles);

/* ---- inspection (tests) ------------------------------------------------- *
 * Copies the live part of the voice pool to the host as 24 SoA fields of
 * `*live` words each (field-major, stride `*live`), in the field order of
 * shaders/common.wgsl:15-43. `cap_words` bounds `fields`. */
int kc_read_pool(kc_synth* s, uint32_t* fields, size_t cap_words, uint32_t* live);

#ifdef __cplusplus
}
#endif

#endif /* KESTREL_CUDA_H */
