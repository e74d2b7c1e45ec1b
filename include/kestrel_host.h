/*
 * kestrel_host.h -- C ABI of the host side that feeds the backend.
 *
 * Kestrel's driver (src/driver.rs) is the *caller* of the Backend trait: it
 * owns the bank, the MIDI timeline, the note-off gate table, the channel
 * controller table and admission, and hands the backend one block of inputs
 * at a time. It is branchy table work that the reference keeps on the CPU by
 * design (src/bank.rs:1-6), and so does this library. It is a C++17
 * restatement of:
 *
 *   src/bank.rs     Region/RegionParams, build_voice, make_params, the
 *                   admission preview tables, params variants
 *   src/sf2.rs      the RIFF walk, preset/instrument flattening
 *                   (build_region) and build_pool
 *   src/sfz.rs      SFZ instruments, with the WAV reader of src/wav.rs
 *   src/resample.rs the load-time 32-tap x 512-phase Blackman sinc
 *   src/voice.rs    GateTable, ChannelTable, admit_key/mix48/rank_gain_q
 *   src/midi.rs     MidiStream (standard MIDI files) and TempoClock
 *   src/driver.rs   next_block: events, admission (strata ranking),
 *                   materialise, controllers, LFO modulation
 *   src/testkit.rs  the synthetic waveforms the seeded banks are built
 *                   from, and the SF2 writer's layout
 *   src/limiter.rs, src/wav.rs  the output stage
 *
 * A soundfont is a SoundFont 2 file, an SFZ instrument, or a seeded synthetic
 * bank (written as SF2 and loaded by the same code); MIDI is a standard MIDI file
 * or a seeded synthetic event stream with the shapes of the benchmark
 * configurations. The block inputs it produces are the backend's arguments
 * verbatim: kc_spawn_cmd records, gate rows, channel rows.
 */
#ifndef KESTREL_HOST_H
#define KESTREL_HOST_H

#include <stddef.h>
#include <stdint.h>

#include "kestrel_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Config fields the host side reads beyond kc_config (src/config.rs). */
typedef struct kh_options {
    float master_volume;            /* 1.0 */
    uint32_t filter_enabled;        /* 1 */
    uint32_t max_layers;            /* 16 */
    uint32_t default_channel_volume;/* 127 */
    uint32_t resample_pool;         /* 1: rebuild the pool at the output rate */
    uint32_t read_ahead;            /* 1: the driver's event source (the synthetic
                                       stream or the MIDI file) runs on its own
                                       thread, ahead of the driver; the events
                                       are the same */
    uint64_t sample_pool_budget;    /* bytes, 2 GiB */
} kh_options;

void kh_options_default(kh_options* o);

/* ---- synthetic soundfonts ------------------------------------------------ */

/* The seeded synthetic banks of the benchmark configurations: `presets`
 * presets over one instrument of 128 zones (zone k plays key k from sample k,
 * root k). Sample k is `sample_frames` frames at `sample_rate` Hz: a sine at
 * the key's pitch plus white noise, looped over its last `loop_frames` frames.
 * Preset 0 uses the base envelope/filter generators below; with
 * `random_generators` every other preset draws its own (seeded), held as
 * preset-level generator offsets. */
typedef struct kh_synth_bank_spec {
    uint32_t presets;            /* 1 or 128 */
    uint32_t sample_frames;      /* 32768 */
    uint32_t sample_rate;        /* 44100 */
    uint32_t loop_frames;        /* 8192 */
    float amplitude;             /* 0.5 */
    float noise;                 /* 0.01 (1% white noise) */
    int16_t attack_tc;           /* -9172: 5 ms */
    int16_t decay_tc;            /* -2786: 200 ms */
    int16_t sustain_cb;          /* 60: -6 dB */
    int16_t release_tc;          /* -2084: 300 ms */
    int16_t filter_fc_cents;     /* 11913: 8 kHz */
    int16_t filter_q_cb;         /* 30: Q 1 */
    uint32_t random_generators;  /* 0/1 */
    uint64_t seed;
} kh_synth_bank_spec;

void kh_synth_bank_spec_default(kh_synth_bank_spec* s);

typedef struct kh_bank kh_bank;

kh_bank* kh_bank_synthetic(const kh_synth_bank_spec* spec, const kc_config* cfg,
                           const kh_options* opt);
/* sf2::load (src/sf2.rs:221-505): a SoundFont 2 file. Only the samples the
 * presets use are read; the pool is resampled to the output rate (halved
 * until it fits options.sample_pool_budget). Null, with kh_last_error set,
 * when the file is not a usable soundfont. The synthetic banks above are the
 * same loader run over the bytes kh_sf2_write_synthetic writes. */
kh_bank* kh_bank_open_sf2(const char* path, const kc_config* cfg, const kh_options* opt);
/* sfz::load (src/sfz.rs:262-415): an SFZ instrument and the WAV files it
 * names (8/16/24/32-bit PCM, 32/64-bit float; loop points, root key and
 * tuning from the smpl chunk, src/wav.rs:160-356), as one preset. Stereo
 * samples become two regions panned hard left and right. */
kh_bank* kh_bank_open_sfz(const char* path, const kc_config* cfg, const kh_options* opt);
/* load_bank (src/lib.rs:32-48): .sf2 / .sf3 / .sfbk or .sfz, by extension. */
kh_bank* kh_bank_open(const char* path, const kc_config* cfg, const kh_options* opt);
/* The loader's warnings, one per line (unreadable samples; unsupported SFZ
 * opcodes with their counts); empty when there were none. */
const char* kh_bank_report(const kh_bank* b);
/* SFZ's note names (`c4` = 60, `c#4`, `eb3`, `c-1`); 0 when `s` is one. */
int kh_sfz_note_name(const char* s, int32_t* out);
/* Where an SFZ opcode value ends in the text after its `=`. */
size_t kh_sfz_value_end(const char* s);
/* The synthetic bank of `spec` as a SoundFont 2 file, in the test kit's
 * layout (src/testkit.rs:173-318; the generate-assets step). */
int kh_sf2_write_synthetic(const kh_synth_bank_spec* spec, const char* path);
void kh_bank_destroy(kh_bank* b);
/* Views into the bank; valid until kh_bank_destroy. */
int kh_bank_pool(const kh_bank* b, const int16_t** pool, uint64_t* len);
int kh_bank_params(const kh_bank* b, const kc_region_params** params, uint32_t* len);
uint32_t kh_bank_regions(const kh_bank* b);
uint32_t kh_bank_presets(const kh_bank* b);
uint32_t kh_bank_max_sample_len(const kh_bank* b);
uint32_t kh_bank_pool_rate(const kh_bank* b);
/* Per entry of the variant-0 params table: the cutoff (Hz) and Q (cB) its
 * lowpass was designed from and whether the filter is on (make_params,
 * src/bank.rs:918-938). Each array holds kh_bank_params' length. */
int kh_bank_filter_inputs(const kh_bank* b, float* fc_hz, float* q_cb, uint8_t* on, uint32_t n);

/* What the loader made of a soundfont: bank::Region (src/bank.rs:56-160),
 * bank::SampleInfo (src/bank.rs:34-54) and the presets' region lists. */
typedef struct kh_region_info {
    uint32_t sample;                /* index into the pool's samples */
    uint8_t key_lo, key_hi, vel_lo, vel_hi;
    int16_t root_key_override, fixed_key, fixed_vel;
    int16_t coarse_tune, fine_tune, scale_tuning;
    int16_t keynum_to_hold, keynum_to_decay;
    uint8_t loop_mode;              /* 0 none, 1 continuous, 2 until release */
    uint8_t exclusive_class;
    float attenuation_cb, pan;
    int32_t addr_start, addr_end, addr_loop_start, addr_loop_end;
    float delay, attack, hold, decay, sustain, release;
    float filter_fc_cents, filter_q_cb;
} kh_region_info;
typedef struct kh_sample_info {
    uint32_t start, len, loop_start, loop_end, rate;
    uint32_t root_key;
    float correction_cents, resample_ratio;
} kh_sample_info;
uint32_t kh_bank_samples(const kh_bank* b);
int kh_bank_region_info(const kh_bank* b, uint32_t i, kh_region_info* out);
int kh_bank_sample_info(const kh_bank* b, uint32_t i, kh_sample_info* out);
/* Preset i's bank and program numbers and region count; `regions` (when
 * not null) receives up to `cap` of its region indexes. */
int kh_bank_preset_info(const kh_bank* b, uint32_t i, uint16_t* bank, uint16_t* program,
                        uint32_t* n_regions, uint32_t* regions, uint32_t cap);

/* ---- synthetic MIDI ------------------------------------------------------ */

/* A seeded event stream with the shapes of the benchmark configurations:
 * Poisson onsets (optionally a share packed into 1 ms clusters), uniform keys
 * and velocities, log-normal durations, optional pitch-bend/CC7/CC11 curves
 * every `cc_period_ms` per channel and program changes every
 * `program_period_s` per channel. Events are produced lazily in tick order, so
 * a 200M-note stream never sits in memory. */
typedef struct kh_midi_spec {
    uint64_t notes;
    double seconds;
    uint32_t channels;           /* 16 */
    uint32_t key_lo, key_hi;     /* 21, 108 */
    uint32_t vel_lo, vel_hi;     /* 1, 127 */
    double dur_median_s;         /* 0.150 */
    double dur_sigma;            /* 1.0 */
    double cluster_share;        /* 0: no clusters; 0.6 for the black-MIDI config */
    uint32_t cluster_lo, cluster_hi; /* notes per 1 ms cluster */
    double cc_period_ms;         /* 0: no controller curves; 10 for config 2 */
    double program_period_s;     /* 0: every channel stays on program 0 */
    uint32_t programs;           /* presets to spread program changes over */
    uint32_t ppq;                /* ticks per quarter note, 9600 */
    uint64_t seed;
} kh_midi_spec;

void kh_midi_spec_default(kh_midi_spec* s);

/* ---- standard MIDI files (src/midi.rs) ------------------------------------ */

/* A standard MIDI file read as one tick-ordered event stream: every track
 * read through its own 256 KiB window and merged by (tick, track index)
 * (MidiStream, src/midi.rs:239-374). For tests and tools; the driver opens
 * files itself (kh_driver_open_smf). */
typedef struct kh_smf kh_smf;
#define KH_EV_NOTE_ON 0u
#define KH_EV_NOTE_OFF 1u
#define KH_EV_CC 2u
#define KH_EV_PROGRAM 3u
#define KH_EV_PITCH_BEND 4u
#define KH_EV_TEMPO 5u
#define KH_EV_OTHER 6u
kh_smf* kh_smf_open(const char* path);
void kh_smf_close(kh_smf* m);
/* format, track count; ppq, or 0 with the SMPTE frames per second and ticks
 * per frame. */
int kh_smf_info(const kh_smf* m, uint16_t* format, uint16_t* tracks, uint32_t* ppq, uint8_t* fps,
                uint8_t* ticks_per_frame);
/* The next event: 1, or 0 at the end. a/b are key/velocity (notes), number/
 * value (CC), program; bend is -8192..8191; tempo in microseconds per quarter. */
int kh_smf_next(kh_smf* m, uint64_t* tick, uint32_t* type, uint8_t* ch, uint8_t* a, uint8_t* b, int16_t* bend,
                uint32_t* tempo);
/* Write the synthetic stream of `spec` (up to max_events events, 0: all) as
 * a format-1 SMF of one track at the spec's ppq, full status bytes, the way
 * MidiWriter does (src/midi.rs:439-506). */
int kh_midi_write_synthetic(const kh_midi_spec* spec, const char* path, uint64_t max_events);

/* ---- the driver ---------------------------------------------------------- */

typedef struct kh_driver kh_driver;

/* One block of backend inputs, produced by kh_driver_prepare. The pointers
 * stay valid until the next prepare call. */
typedef struct kh_block {
    const uint32_t* gates;        /* tiles * 2048 */
    size_t n_gates;
    const uint32_t* chan;         /* tiles * 64 */
    size_t n_chan;
    int bend, gain, variant;      /* set_channels flags */
    const kc_spawn_cmd* cmds;     /* admitted and materialised, candidate order */
    size_t n_cmds;
    uint32_t n_variants;          /* params variants to install first (kh_driver_variant) */
    uint32_t live;                /* voices alive when admission ran */
    uint32_t want;                /* candidates queued */
    uint32_t take;                /* candidates admitted */
    uint64_t block_index;
    uint64_t notes;               /* note-ons handled so far */
    uint64_t want_energy;         /* summed opening amplitude (15-bit rank gains) of the
                                     queued layers, and of the admitted ones */
    uint64_t take_energy;         /* (DriverStats::last_want/take_energy, src/driver.rs:178-182) */
} kh_block;

kh_driver* kh_driver_open(const kc_config* cfg, const kh_options* opt, const kh_bank* bank,
                          const kh_midi_spec* midi);
/* The same driver reading a standard MIDI file (Driver::open,
 * src/driver.rs:343-413). Null with kh_last_error() set if it cannot be read. */
kh_driver* kh_driver_open_smf(const kc_config* cfg, const kh_options* opt, const kh_bank* bank, const char* path);
void kh_driver_destroy(kh_driver* d);

/* Driver::next_block (src/driver.rs:434-594) up to the backend's spawn:
 * drains this block's events, publishes gate and channel rows, runs admission
 * against `live` (the backend's active_voices, as the reference reads
 * backend.stats() at src/driver.rs:557), and materialises the admitted
 * voices. */
int kh_driver_prepare(kh_driver* d, uint32_t live, kh_block* out);
/* The i-th params variant to install before this block's spawn. */
int kh_driver_variant(kh_driver* d, uint32_t i, uint32_t* index, const kc_region_params** data,
                      size_t* n);
/* The rest of next_block after render (src/driver.rs:619-642): returns
 * *more = 0 once the file and its tail are done. */
int kh_driver_finish(kh_driver* d, uint64_t active_voices, int* more);

/* The same two calls split for a pipelined loop, which prepares block n + 1
 * while the backend renders block n. prepare = collect, then admit:
 * kh_driver_collect drains the block's events (gate and controller rows,
 * candidates, variants) and needs nothing from the backend; kh_driver_admit
 * runs admission against `live` and fills `out`. finish = advance, then
 * more: kh_driver_advance ends the block; kh_driver_more answers whether
 * another block follows, from the state the last admitted block left, so it
 * may be called after the next block's collect. The order
 *   collect(0) admit(0) advance  [collect(n+1) more(n) admit(n+1) advance]...
 * gives the same blocks and answers as prepare/finish, and so does admitting
 * block n + 1 before more(n) when kh_driver_admit_ready says it may. */
int kh_driver_collect(kh_driver* d);
int kh_driver_admit(kh_driver* d, uint32_t live, kh_block* out);
/* 1 when the collected block's admission does not depend on `live` (every
 * queued layer fits in what one block may steal): kh_driver_admit may then
 * run before the previous block's render has ended, with any `live` (the
 * block's `live` field then reports that value, not the pool's). */
int kh_driver_admit_ready(const kh_driver* d);
int kh_driver_advance(kh_driver* d);
int kh_driver_more(kh_driver* d, uint64_t active_voices, int* more);

const char* kh_last_error(void);

/* ---- the pieces the reference's own unit tests exercise ------------------ *
 * The gate table (src/voice.rs:212-452) on its own, and the bank's DSP
 * helpers, so the reference's in-module tests (src/voice.rs:660-766,
 * src/bank.rs:981-1035, src/resample.rs:109-171) can be restated against
 * this library. */
typedef struct kh_gates kh_gates;
kh_gates* kh_gates_new(uint32_t block_frames, uint32_t gate_frames);
void kh_gates_destroy(kh_gates* g);
void kh_gates_begin_block(kh_gates* g);
void kh_gates_end_block(kh_gates* g);
uint32_t kh_gates_note_on(kh_gates* g, uint8_t ch, uint8_t key, uint32_t frame);
void kh_gates_note_off(kh_gates* g, uint8_t ch, uint8_t key, uint32_t frame);
void kh_gates_set_sustain(kh_gates* g, uint8_t ch, int down, uint32_t frame);
void kh_gates_set_sostenuto(kh_gates* g, uint8_t ch, int down, uint32_t frame);
uint32_t kh_gates_row(const kh_gates* g, uint32_t tile, uint32_t slot);
uint32_t kh_gates_tiles(const kh_gates* g);
uint64_t kh_gates_sounding(const kh_gates* g);

float kh_velocity_atten_cb(uint8_t vel, float veltrack);
void kh_biquad_lowpass(float fc, float q_cb, float sr, float* b0, float* b1, float* a1, float* a2);
float kh_timecents_to_secs(float tc);
/* resample::resample_i16; `out` holds at least round(n * ratio) + 1 samples.
 * Returns the output length. */
size_t kh_resample_i16(const int16_t* src, size_t n, double ratio, int16_t* out, size_t cap);

/* ---- the output stage ------------------------------------------------------
 * What Driver::next_block does to the backend's block after render
 * (src/driver.rs:596-606): the configured limiter, then clamp_block. Host
 * side, on the mixed stereo block; state carries across blocks. */
#define KH_LIMITER_OFF 0u
#define KH_LIMITER_OMNI 1u       /* the OmniConverter loudness follower (src/limiter.rs:13-116) */
#define KH_LIMITER_BRICKWALL 2u  /* lookahead true-peak brickwall (src/limiter.rs:164-441), the default */

typedef struct kh_limiter kh_limiter;
/* Config defaults: mode brickwall, ceiling 0 dB, lookahead 2 ms, release
 * 60 ms, sustain 0 ms, true peak on (src/config.rs:387-393); ranges as
 * Config::validate (src/config.rs:472-494). */
kh_limiter* kh_limiter_create(uint32_t mode, uint32_t sample_rate, double ceiling_db, double lookahead_ms,
                              double release_ms, double sustain_ms, int true_peak);
void kh_limiter_destroy(kh_limiter* l);
/* Frames the brickwall delays the render by (lookahead + detector delay). */
uint32_t kh_limiter_latency(const kh_limiter* l);
/* The limiter, then clamp_block, in place on n interleaved samples. Returns
 * how many samples clamp_block had to move (Stats::clipped). */
uint64_t kh_limiter_process(kh_limiter* l, float* buf, size_t n);
/* Brickwall only: the largest detected input peak and the smallest gain. */
int kh_limiter_report(const kh_limiter* l, double* peak_in, double* min_gain);
/* clamp_block (src/limiter.rs:120-129): clamp to [-1, 1]; returns the count moved. */
uint64_t kh_clamp_block(float* buf, size_t n);

/* ---- WAV output (src/wav.rs:50-159) ---------------------------------------- */
#define KH_WAV_PCM16 0u
#define KH_WAV_FLOAT32 1u
typedef struct kh_wav kh_wav;
/* A RIFF/WAVE file with a 44-byte header whose sizes are patched at finish
 * (saturated at 4 GiB, as the reference does). */
kh_wav* kh_wav_create(const char* path, uint32_t sample_rate, uint16_t channels, uint32_t format);
/* Append n interleaved samples: f32 as is, or pcm16 as
 * round(clamp(s, -1, 1) * 32767). */
int kh_wav_write(kh_wav* w, const float* samples, size_t n);
/* Patch the header, close the file and free the writer. */
int kh_wav_finish(kh_wav* w, uint64_t* data_bytes);

/* A batch resampler the bank builder hands every sample it converts at load
 * (build_pool, src/sf2.rs:585-703) instead of running the host loop, e.g.
 * kc_resample_i16_batch on a GPU. Source i (src_len[i] frames) at ratio[i]
 * goes to dst[i], which holds dst_len[i] = max(round(src_len[i] * ratio[i]),
 * 1) frames; table[i] is that ratio's 512 x 32 f32 sinc table, phase-major,
 * built by the host (SincBank::new, src/resample.rs:18-49). It must produce
 * the host loop's output bit for bit. Returns 0 on success; on failure the
 * bank falls back to the host loop. */
typedef int (*kh_resample_fn)(void* user, uint32_t n, const int16_t* const* src, const uint32_t* src_len,
                              const double* ratio, const float* const* table, int16_t* const* dst,
                              const uint32_t* dst_len);
/* Install (or, with fn = NULL, remove) the process-wide resampler. Set it
 * before banks are built; banks built concurrently may share it. */
void kh_set_resampler(kh_resample_fn fn, void* user);
/* The sinc table the host builds for a ratio: PHASES x TAPS = 512 x 32 f32. */
int kh_sinc_table(double ratio, float* out, size_t cap);
uint64_t kh_mix48(uint64_t index);
uint64_t kh_rank_gain_q(float gain_l, float gain_r);

#ifdef __cplusplus
}
#endif

#endif /* KESTREL_HOST_H */
