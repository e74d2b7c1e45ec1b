/*
 * kestrel_serve.h -- C ABI of the render server.
 *
 * No counterpart in the reference, which renders one MIDI file per process
 * (src/bin/kestrel.rs). A server takes a list of render jobs -- each its own
 * config, seeded synthetic soundfont and MIDI stream, with an arrival time --
 * and runs them to completion on one GPU in one of two modes:
 *
 *   KS_MODE_BATCHED     continuous batching: jobs are admitted as they arrive
 *                       while their estimated device bytes fit the VRAM budget
 *                       and a batch slot is free; every resident job's voice
 *                       pool and envelopes stay on the device, and each step
 *                       renders one block of every resident job through one
 *                       kc_batch_render (one launch sequence for all jobs).
 *                       A pool of host threads builds arriving jobs' banks and
 *                       drivers and prepares each step's block inputs; a job
 *                       that finishes frees its slot and memory at once.
 *   KS_MODE_SEQUENTIAL  the plain path: one job at a time in arrival order,
 *                       each block through kc_render on one thread, as a user
 *                       of the reference renders files one after another.
 *   KS_MODE_PARALLEL    the plain path on host_threads threads at once: each
 *                       thread takes the next job in arrival order and
 *                       renders it to completion through kc_render on its own
 *                       context and stream, admitted by the same VRAM budget.
 *                       Many contexts share the device, none batched.
 *
 * Results report each job's arrival, admission, first block and completion on
 * the server clock, its voice-samples, and a 64-bit hash of its output bytes:
 * a job's hash is the same in either mode and whatever else runs beside it
 * (kc_batch_render is byte-identical to kc_render per job).
 */
#ifndef KESTREL_SERVE_H
#define KESTREL_SERVE_H

#include <stddef.h>
#include <stdint.h>

#include "kestrel_cuda.h"
#include "kestrel_host.h"

#ifdef __cplusplus
extern "C" {
#endif

#define KS_MODE_BATCHED 0u
#define KS_MODE_SEQUENTIAL 1u
#define KS_MODE_PARALLEL 2u

typedef struct ks_job_spec {
    double arrival_s;            /* seconds after the server starts */
    kc_config cfg;               /* its backend config (pool size, rules) */
    kh_options opt;
    kh_synth_bank_spec bank;     /* its own seeded soundfont */
    kh_midi_spec midi;           /* its MIDI stream */
    uint64_t max_blocks;         /* 0: until the file and its tail are done */
} ks_job_spec;

/* Called once per rendered block of a job, from a server thread (calls for
 * one job are in block order and never concurrent; calls for different jobs
 * may be). */
typedef void (*ks_block_fn)(void* user, uint32_t job, uint64_t block, const float* out, size_t n);

typedef struct ks_server_config {
    uint32_t mode;               /* KS_MODE_* */
    uint32_t device;
    uint32_t max_jobs;           /* resident jobs (batch width), 1..=1024 */
    uint32_t host_threads;       /* 0: one per hardware thread */
    uint64_t vram_budget;        /* bytes for resident jobs; 0: free memory at start minus 8 GiB */
    uint32_t use_graph;          /* replay the batch's captured graph */
    uint32_t realtime_arrivals;  /* 1: a job is visible at arrival_s on the wall clock; 0: all at start */
    ks_block_fn on_block;        /* optional */
    void* user;
    uint32_t autotune;           /* 1: before serving, run ks_autotune (voices per lane, sort digit
                                    width) on the job with the largest voice pool and give every
                                    job the winner */
    uint32_t device_resample;    /* 1 (default): banks built during the run convert their samples
                                    on the server's GPU (kc_resample_i16_batch); 0: host loop */
    uint32_t reserved[6];
} ks_server_config;

typedef struct ks_job_result {
    double arrival_s;            /* server clock, seconds */
    double admit_s;              /* resident on the device */
    double first_block_s;
    double done_s;
    double setup_s;              /* host time building its bank and driver */
    uint64_t blocks;
    uint64_t voice_samples;      /* sum over blocks of voices rendered x block_frames */
    uint64_t out_hash;           /* hash of the output bytes, block by block */
    uint64_t device_bytes;       /* what admission charged */
    uint32_t max_live;
    float peak;                  /* max block peak */
    int status;                  /* KC_OK or the failing call's status */
    uint32_t pad;
} ks_job_result;

typedef struct ks_run_stats {
    double wall_s;               /* server start to the last completion */
    double gpu_ms;               /* device time of the render launch sequences: summed over batch
                                    steps (batched) or over every job's blocks (sequential,
                                    parallel; in parallel mode the jobs' blocks overlap) */
    double setup_s;              /* host time spent on banks and drivers, summed */
    uint64_t voice_samples;
    uint64_t job_blocks;
    uint64_t steps;              /* batch steps, or blocks in sequential mode */
    uint64_t peak_device_bytes;  /* largest admitted total */
    uint32_t max_resident;
    uint32_t host_threads;
    uint32_t tuned_voices_per_lane;  /* the autotuner's choice (0: not tuned) */
    uint32_t tuned_sort_radix_bits;
    double tune_s;                   /* wall seconds the autotuner took (not in wall_s) */
} ks_run_stats;

/* ---- autotuner ------------------------------------------------------------
 * Picks voices per lane, pool-sort digit width and (when allowed) block
 * length for a job. For each block length it renders the job's first
 * preroll_blocks blocks, snapshots the context, records the next timed_blocks
 * blocks' inputs, then replays them on a clone of the snapshot for every
 * (voices per lane, digit width) candidate (kc_synth_clone_config) and times
 * the replays on the device. The fastest candidate by voice-samples per
 * device second wins. Voices per lane and digit width never change the voice
 * state a block leaves; block length changes when blocks are admitted and is
 * tried only when the caller lists lengths. */
typedef struct ks_tune_space {
    uint32_t voices_per_lane_mask; /* bit v-1: try v voices per lane (v = 1, 2); 0 = both */
    uint32_t radix_mask;           /* bit r: try r-bit sort digits (4..10); 0 = {6, 8, 10} */
    uint32_t block_frames[4];      /* lengths to try (0 = unused); all 0 = the job's own */
    uint32_t preroll_blocks;       /* untimed blocks before the snapshot; 0 = 16 */
    uint32_t timed_blocks;         /* replayed and timed per candidate; 0 = 4 */
    uint32_t reserved[6];
} ks_tune_space;

typedef struct ks_tune_result {
    uint32_t voices_per_lane;
    uint32_t sort_radix_bits;
    uint32_t block_frames;
    uint32_t blocks;               /* blocks timed */
    double device_ms;              /* summed pass time of the timed blocks */
    uint64_t voice_samples;        /* voices rendered x block_frames over them */
    double voice_samples_per_s;
} ks_tune_result;

/* `best` receives the job's config with the winning tunables. `results`
 * (capacity `cap`, may be NULL) receives every candidate's timing; *n the
 * number of candidates. */
int ks_autotune(const ks_job_spec* job, const ks_tune_space* space, kc_config* best, ks_tune_result* results,
                uint32_t cap, uint32_t* n);

void ks_server_config_default(ks_server_config* c);
/* Runs every job to completion. `results` holds n_jobs entries (in the order
 * of `jobs`). Returns KC_OK, or the status of a failure that stopped the
 * server (a job's own failure is recorded in its result and the rest go on). */
int ks_serve(const ks_server_config* cfg, const ks_job_spec* jobs, uint32_t n_jobs, ks_job_result* results,
             ks_run_stats* stats);
/* The output hash's step: h' = ks_hash_block(h, block bytes). Starts at 0. */
uint64_t ks_hash_block(uint64_t h, const float* out, size_t n);
const char* ks_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* KESTREL_SERVE_H */
