/*
 * oracle.h -- CPU restatement of Kestrel's reference CPU backend.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker the CUDA backend is
 * compared against (tests/, __graft_entry__.smoke(), and the cpu_baseline /
 * --impl reference legs of bench.py). No product code path may link or call
 * it. It restates src/cpu.rs statement for statement (plus the config.rs
 * arithmetic it uses); see oracle/cpu_synth.cpp for the per-function citations.
 *
 * Parity pinning: the reference ships no golden vectors for this path (its
 * tests/ directory is git-ignored, src/README.md:33-39), so this restatement
 * is pinned against the reference's own in-module known-answer tests
 * (src/fixed.rs:116-167, src/voice.rs:660-766, src/bank.rs:981-1035,
 * src/resample.rs:109-171) and against analytic known answers (a looped sine
 * with an instant envelope renders to exactly the sample, src/testkit.rs:318).
 * The Rust crate itself cannot be built here (no cargo/rustc), so block-level
 * parity with the Rust binary is unpinned beyond those.
 */
#ifndef KESTREL_ORACLE_H
#define KESTREL_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#include "../include/kestrel_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ko_synth ko_synth;

ko_synth* ko_create(const kc_config* cfg, const int16_t* pool, uint64_t pool_len,
                    const kc_region_params* params, uint32_t params_len);
void ko_destroy(ko_synth* s);
int ko_set_gates(ko_synth* s, const uint32_t* rows, size_t n);
int ko_set_channels(ko_synth* s, const uint32_t* rows, size_t n, int bend, int gain,
                    int variant);
int ko_set_params_variant(ko_synth* s, uint32_t index, const kc_region_params* data,
                          size_t n);
int ko_spawn(ko_synth* s, const kc_spawn_cmd* cmds, size_t n);
/* Render one block. `mix64` (optional, block_frames*2 doubles) receives the
 * f64 accumulator before it is narrowed to f32. `threads` > 1 splits the voice
 * loop into contiguous chunks, each with its own f64 accumulator, summed in
 * chunk order: a timing aid for the CPU baseline, not bit-identical to 1. */
int ko_render(ko_synth* s, float* out, size_t n, double* mix64, int threads);
int ko_stats(const ko_synth* s, kc_block_stats* out);
/* Same layout as kc_read_pool: 24 fields, field-major, stride *live. */
int ko_read_pool(const ko_synth* s, uint32_t* fields, size_t cap_words, uint32_t* live);
/* Replace the pool with `live` voices in that layout (a pool read from
 * another backend between blocks) and set the cumulative counters. Lets a
 * test hand a device context's steady state to the oracle and compare the
 * next block at full size. */
int ko_load_pool(ko_synth* s, const uint32_t* fields, uint32_t live, uint64_t stolen, uint64_t dropped);

/* config.rs arithmetic, restated for the tests. */
uint32_t ko_max_steal(const kc_config* cfg);
uint32_t ko_steal_span(const kc_config* cfg);
uint32_t ko_pool_slots(const kc_config* cfg);
uint32_t ko_admit_take(const kc_config* cfg, uint32_t live, uint32_t queued);

/* fixed.rs, restated for the tests. */
uint64_t ko_fixed_from_f64(double v);
uint64_t ko_fixed_scale(uint64_t v, uint32_t factor);
uint32_t ko_bend_factor(double semitones);
float ko_catmull_rom(float sm1, float s0, float s1, float s2, float t);

#ifdef __cplusplus
}
#endif

#endif
