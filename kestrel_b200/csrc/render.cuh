// render.cuh -- the per-voice render pass and the mixdown reduction.
//
// One lane owns one voice for the whole block, its state in registers, exactly
// the reference's execution model (shaders/render.wgsl:146-421): the
// sequential parts of the DSP (32.32 phase accumulator, envelope, biquad
// memory) never round-trip through memory. What differs is how the block mix
// is formed on sm_100a:
//
//   * every 16 frames a warp writes its 32 voices x 32 output slots
//     (16 frames x 2 channels) into its own padded shared-memory tile, one
//     64-bit (left, right) store per lane and frame, and transpose-reduces
//     it: lane l sums half a frame row with four-wide loads and trades one
//     channel with its neighbour, so each lane ends with one output slot.
//     No block-wide barrier is ever taken.
//   * each warp owns a 32 KiB slice of the partial buffer (L2-resident); its
//     later voice batches accumulate into it in batch order.
//   * a second kernel folds the warps' slices in a fixed order.
//
// No float atomics anywhere, and every summation order is a function of the
// live count and the grid alone, so reruns are byte-identical.
//
// Bit-exactness: the envelope, the steal-key inputs and the 32.32 phase are
// computed with explicitly rounded intrinsics (__fadd_rn/__fmul_rn), which can
// never be contracted into an FMA, statement for statement as src/cpu.rs:
// 403-613 orders them. With STRICT the interpolation, biquad and fade are
// written the same way, so each voice's per-frame sample is bit-identical to
// the CPU restatement's f32 value; the stereo gain is a rounded product too,
// except in the factored tile (one voice per lane, f32 tree), whose fold
// fuses each gain product into the sum. Only the mix's summation (its order,
// and there its rounding) differs from the CPU's.
#pragma once

#include <cstdint>

#include "common.cuh"

namespace kc {

struct RenderArgs {
    uint32_t* pool;            // current pool, field-major
    uint32_t cap;              // field stride in words
    const int16_t* pcm;        // sample pool, i16 as the bank holds it
    const float* pcmf;         // the same pool converted once to f32 (F32 kernels), followed
                               // by ZERO_PAD zero frames (the taps of neutral lanes)
    const float2* pcmp;        // per frame of pcmf: (tap, (next tap - tap) * 2^-32) (F32 kernels)
    uint32_t pcm_len;          // frames in it
    const kc_region_params* params;  // n_slots copies of params_per
    uint32_t params_per;
    uint32_t n_slots;
    const uint32_t* gates;     // tiles x 2048
    const uint32_t* chan;      // tiles x 64
    const BlockCtl* ctl;
    DevState* st;
    float* partial;            // [warps][2 * block_frames]
    float* partial_c;          // two-sum carries, same shape (MIX two-sum only)
    uint32_t block_frames;
    uint32_t gate_frames;
    uint32_t fade;             // steal_fade_frames
    float env_floor;
    uint32_t exp_decay;
    uint32_t exp_release;
};

// Zero frames after the f32 pool: a neutral lane (below) reads its taps there.
constexpr uint32_t ZERO_PAD = 32;

// One in-bounds tap. The f32 pool holds exactly the value CpuSynth::fetch
// (src/cpu.rs:187-194) computes from the i16 sample -- v / 32767 clamped at
// -1 -- converted once when the context is created (k_convert_pool), so the
// conversion leaves the per-frame path; kernels given only the i16 pool
// (F32 = false) convert per tap.
template <bool F32>
__device__ __forceinline__ float tap(const RenderArgs& a, uint32_t i) {
    if (F32) return __ldg(a.pcmf + i);
    return fmaxf(__fmul_rn((float)__ldg(a.pcm + i), 1.0f / 32767.0f), -1.0f);
}

// Sample fetch, CpuSynth::fetch (src/cpu.rs:187-194): out-of-range reads as
// zero.
template <bool F32>
__device__ __forceinline__ float fetch_sample(const RenderArgs& a, uint32_t base, uint32_t idx) {
    const uint32_t i = base + idx;
    return i < a.pcm_len ? tap<F32>(a, i) : 0.0f;
}

// CpuSynth::advance_index (src/cpu.rs:242-259), general form in i64.
__device__ __forceinline__ uint32_t neighbour(uint32_t idx, int off, bool looping, uint32_t ls,
                                             uint32_t le, uint32_t len) {
    const int64_t raw = (int64_t)idx + off;
    if (looping) {
        if (raw >= (int64_t)le) {
            int64_t span = (int64_t)le - (int64_t)ls;
            if (span < 1) span = 1;
            return (uint32_t)((int64_t)ls + (raw - (int64_t)ls) % span);
        }
        if (raw < 0) return 0;
        return (uint32_t)raw;
    }
    int64_t hi = (int64_t)len - 1;
    int64_t r = raw < 0 ? 0 : raw;
    return (uint32_t)(r > hi ? hi : r);
}

struct VoiceRegs {
    uint64_t phase, step, base_step;
    uint32_t base, len, ls, le;
    uint32_t stage;
    float level;
    float gl, gr, bgl, bgr;
    float z1, z2;
    // region params in force: the filter; the envelope's rates and levels
    // are read from the params table where they are needed (env_params), so
    // they hold no registers through the hot tiles
    float b0, b1, a1, a2;
    bool filt;
    bool loop_en, lur;
    uint32_t params_base, variant, born, born_gate;
    uint32_t slot, ordinal, start_rel, stop_rel;
    bool neutral;   // dead, and set to contribute exactly +0 on every path (neutralize)
};

// A voice that died (or a lane past the live count) keeps its lane idle for
// the rest of the block, and an idle lane would keep the whole warp off the
// hot paths. Instead the dead voice is made neutral: level, gains, filter
// state and coefficients +0, taps at the zero pad after the f32 pool, step 0.
// Every hot-path frame then computes +0 for it (all products are +0 * +0 and
// all sums +0 + +0, whatever the path), and its phase never moves. Its stage
// stays DEAD, so compaction drops it; nothing reads a dead voice's other
// fields. Only kernels with the padded f32 pool (F32) do this.
__device__ __forceinline__ void neutralize(VoiceRegs& v, const RenderArgs& a) {
    v.level = 0.0f;
    v.gl = v.gr = v.bgl = v.bgr = 0.0f;
    v.z1 = v.z2 = 0.0f;
    v.b0 = v.b1 = v.a1 = v.a2 = 0.0f;
    v.base = a.pcm_len;
    v.phase = 0;
    v.step = v.base_step = 0;
    v.neutral = true;
}

// The voice's params entry: three float4 words (kc_region_params).
__device__ __forceinline__ const float4* params_entry(const VoiceRegs& v, const RenderArgs& a) {
    const uint32_t s = v.variant < a.n_slots ? v.variant : 0u;
    return reinterpret_cast<const float4*>(a.params + (size_t)s * a.params_per + v.params_base);
}

__device__ __forceinline__ void load_params(VoiceRegs& v, const RenderArgs& a) {
    const float4* p = params_entry(v, a);
    const float4 q1 = __ldg(p + 1), q2 = __ldg(p + 2);
    v.b0 = q1.z; v.b1 = q1.w;
    v.a1 = q2.x; v.a2 = q2.y;
    v.filt = (__float_as_uint(q2.z) & KC_RP_FILTER) != 0u;
}

// The envelope's rates and levels of the params entry in force (the table
// does not change during a block, and the entry only at a gate row's
// variant switch).
struct EnvParams {
    float ar, ae, dc, dt, sus, rc;
};
__device__ __forceinline__ EnvParams env_params(const VoiceRegs& v, const RenderArgs& a) {
    const float4* p = params_entry(v, a);
    const float4 q0 = __ldg(p);
    const float2 q1 = __ldg(reinterpret_cast<const float2*>(p + 1));
    return EnvParams{q0.x, q0.y, q0.z, q0.w, q1.x, q1.y};
}

// Per-frame voice step. Returns the filtered, faded sample y (before the
// stereo gains). Mirrors src/cpu.rs:490-601 for one frame; the caller has
// already applied the f < start_rel and DEAD gates.
template <int INTERP, bool STRICT, bool F32>
__device__ __forceinline__ float voice_frame(VoiceRegs& v, const RenderArgs& a, const EnvParams& p, uint32_t f,
                                             bool looping) {
    const uint32_t idx = (uint32_t)(v.phase >> 32);
    if (!looping && idx >= v.len) {
        v.stage = ENV_DEAD;
        return 0.0f;
    }
    // Envelope before the sample (src/cpu.rs:508-549).
    if (v.stage == ENV_ATTACK) {
        v.level = __fadd_rn(v.level, p.ar);
        if (v.level >= p.ae) {
            v.stage = ENV_DECAY;
            v.level = 1.0f;
        }
    } else if (v.stage == ENV_DECAY) {
        v.level = a.exp_decay ? __fmul_rn(v.level, p.dc) : __fsub_rn(v.level, p.dc);
        if (v.level <= p.dt) {
            if (p.sus <= a.env_floor) {
                v.stage = ENV_DEAD;
                v.level = 0.0f;
            } else {
                v.stage = ENV_SUSTAIN;
                v.level = p.sus;
            }
        }
    } else if (v.stage == ENV_RELEASE) {
        v.level = a.exp_release ? __fmul_rn(v.level, p.rc) : __fsub_rn(v.level, p.rc);
        if (v.level <= a.env_floor) {
            v.stage = ENV_DEAD;
            v.level = 0.0f;
        }
    }

    // Interpolation (src/cpu.rs:261-302).
    float s;
    const float frac = __fmul_rn(__uint2float_rn((uint32_t)v.phase), 2.3283064365386963e-10f);
    if (INTERP == KC_INTERP_NEAREST) {
        s = fetch_sample<F32>(a, v.base, idx);
    } else if (INTERP == KC_INTERP_LINEAR) {
        uint32_t i1;
        if (looping) {
            i1 = idx + 1u < v.le && idx != 0xFFFFFFFFu ? idx + 1u
                                                       : neighbour(idx, 1, true, v.ls, v.le, v.len);
        } else {
            i1 = idx + 1u < v.len ? idx + 1u : v.len - 1u;
        }
        const float s0 = fetch_sample<F32>(a, v.base, idx);
        const float s1 = fetch_sample<F32>(a, v.base, i1);
        if (STRICT) {
            s = __fadd_rn(s0, __fmul_rn(__fsub_rn(s1, s0), frac));
        } else {
            s = fmaf(s1 - s0, frac, s0);
        }
    } else {
        const uint32_t im1 = neighbour(idx, -1, looping, v.ls, v.le, v.len);
        const uint32_t i1 = neighbour(idx, 1, looping, v.ls, v.le, v.len);
        const uint32_t i2 = neighbour(idx, 2, looping, v.ls, v.le, v.len);
        const float sm1 = fetch_sample<F32>(a, v.base, im1);
        const float s0 = fetch_sample<F32>(a, v.base, idx);
        const float s1 = fetch_sample<F32>(a, v.base, i1);
        const float s2 = fetch_sample<F32>(a, v.base, i2);
        // catmull_rom, src/cpu.rs:297-302, left to right, always rounded per op.
        const float ca = __fadd_rn(__fsub_rn(__fadd_rn(__fmul_rn(-0.5f, sm1), __fmul_rn(1.5f, s0)),
                                             __fmul_rn(1.5f, s1)),
                                   __fmul_rn(0.5f, s2));
        const float cb = __fsub_rn(__fadd_rn(__fsub_rn(sm1, __fmul_rn(2.5f, s0)), __fmul_rn(2.0f, s1)),
                                   __fmul_rn(0.5f, s2));
        const float cc = __fadd_rn(__fmul_rn(-0.5f, sm1), __fmul_rn(0.5f, s1));
        s = __fadd_rn(__fmul_rn(__fadd_rn(__fmul_rn(__fadd_rn(__fmul_rn(ca, frac), cb), frac), cc), frac), s0);
    }

    const float g = fminf(v.level, 1.0f);
    const float x = __fmul_rn(s, g);
    float y = x;
    if (v.filt) {
        // Transposed direct form II, b2 == b0 (src/cpu.rs:564-572).
        if (STRICT) {
            const float bx = __fmul_rn(v.b0, x);
            y = __fadd_rn(bx, v.z1);
            v.z1 = __fadd_rn(__fsub_rn(__fmul_rn(v.b1, x), __fmul_rn(v.a1, y)), v.z2);
            v.z2 = __fsub_rn(bx, __fmul_rn(v.a2, y));
        } else {
            y = fmaf(v.b0, x, v.z1);
            v.z1 = fmaf(v.b1, x, fmaf(-v.a1, y, v.z2));
            v.z2 = fmaf(v.b0, x, -(v.a2 * y));
        }
    }
    // Steal fade after the filter (src/cpu.rs:574-587).
    if (v.stop_rel != 0u && f + 1u >= v.stop_rel) {
        const uint32_t d = f + 1u - v.stop_rel;
        if (d >= a.fade) {
            v.stage = ENV_DEAD;
            y = 0.0f;
        } else {
            y = __fmul_rn(y, __fsub_rn(1.0f, __fdiv_rn((float)d, (float)a.fade)));
        }
    }
    // Phase advance and loop wrap (src/cpu.rs:592-601).
    v.phase += v.step;
    if (looping) {
        uint32_t hi = (uint32_t)(v.phase >> 32);
        if (hi >= v.le) {
            uint32_t span = v.le - v.ls;
            if (span < 1u) span = 1u;
            hi = v.ls + (hi - v.ls) % span;
            v.phase = ((uint64_t)hi << 32) | (uint32_t)v.phase;
        }
    }
    return y;
}

// ---- the fast path -----------------------------------------------------------
// Most 16-frame tiles of most voices need none of the per-frame branches of
// voice_frame: the voice started before the tile, is not being stolen, and its
// phase neither wraps a loop nor reaches the sample end inside the tile. For
// such a tile (checked per lane, taken when the whole warp qualifies) each
// frame is straight-line code. The envelope step becomes one exactly rounded
// FMA with per-stage constants:
//   attack   level*1 + attack_rate      == level + attack_rate
//   decay    level*decay_coef + 0        == level * decay_coef   (exponential)
//            level*1 - decay_coef        == level - decay_coef   (linear)
//   sustain  level*1 + 0                 == level
//   release  like decay with release_coef
// (a single rounding of an exact product or sum is the rounding of the
// reference's own operation), and the stage test "level >= attack_end",
// "level <= decay_target", "level <= env_floor" becomes sgn*level >= thr with
// sgn = +-1 (negation is exact). A hit leaves the straight line for the
// transition code, which is the reference's statement for statement.
struct EnvStep {
    float em, ea, sgn, thr;
};

__device__ __forceinline__ EnvStep env_constants(const VoiceRegs& v, const RenderArgs& a) {
    EnvStep e;
    e.em = 1.0f; e.ea = 0.0f; e.sgn = 1.0f; e.thr = __int_as_float(0x7f800000);  // sustain: never
    if (v.stage == ENV_ATTACK || v.stage == ENV_DECAY || v.stage == ENV_RELEASE) {
        const EnvParams p = env_params(v, a);
        if (v.stage == ENV_ATTACK) {
            e.ea = p.ar; e.thr = p.ae;
        } else if (v.stage == ENV_DECAY) {
            if (a.exp_decay) e.em = p.dc; else e.ea = -p.dc;
            e.sgn = -1.0f; e.thr = -p.dt;
        } else {
            if (a.exp_release) e.em = p.rc; else e.ea = -p.rc;
            e.sgn = -1.0f; e.thr = -a.env_floor;
        }
    }
    return e;
}

// The stage transition after a threshold hit (src/cpu.rs:512-549), then the
// new stage's constants. Returns false when the voice died on this frame.
__device__ __forceinline__ bool env_transition(VoiceRegs& v, const RenderArgs& a, EnvStep& e) {
    if (v.stage == ENV_ATTACK) {
        v.stage = ENV_DECAY;
        v.level = 1.0f;
    } else if (v.stage == ENV_DECAY) {
        const float sus = env_params(v, a).sus;
        if (sus <= a.env_floor) {
            v.stage = ENV_DEAD;
            v.level = 0.0f;
        } else {
            v.stage = ENV_SUSTAIN;
            v.level = sus;
        }
    } else if (v.stage == ENV_RELEASE) {
        v.stage = ENV_DEAD;
        v.level = 0.0f;
    }
    e = env_constants(v, a);
    return v.stage != ENV_DEAD;
}

// Can this lane run the tile starting at f0 on the fast path? Idle lanes
// (no voice, dead, or starting after the tile) qualify trivially.
// NF is the span checked: one 16-frame tile, the two tiles of a 32-frame
// gate tile, or the eight tiles of 128 frames.
template <uint32_t NF>
__device__ __forceinline__ bool fast_ok(const VoiceRegs& v, const RenderArgs& a, uint32_t f0, bool looping,
                                        bool& active) {
    static_assert(NF == 16 || NF == 32 || NF == 128, "span");
    constexpr uint32_t LOG2 = NF == 128 ? 7 : (NF == 32 ? 5 : 4);
    active = v.neutral;  // runs every path, contributing +0
    if (v.neutral) return true;
    if (v.stage == ENV_DEAD || v.start_rel >= f0 + NF) return true;
    if (v.start_rel > f0) return false;                       // starts inside the span
    if (v.stop_rel != 0u && v.stop_rel <= f0 + NF) return false;  // fade begins inside
    if (v.step >> (63 - LOG2)) return false;
    const uint64_t end = v.phase + (v.step << LOG2);
    if (end < v.phase) return false;
    const uint32_t hi = (uint32_t)(end >> 32);
    if (hi == 0xFFFFFFFFu) return false;
    if (looping ? hi + 1u >= v.le : hi + 1u >= v.len) return false;   // wrap, end or clamp
    if ((uint64_t)v.base + hi + 1u >= (uint64_t)a.pcm_len) return false;
    active = true;
    return true;
}

// Packed two-lane f32 arithmetic (sm_100 `.f32x2`): one instruction issues
// both halves, and each half rounds exactly as the scalar `.rn` instruction
// does. No packed add on this path consumes a packed product: the assembler
// contracts such a pair into one packed FMA even with an explicit rounding
// mode (measured: a strict biquad written that way left different filter
// state), so every packed product here feeds scalar adds, another product or
// an FMA's multiplicand.
__device__ __forceinline__ float2 mul2_rn(float2 a, float2 b) {
    float2 r;
    asm("{\n\t.reg .b64 pa, pb, pd;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
        "mul.rn.f32x2 pd, pa, pb;\n\tmov.b64 {%0, %1}, pd;\n\t}"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
__device__ __forceinline__ float2 fma2_rn(float2 a, float2 b, float2 c) {
    float2 r;
    asm("{\n\t.reg .b64 pa, pb, pc, pd;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
        "mov.b64 pc, {%6, %7};\n\tfma.rn.f32x2 pd, pa, pb, pc;\n\tmov.b64 {%0, %1}, pd;\n\t}"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
    return r;
}

// The biquad (transposed direct form II, b2 == b0, src/cpu.rs:564-572) on one
// sample. PACKED issues each pair of independent products, (b0 x, b1 x) and
// (a1 y, a2 y), as one packed multiply, with the same roundings: two
// instructions fewer per frame. The unit- and integral-step hot tiles use it
// (measured faster there); the fractional-step tile does not (every packed
// form measured slower on that path).
template <bool STRICT, bool PACKED = false>
__device__ __forceinline__ float biquad_core(VoiceRegs& v, float x) {
    float y;
    if (STRICT && !PACKED) {
        const float bx = __fmul_rn(v.b0, x);
        y = __fadd_rn(bx, v.z1);
        v.z1 = __fadd_rn(__fsub_rn(__fmul_rn(v.b1, x), __fmul_rn(v.a1, y)), v.z2);
        v.z2 = __fsub_rn(bx, __fmul_rn(v.a2, y));
    } else if (STRICT) {
        const float2 bb = mul2_rn(make_float2(v.b0, v.b1), make_float2(x, x));
        y = __fadd_rn(bb.x, v.z1);
        const float2 ay = mul2_rn(make_float2(v.a1, v.a2), make_float2(y, y));
        v.z1 = __fadd_rn(__fsub_rn(bb.y, ay.x), v.z2);
        v.z2 = __fsub_rn(bb.x, ay.y);
    } else if (!PACKED) {
        y = fmaf(v.b0, x, v.z1);
        v.z1 = fmaf(v.b1, x, fmaf(-v.a1, y, v.z2));
        v.z2 = fmaf(v.b0, x, -(v.a2 * y));
    } else {
        // (-a2 y) as fma(-a2, y, -0): the exact negated product.
        y = __fmaf_rn(v.b0, x, v.z1);
        const float2 z = fma2_rn(make_float2(v.b1, v.b0), make_float2(x, x),
                                 fma2_rn(make_float2(-v.a1, -v.a2), make_float2(y, y), make_float2(v.z2, -0.0f)));
        v.z1 = z.x;
        v.z2 = z.y;
    }
    return y;
}

// y = x when the region's filter is off.
template <bool STRICT, bool PACKED = false>
__device__ __forceinline__ float biquad(VoiceRegs& v, float x) {
    return v.filt ? biquad_core<STRICT, PACKED>(v, x) : x;
}

template <bool STRICT>
__device__ __forceinline__ float lerp(float s0, float s1, float frac) {
    return STRICT ? __fadd_rn(s0, __fmul_rn(__fsub_rn(s1, s0), frac)) : fmaf(s1 - s0, frac, s0);
}

template <bool STRICT, bool F32>
__device__ __forceinline__ float fast_frame(VoiceRegs& v, const RenderArgs& a, EnvStep& e, bool& active) {
    // Envelope, exactly rounded in one FMA.
    v.level = __fmaf_rn(v.level, e.em, e.ea);
    if (__fmul_rn(e.sgn, v.level) >= e.thr) active = env_transition(v, a, e);
    // Linear interpolation between two adjacent, in-bounds taps.
    const uint32_t i0 = v.base + (uint32_t)(v.phase >> 32);
    const float s0 = tap<F32>(a, i0);
    const float s1 = tap<F32>(a, i0 + 1u);
    const float frac = __fmul_rn(__uint2float_rn((uint32_t)v.phase), 2.3283064365386963e-10f);
    const float y = biquad<STRICT>(v, __fmul_rn(lerp<STRICT>(s0, s1, frac), fminf(v.level, 1.0f)));
    v.phase += v.step;
    return y;
}

// The hot path: a tile in which no lane is idle and no envelope transition
// can happen. `no_transition` is conservative: it proves, with a margin far
// above the rounding of NF sequential steps (at most 32 roundings of half an
// ulp each, about 2e-6 relative), that the threshold cannot be crossed inside
// the span. It only accepts monotone steps (a non-negative attack rate; a
// decay or release that multiplies by a coefficient in [0, 1] or subtracts a
// non-negative one, from a non-negative level), so the last frame's level
// bounds every frame's. When it holds, the frame is branch-free and the
// compiler can overlap consecutive frames (and the lane's voices).
//
// The margin covers, relative to the level: NF sequential roundings of half an
// ulp (NF * 2^-24), the rounding of em^NF by squaring (each squaring doubles
// the relative error and adds one rounding: up to (NF - 1) * 2^-24) and that
// of the test itself. 1e-5 (168 * 2^-24) covers NF <= 32 with room; 128-frame
// spans need (2 * 128 + 2) * 2^-24 = 1.5e-5 and take 4e-5.
template <uint32_t NF>
__device__ __forceinline__ bool no_transition(const VoiceRegs& v, const EnvStep& e) {
    constexpr float N = (float)NF;
    constexpr float MARGIN = NF > 32 ? 4.0e-5f : 1.0e-5f;
    if (v.stage == ENV_SUSTAIN) return true;
    if (v.stage == ENV_ATTACK) {
        // level grows by attack_rate per frame towards attack_end
        return e.ea >= 0.0f && v.level + N * e.ea + MARGIN * fabsf(e.thr) < e.thr;
    }
    const float thr = -e.thr;  // decay target or floor
    if (!(v.level >= 0.0f)) return false;
    if (e.em != 1.0f) {
        if (!(e.em >= 0.0f && e.em <= 1.0f)) return false;
        float m = e.em * e.em;  // em^NF by squaring
        m *= m;
        m *= m;
        m *= m;
        if (NF >= 32) m *= m;
        if (NF >= 128) {
            m *= m;
            m *= m;
        }
        return v.level * m * (1.0f - MARGIN) > thr;
    }
    return e.ea <= 0.0f && v.level + N * e.ea - MARGIN * v.level > thr;  // linear: ea = -coef
}

// Under no_transition, is min(level, 1) == level on every frame of the tile?
// An attack stays below attack_end; every other accepted step is
// non-increasing from the tile's first level.
__device__ __forceinline__ bool level_at_most_one(const VoiceRegs& v, const EnvStep& e) {
    if (v.stage == ENV_ATTACK) return e.thr <= 1.0f;
    return v.level <= 1.0f;
}

__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
    s = __fadd_rn(a, b);
    const float bb = __fsub_rn(s, a);
    e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
}

constexpr uint32_t RENDER_WARPS = 8;        // warps per CTA
// The warp's mix tile: one row per frame of the 16-frame tile, each row the
// 32 lanes' (left, right) pairs -- lanes 0-15 at floats 0-31, lanes 16-31 at
// floats 36-67 -- in a 72-float row. A lane stores its pair with one 64-bit
// store (each half-warp writes 128 contiguous bytes); for the fold, lane l
// reads half (l & 1) of row (l >> 1) with four-wide loads, and the 8 lanes of
// each quarter-warp phase land on 8 distinct 4-bank groups
// ((72 * row + 36 * half) mod 32 = 8 * row + 4 * half).
constexpr uint32_t SM_ROW = 72;             // floats per frame row
constexpr uint32_t SM_HALF = 36;            // offset of lanes 16-31 in a row
// The factored tile (one voice per lane, f32 tree mix): a lane stores its
// voice's sample alone, one 32-bit store per frame into a 36-float row, and
// its two gains once per tile; the fold multiplies by the gains. Half the
// shared-memory traffic of the pair tile, and the per-frame gain multiplies
// leave the voice loop. Lane l's fold reads row l >> 1 (both lanes of a row
// read the same words, a broadcast) and gain row l & 1; rows start on 4-bank
// steps ((36 * row) mod 32 = 4 * row), so 8 rows are one wavefront.
// Inside a carried span, two unit or integral-step tiles with no gate row
// between them run as one 32-frame tile: 32 rows, one gain store and load for
// both halves, and half the per-tile dispatch.
constexpr uint32_t SMY_ROW = 36;            // floats per frame row
constexpr uint32_t SMG_OFF = 2 * MIX_TILE * SMY_ROW;  // the two gain rows
constexpr uint32_t SMG_ROW = 36;
constexpr uint32_t SM_WARP = SMG_OFF + 2 * SMG_ROW;   // floats per warp
static_assert(MIX_TILE * SM_ROW <= SM_WARP, "the pair tile fits the warp's space");

// Load one voice's state into registers (the reference loads the same fields,
// shaders/render.wgsl:203-237).
__device__ __forceinline__ void load_voice(VoiceRegs& v, const RenderArgs& a, uint32_t vi, bool live) {
    v.stage = ENV_DEAD;
    v.phase = 0; v.step = 0; v.base_step = 0;
    v.base = 0; v.len = 1; v.ls = 0; v.le = 1;
    v.level = 0.0f; v.gl = v.gr = v.bgl = v.bgr = 0.0f; v.z1 = v.z2 = 0.0f;
    v.b0 = v.b1 = v.a1 = v.a2 = 0.0f;
    v.filt = false; v.loop_en = false; v.lur = false;
    v.params_base = 0; v.variant = 0; v.born = 0; v.born_gate = 0;
    v.slot = 0; v.ordinal = 0; v.start_rel = 0; v.stop_rel = 0;
    v.neutral = false;
    if (!live) return;
    const uint32_t cap = a.cap;
    const uint32_t* P = a.pool + vi;
    v.phase = ((uint64_t)P[F_PHASE_HI * cap] << 32) | P[F_PHASE_LO * cap];
    v.base_step = ((uint64_t)P[F_STEP_HI * cap] << 32) | P[F_STEP_LO * cap];
    v.step = v.base_step;
    v.base = P[F_SMP_BASE * cap];
    v.len = P[F_SMP_LEN * cap];
    v.ls = P[F_LOOP_START * cap];
    v.le = P[F_LOOP_END * cap];
    const uint32_t fl = P[F_FLAGS * cap];
    v.loop_en = (fl & KC_VF_LOOP) != 0u;
    v.lur = (fl & KC_VF_LOOP_UNTIL_RELEASE) != 0u;
    v.stage = P[F_ENV_STAGE * cap];
    v.level = __uint_as_float(P[F_ENV_LEVEL * cap]);
    v.bgl = __uint_as_float(P[F_GAIN_L * cap]);
    v.bgr = __uint_as_float(P[F_GAIN_R * cap]);
    v.gl = v.bgl; v.gr = v.bgr;
    v.z1 = __uint_as_float(P[F_FILT_Z1 * cap]);
    v.z2 = __uint_as_float(P[F_FILT_Z2 * cap]);
    v.params_base = P[F_PARAMS * cap];
    v.slot = P[F_GATE_SLOT * cap];
    v.ordinal = P[F_ORDINAL * cap];
    v.start_rel = P[F_START_REL * cap];
    v.born = P[F_BORN_VARIANT * cap];
    v.stop_rel = P[F_STOP_REL * cap];
    v.variant = v.born ? v.born - 1u : 0u;
    // A pool the caller owns (kc_render_block_noalloc) may hold indexes that
    // kc_spawn's validation never saw: an out-of-range gate slot or params
    // index raises an error bit and reads slot / entry 0 instead of reading
    // past its table.
    if (v.slot >= KC_GATE_SLOTS) {
        atomicOr(&a.st->error, ERR_SLOT_RANGE);
        v.slot = 0;
    }
    v.born_gate = v.start_rel / a.gate_frames;
    if (v.params_base >= a.params_per) {
        atomicOr(&a.st->error, ERR_PARAMS_RANGE);
        v.params_base = 0;
    }
    load_params(v, a);
}

// Write back what a block changes (src/cpu.rs:605-612).
__device__ __forceinline__ void store_voice(const VoiceRegs& v, const RenderArgs& a, uint32_t vi) {
    const uint32_t cap = a.cap;
    uint32_t* P = a.pool + vi;
    P[F_PHASE_LO * cap] = (uint32_t)v.phase;
    P[F_PHASE_HI * cap] = (uint32_t)(v.phase >> 32);
    P[F_ENV_STAGE * cap] = v.stage;
    P[F_ENV_LEVEL * cap] = __float_as_uint(v.level);
    P[F_FILT_Z1 * cap] = __float_as_uint(v.z1);
    P[F_FILT_Z2 * cap] = __float_as_uint(v.z2);
    P[F_START_REL * cap] = 0u;
    P[F_BORN_VARIANT * cap] = 0u;
    P[F_STOP_REL * cap] = 0u;
}

// Gate and controller rows at the start of a gate tile (src/cpu.rs:450-487).
template <bool CHAN>
__device__ __forceinline__ void tile_update(VoiceRegs& v, const RenderArgs& a, uint32_t gt, uint32_t chan_active) {
    if (v.stage == ENV_DEAD) return;
    if (v.stage < ENV_RELEASE && __ldg(a.gates + (size_t)gt * KC_GATE_SLOTS + v.slot) >= v.ordinal) {
        v.stage = ENV_RELEASE;
        v.level = fminf(v.level, 1.0f);
    }
    if (CHAN && chan_active) {
        // the slot's channel (GateTable::slot, src/voice.rs:260-262: ch * 128 + key)
        const uint32_t channel = (v.slot >> 7) & 15u;
        const uint4 row = __ldg(reinterpret_cast<const uint4*>(a.chan) + gt * KC_BEND_CHANNELS + channel);
        if (chan_active & 1u) v.step = scale_step(v.base_step, row.x);
        if (chan_active & 2u) {
            v.gl = __fmul_rn(v.bgl, __uint_as_float(row.y));
            v.gr = __fmul_rn(v.bgr, __uint_as_float(row.z));
        }
        if (chan_active & 4u) {
            const bool born_here = v.born != 0u && gt <= v.born_gate;
            if (row.w != v.variant && !born_here) {
                v.variant = row.w;
                load_params(v, a);
            }
        }
    }
}

// Add one voice's frame to the lane's stereo accumulators. The first voice
// of a lane stores, later ones add in a fixed order.
template <bool STRICT, bool FIRST>
__device__ __forceinline__ void acc_out(float& yl, float& yr, float y, const VoiceRegs& v) {
    if (FIRST) {
        yl = __fmul_rn(y, v.gl);
        yr = __fmul_rn(y, v.gr);
    } else if (STRICT) {
        yl = __fadd_rn(yl, __fmul_rn(y, v.gl));
        yr = __fadd_rn(yr, __fmul_rn(y, v.gr));
    } else {
        yl = fmaf(y, v.gl, yl);
        yr = fmaf(y, v.gr, yr);
    }
}

// The paths a tile can take, fastest first.
constexpr int P_UNIT = 0, P_INT = 1, P_HOT = 2, P_FAST = 3, P_GENERAL = 4;
// Filter mode of a hot tile, uniform over the warp: every lane's region
// filters, none does, or it varies by lane (tested per frame). Neutral lanes
// fit any mode (their coefficients and state are +0).
constexpr int FM_NONE = 0, FM_ALL = 1, FM_LANE = 2;

// Classify the NF frames from f0 for the whole warp: ok (linear: every lane
// on the fast path), hot (no idle lane, no transition, level <= 1
// throughout), integral (zero phase fractions), unit (step exactly 1.0).
// Fills the per-voice looping/active flags and envelope constants the paths
// use. Warp-uniform result.
template <int INTERP, int V, uint32_t NF>
__device__ __forceinline__ int classify(const VoiceRegs (&v)[V], const RenderArgs& a, uint32_t f0, bool (&looping)[V],
                                        bool (&active)[V], EnvStep (&e)[V], int& fm) {
    constexpr bool FASTPATHS = INTERP != KC_INTERP_CUBIC;
    bool ok = FASTPATHS;
#pragma unroll
    for (int k = 0; k < V; ++k) {
        looping[k] = v[k].loop_en && !(v[k].lur && v[k].stage >= ENV_RELEASE);
        active[k] = false;
        if (FASTPATHS) ok = fast_ok<NF>(v[k], a, f0, looping[k], active[k]) && ok;
    }
    bool hot = ok, integral = true, unit = true;
#pragma unroll
    for (int k = 0; k < V; ++k) {
        e[k] = env_constants(v[k], a);
        hot = hot && active[k] && no_transition<NF>(v[k], e[k]) && level_at_most_one(v[k], e[k]);
        integral = integral && ((uint32_t)v[k].phase | (uint32_t)v[k].step) == 0u;
        unit = unit && (v[k].neutral || v[k].step == (1ull << 32));
    }
    bool all_f = true, no_f = true;
#pragma unroll
    for (int k = 0; k < V; ++k) {
        all_f = all_f && (v[k].neutral || v[k].filt);
        no_f = no_f && (v[k].neutral || !v[k].filt);
    }
    fm = __all_sync(0xFFFFFFFFu, all_f) ? FM_ALL : (__all_sync(0xFFFFFFFFu, no_f) ? FM_NONE : FM_LANE);
    if (FASTPATHS && __all_sync(0xFFFFFFFFu, hot && integral && unit)) return P_UNIT;
    if (FASTPATHS && __all_sync(0xFFFFFFFFu, hot && integral)) return P_INT;
    if (INTERP == KC_INTERP_LINEAR && __all_sync(0xFFFFFFFFu, hot)) return P_HOT;
    if (INTERP == KC_INTERP_LINEAR && __all_sync(0xFFFFFFFFu, ok)) return P_FAST;
    return P_GENERAL;
}

// This lane's (left, right) pair for frame i of the tile.
__device__ __forceinline__ void put_pair(float* sm, uint32_t lane, uint32_t i, float yl, float yr) {
    *reinterpret_cast<float2*>(sm + i * SM_ROW + (lane >> 4) * SM_HALF + (lane & 15u) * 2u) = make_float2(yl, yr);
}

// Frame i's output of this lane from its voices' samples y[k]: the sample
// itself in a factored tile, else the gained pair, voices summed in k order.
template <bool FACTOR, bool STRICT, int V>
__device__ __forceinline__ void emit(float* sm, uint32_t lane, uint32_t i, const float (&y)[V],
                                     const VoiceRegs (&v)[V]) {
    if constexpr (FACTOR) {
        static_assert(V == 1, "a factored tile holds one voice per lane");
        sm[i * SMY_ROW + lane] = y[0];
    } else {
        float yl, yr;
#pragma unroll
        for (int k = 0; k < V; ++k) {
            if (k == 0) acc_out<STRICT, true>(yl, yr, y[k], v[k]);
            else acc_out<STRICT, false>(yl, yr, y[k], v[k]);
        }
        put_pair(sm, lane, i, yl, yr);
    }
}

template <bool STRICT, int FM, bool PACKED = false>
__device__ __forceinline__ float biquad_fm(VoiceRegs& v, float x) {
    if (FM == FM_NONE) return x;
    if (FM == FM_LANE) return biquad<STRICT, PACKED>(v, x);
    return biquad_core<STRICT, PACKED>(v, x);  // FM_ALL: no per-lane test
}

// Taps from a base index. The pointer is formed once, so a tap at a fixed
// offset from it needs no address arithmetic of its own.
template <bool F32>
struct Taps {
    const float* p = nullptr;
    Taps() = default;
    __device__ __forceinline__ Taps(const RenderArgs& a, uint32_t base) : p(a.pcmf + base) {}
    __device__ __forceinline__ float operator[](uint32_t i) const { return __ldg(p + i); }
};
template <>
struct Taps<false> {
    const int16_t* p = nullptr;
    Taps() = default;
    __device__ __forceinline__ Taps(const RenderArgs& a, uint32_t base) : p(a.pcm + base) {}
    __device__ __forceinline__ float operator[](uint32_t i) const {
        return fmaxf(__fmul_rn((float)__ldg(p + i), 1.0f / 32767.0f), -1.0f);
    }
};

// The hot tiles (no idle lane, no transition, level <= 1 throughout).
//  P_UNIT  every step exactly 1.0 and every phase fraction zero (the sample at
//          its root pitch at the pool rate -- every unbent note of a bank
//          sampled per key): frame i reads tap i past the tile's first.
//  P_INT   whole-number steps, zero fractions: frac is 0 on every frame, and
//          the linear interpolation s0 + (s1 - s0) * 0 is exactly s0 (s0 is
//          never -0: it is v / 32767 clamped at -1, so +0 for a zero tap), in
//          both the strict and the fused form; nearest reads the same tap. The
//          second tap and the lerp drop out and the phase advances by the
//          step's integer part.
//  P_HOT   fractional phases: two taps and the lerp, the 32.32 phase per frame.
// fast_ok proved every tap in bounds and phase + 16 * step free of overflow,
// so P_UNIT and P_INT write the phase back once at the end of the tile.
// Each tile also prefetches into L1 the line its lane reads next (the tile
// after this one), so the next tile's first taps do not wait on L2.
template <int KIND, int FM, bool STRICT, bool F32, int V, bool FACTOR, uint32_t NT = MIX_TILE>
__device__ __forceinline__ void hot_tile(VoiceRegs (&v)[V], const RenderArgs& a, const EnvStep (&e)[V], float* sm,
                                         uint32_t lane) {
    static_assert(NT == MIX_TILE || (NT == 2 * MIX_TILE && FACTOR), "a 32-frame tile is a factored one");
    constexpr uint32_t LOG_NT = NT == MIX_TILE ? 4 : 5;
    if constexpr (KIND == P_UNIT) {
        Taps<F32> t[V];
#pragma unroll
        for (int k = 0; k < V; ++k) t[k] = Taps<F32>(a, v[k].base + (uint32_t)(v[k].phase >> 32));
        if constexpr (F32) {
#pragma unroll
            for (int k = 0; k < V; ++k) {
                // The last tap of the next tile's line, clamped into the f32
                // pool and its zero pad (a neutral lane sits at the pad).
                const uint32_t nx = min(v[k].base + (uint32_t)(v[k].phase >> 32) + NT + 31u, a.pcm_len + 31u);
                asm volatile("prefetch.global.L1 [%0];" ::"l"(a.pcmf + nx));
            }
        }
#pragma unroll
        for (uint32_t i = 0; i < NT; ++i) {
            float y[V];
#pragma unroll
            for (int k = 0; k < V; ++k) {
                v[k].level = __fmaf_rn(v[k].level, e[k].em, e[k].ea);
                y[k] = biquad_fm<STRICT, FM, true>(v[k], __fmul_rn(t[k][i], v[k].level));
            }
            emit<FACTOR, STRICT, V>(sm, lane, i, y, v);
        }
        // NT frames of step 1.0 (a neutral lane's step is 0)
#pragma unroll
        for (int k = 0; k < V; ++k) v[k].phase += v[k].step << LOG_NT;
    } else if constexpr (KIND == P_INT) {
        uint32_t off[V];
#pragma unroll
        for (int k = 0; k < V; ++k) off[k] = v[k].base + (uint32_t)(v[k].phase >> 32);
#pragma unroll
        for (uint32_t i = 0; i < NT; ++i) {
            float y[V];
#pragma unroll
            for (int k = 0; k < V; ++k) {
                v[k].level = __fmaf_rn(v[k].level, e[k].em, e[k].ea);
                y[k] = biquad_fm<STRICT, FM, true>(v[k], __fmul_rn(tap<F32>(a, off[k]), v[k].level));
                off[k] += (uint32_t)(v[k].step >> 32);
            }
            emit<FACTOR, STRICT, V>(sm, lane, i, y, v);
        }
#pragma unroll
        for (int k = 0; k < V; ++k) v[k].phase += v[k].step << LOG_NT;
    } else if constexpr (F32) {
        // The tap index rides in the high word of q = phase + (base << 32)
        // (fast_ok proved base + index + 1 < pcm_len, so it cannot carry out),
        // and one 64-bit load fetches the pair (s0, d') with
        // d' = (s1 - s0) * 2^-32 from the tap-pair table. Then
        // d' * f32(lo) == (s1 - s0) * (f32(lo) * 2^-32) exactly -- the
        // power-of-two scale commutes with the rounding, nothing here is
        // subnormal -- so s0 + that is the reference's interpolation
        // (src/cpu.rs:279-283) bit for bit, in three operations instead of
        // five and one load instead of two.
        // q is kept as two 32-bit words advanced by one add-with-carry pair,
        // and the pair's address is one wide multiply-add of the high word:
        // 3.7 instructions a frame fewer than the 64-bit add, shift and
        // address arithmetic the compiler makes of q += step (measured).
        uint32_t qh[V], ql[V];
#pragma unroll
        for (int k = 0; k < V; ++k) {
            const uint64_t q = v[k].phase + ((uint64_t)v[k].base << 32);
            qh[k] = (uint32_t)(q >> 32);
            ql[k] = (uint32_t)q;
            // The next tile's first pair and the line after it: fast_ok
            // bounded the span's last index below pcm_len, and the table runs
            // ZERO_PAD entries past it.
            const float2* nx = a.pcmp + (uint32_t)((q + (v[k].step << LOG_NT)) >> 32);
            asm volatile("prefetch.global.L1 [%0];" ::"l"(nx));
            asm volatile("prefetch.global.L1 [%0];" ::"l"(nx + 16));
        }
#pragma unroll
        for (uint32_t i = 0; i < NT; ++i) {
            float y[V];
#pragma unroll
            for (int k = 0; k < V; ++k) {
                v[k].level = __fmaf_rn(v[k].level, e[k].em, e[k].ea);
                const float2* pt;
                asm("mad.wide.u32 %0, %1, 8, %2;" : "=l"(pt) : "r"(qh[k]), "l"(a.pcmp));
                const float2 t = __ldg(pt);
                const float fl = __uint2float_rn(ql[k]);
                const float s = STRICT ? __fadd_rn(t.x, __fmul_rn(t.y, fl)) : __fmaf_rn(t.y, fl, t.x);
                y[k] = biquad_fm<STRICT, FM>(v[k], __fmul_rn(s, v[k].level));
                asm("add.cc.u32 %0, %0, %2;\n\taddc.u32 %1, %1, %3;"
                    : "+r"(ql[k]), "+r"(qh[k])
                    : "r"((uint32_t)v[k].step), "r"((uint32_t)(v[k].step >> 32)));
            }
            emit<FACTOR, STRICT, V>(sm, lane, i, y, v);
        }
#pragma unroll
        for (int k = 0; k < V; ++k)
            v[k].phase = (((uint64_t)qh[k] << 32) | ql[k]) - ((uint64_t)v[k].base << 32);
    } else {
#pragma unroll
        for (uint32_t i = 0; i < NT; ++i) {
            float y[V];
#pragma unroll
            for (int k = 0; k < V; ++k) {
                v[k].level = __fmaf_rn(v[k].level, e[k].em, e[k].ea);
                const uint32_t i0 = v[k].base + (uint32_t)(v[k].phase >> 32);
                const Taps<F32> t(a, i0);
                const float frac = __fmul_rn(__uint2float_rn((uint32_t)v[k].phase), 2.3283064365386963e-10f);
                y[k] = biquad_fm<STRICT, FM>(v[k], __fmul_rn(lerp<STRICT>(t[0], t[1], frac), v[k].level));
                v[k].phase += v[k].step;
            }
            emit<FACTOR, STRICT, V>(sm, lane, i, y, v);
        }
    }
}

// Run a hot tile of kind `path` (P_UNIT, P_INT or, for linear
// interpolation, P_HOT) with filter mode FM.
template <int INTERP, int FM, bool STRICT, bool F32, int V, bool FACTOR, uint32_t NT = MIX_TILE>
__device__ __forceinline__ void hot_dispatch(int path, VoiceRegs (&v)[V], const RenderArgs& a, const EnvStep (&e)[V],
                                             float* sm, uint32_t lane) {
    if (path == P_UNIT) hot_tile<P_UNIT, FM, STRICT, F32, V, FACTOR, NT>(v, a, e, sm, lane);
    else if (path == P_INT) hot_tile<P_INT, FM, STRICT, F32, V, FACTOR, NT>(v, a, e, sm, lane);
    else if constexpr (INTERP == KC_INTERP_LINEAR)
        hot_tile<P_HOT, FM, STRICT, F32, V, FACTOR, NT>(v, a, e, sm, lane);
}

template <int INTERP, bool STRICT, bool F32, int V, bool FACTOR, uint32_t NT>
__device__ __forceinline__ void hot_dispatch_fm(int fm, int path, VoiceRegs (&v)[V], const RenderArgs& a,
                                                const EnvStep (&e)[V], float* sm, uint32_t lane) {
    if (fm == FM_ALL) hot_dispatch<INTERP, FM_ALL, STRICT, F32, V, FACTOR, NT>(path, v, a, e, sm, lane);
    else if (fm == FM_NONE) hot_dispatch<INTERP, FM_NONE, STRICT, F32, V, FACTOR, NT>(path, v, a, e, sm, lane);
    else hot_dispatch<INTERP, FM_LANE, STRICT, F32, V, FACTOR, NT>(path, v, a, e, sm, lane);
}

// Render every batch of 32*V voices this warp owns. Lane l of batch b holds
// voices b*32V + k*32 + l for k < V, so each of the V loads per field is one
// coalesced line, and its V voices' frames are summed in k order before the
// warp transpose-reduce. F32 selects the pre-converted f32 sample pool.
template <int INTERP, bool CHAN, bool STRICT, int MIX, int V, bool F32 = true, bool DOUBLE = false>
__device__ __forceinline__ void render_batches(const RenderArgs& a, float* sm, uint32_t gw, uint32_t tw, uint32_t n) {
    const uint32_t lane = lane_id();
    constexpr bool FACTOR = V == 1 && MIX == KC_MIX_F32_TREE;
    static_assert(!DOUBLE || FACTOR, "32-frame tiles are factored ones");
    uint32_t hot_tiles = 0;   // tiles classified onto a hot path (unit, integral or fractional step)
    const uint32_t per = 32u * V;
    const uint32_t nbatch = (n + per - 1u) / per;
    const uint32_t samples = a.block_frames * 2u;
    const uint32_t chan_active = CHAN ? a.ctl->chan_active : 0u;
    float* __restrict__ part = a.partial + (size_t)gw * samples;
    float* __restrict__ part_c = MIX == KC_MIX_TWO_SUM ? a.partial_c + (size_t)gw * samples : nullptr;
    // KC_MIX_F64: the same buffer holds one slice of doubles per warp.
    double* __restrict__ part_d = MIX == KC_MIX_F64 ? reinterpret_cast<double*>(a.partial) + (size_t)gw * samples
                                                    : nullptr;

    for (uint32_t b = gw; b < nbatch; b += tw) {
        VoiceRegs v[V];
#pragma unroll
        for (int k = 0; k < V; ++k) {
            const uint32_t vi = b * per + k * 32u + lane;
            load_voice(v[k], a, vi, vi < n);
        }
        const bool first = b == gw;

        // A tile's path comes from classifying it alone, or from classifying
        // a longer span at once -- 128 frames, else the 32-frame gate tile --
        // whose later tiles then reuse the result (and the envelope
        // constants, which no hot frame changes). A gate row met inside a
        // carried span that changes any lane's stage (a release), step (a
        // bend) or params variant ends the carry.
        EnvStep e[V];
        bool looping[V], active[V];
        int carried = -1, fm = FM_LANE;
        uint32_t carry_left = 0;  // tiles of the current span still to run on `carried`
        uint32_t next_gate = 0, gt = 0;
        const bool span32 = a.gate_frames % 32u == 0u;
        for (uint32_t f0 = 0, nt = MIX_TILE; f0 < a.block_frames; f0 += nt) {
            if (f0 == next_gate) {
                bool changed = false;
#pragma unroll
                for (int k = 0; k < V; ++k) {
                    const uint32_t st = v[k].stage, var = v[k].variant;
                    const uint64_t sp = v[k].step;
                    tile_update<CHAN>(v[k], a, gt, chan_active);
                    changed = changed || st != v[k].stage || sp != v[k].step || var != v[k].variant;
                }
                if (carry_left && __any_sync(0xFFFFFFFFu, changed)) carry_left = 0;
                ++gt;
                next_gate += a.gate_frames;
            }
            // This tile's word of the partial slice, fetched before the frames
            // so its latency is spent rendering (f32 tree mix). The slice is
            // read and written once per batch, never again from this SM's L1
            // before it is evicted, so its loads and stores go to L2 only
            // (.cg) and leave L1 to the taps (measured: steal workload
            // 28.89 -> 28.68 ms a block).
            const uint32_t j = f0 * 2u + lane;
            float part_prev = 0.0f;
            if (MIX == KC_MIX_F32_TREE && !first) part_prev = __ldcg(part + j);
            int path;
            if (carry_left) {
                path = carried;
                --carry_left;
            } else {
                if (F32) {
#pragma unroll
                    for (int k = 0; k < V; ++k)
                        if (v[k].stage == ENV_DEAD && !v[k].neutral) neutralize(v[k], a);
                }
                path = P_GENERAL;
                if (span32 && (f0 & 127u) == 0u && f0 + 128u <= a.block_frames) {
                    path = classify<INTERP, V, 128>(v, a, f0, looping, active, e, fm);
                    if (path <= P_HOT) carry_left = 128u / MIX_TILE - 1u;
                }
                if (!carry_left && span32 && (f0 & 31u) == 0u) {
                    path = classify<INTERP, V, 32>(v, a, f0, looping, active, e, fm);
                    if (path <= P_HOT) carry_left = 32u / MIX_TILE - 1u;
                }
                if (!carry_left) path = classify<INTERP, V, 16>(v, a, f0, looping, active, e, fm);
                carried = path;

            }
            // A hot tile (unit, integral or fractional step) whose successor
            // is in the same span and behind no gate row runs with it as one
            // 32-frame tile.
            nt = MIX_TILE;
            float part_prev2 = 0.0f;
            if (DOUBLE && path <= P_HOT && carry_left && f0 + MIX_TILE != next_gate) {
                nt = 2u * MIX_TILE;
                --carry_left;
                if (!first) part_prev2 = __ldcg(part + j + 2u * MIX_TILE);
            }
            // counted as run (a carried span cut short by a gate row is
            // classified again, so counting it ahead would count tiles twice)
            if (path <= P_HOT) hot_tiles += nt / MIX_TILE;
            if (path <= P_HOT) {
                bool done = false;
                if constexpr (DOUBLE) {
                    if (nt != MIX_TILE) {
                        hot_dispatch_fm<INTERP, STRICT, F32, V, FACTOR, 2 * MIX_TILE>(fm, path, v, a, e, sm, lane);
                        done = true;
                    }
                }
                if (!done) hot_dispatch_fm<INTERP, STRICT, F32, V, FACTOR, MIX_TILE>(fm, path, v, a, e, sm, lane);
            } else if (INTERP == KC_INTERP_LINEAR && path == P_FAST && FACTOR) {
#pragma unroll
                for (uint32_t i = 0; i < MIX_TILE; ++i) {
                    const float y = active[0] ? fast_frame<STRICT, F32>(v[0], a, e[0], active[0]) : 0.0f;
                    sm[i * SMY_ROW + lane] = y;
                }
            } else if (INTERP == KC_INTERP_LINEAR && path == P_FAST) {
#pragma unroll
                for (uint32_t i = 0; i < MIX_TILE; ++i) {
                    float yl = 0.0f, yr = 0.0f;
#pragma unroll
                    for (int k = 0; k < V; ++k) {
                        if (active[k]) {
                            const float y = fast_frame<STRICT, F32>(v[k], a, e[k], active[k]);
                            if (k == 0) acc_out<STRICT, true>(yl, yr, y, v[k]);
                            else acc_out<STRICT, false>(yl, yr, y, v[k]);
                        }
                    }
                    put_pair(sm, lane, i, yl, yr);
                }
            } else if (FACTOR) {
                const EnvParams ep = env_params(v[0], a);
#pragma unroll 1
                for (uint32_t i = 0; i < MIX_TILE; ++i) {
                    const uint32_t f = f0 + i;
                    float y = 0.0f;
                    if (v[0].stage != ENV_DEAD && f >= v[0].start_rel)
                        y = voice_frame<INTERP, STRICT, F32>(v[0], a, ep, f, looping[0]);
                    sm[i * SMY_ROW + lane] = y;
                }
            } else {
                EnvParams ep[V];
#pragma unroll
                for (int k = 0; k < V; ++k) ep[k] = env_params(v[k], a);
#pragma unroll 1
                for (uint32_t i = 0; i < MIX_TILE; ++i) {
                    const uint32_t f = f0 + i;
                    float yl = 0.0f, yr = 0.0f;
#pragma unroll
                    for (int k = 0; k < V; ++k) {
                        if (v[k].stage != ENV_DEAD && f >= v[k].start_rel) {
                            const float y = voice_frame<INTERP, STRICT, F32>(v[k], a, ep[k], f, looping[k]);
                            if (k == 0) acc_out<STRICT, true>(yl, yr, y, v[k]);
                            else acc_out<STRICT, false>(yl, yr, y, v[k]);
                        }
                    }
                    put_pair(sm, lane, i, yl, yr);
                }
            }
            // Lane l owns output slot l of the tile: frame l >> 1, channel
            // l & 1, summed over the warp's 32 lanes.
            const uint32_t h = lane & 1u;
            if constexpr (FACTOR) {
                // The gains hold for the whole tile (only a gate row changes
                // them). Slot = sum over lanes of sample x gain: per half-warp
                // two packed chains of four (even lanes, odd lanes) in lane
                // order, each pair then added, then the halves.
                sm[SMG_OFF + lane] = v[0].gl;
                sm[SMG_OFF + SMG_ROW + lane] = v[0].gr;
                __syncwarp();
                const float4* y4 = reinterpret_cast<const float4*>(sm + (lane >> 1) * SMY_ROW);
                const float4* g4 = reinterpret_cast<const float4*>(sm + SMG_OFF + h * SMG_ROW);
                if (!DOUBLE || nt == MIX_TILE) {
                    float s[2];
#pragma unroll
                    for (int c = 0; c < 2; ++c) {
                        float2 t = make_float2(0.0f, 0.0f);
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            const float4 yq = y4[4 * c + q], gq = g4[4 * c + q];
                            t = q ? fma2_rn(make_float2(yq.x, yq.y), make_float2(gq.x, gq.y), t)
                                  : mul2_rn(make_float2(yq.x, yq.y), make_float2(gq.x, gq.y));
                            t = fma2_rn(make_float2(yq.z, yq.w), make_float2(gq.z, gq.w), t);
                        }
                        s[c] = __fadd_rn(t.x, t.y);
                    }
                    __syncwarp();
                    const float sum = __fadd_rn(s[0], s[1]);
                    __stcg(part + j, first ? sum : __fadd_rn(part_prev, sum));
                } else {
                    // Slots j (frame l >> 1) and j + 32 (frame 16 + (l >> 1)),
                    // each summed as in a 16-frame tile, sharing the gain loads.
                    const float4* z4 = y4 + MIX_TILE * SMY_ROW / 4;
                    float s[2], u[2];
#pragma unroll
                    for (int c = 0; c < 2; ++c) {
                        float2 t = make_float2(0.0f, 0.0f), w = t;
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            const float4 gq = g4[4 * c + q], yq = y4[4 * c + q], zq = z4[4 * c + q];
                            const float2 g0 = make_float2(gq.x, gq.y), g1 = make_float2(gq.z, gq.w);
                            t = q ? fma2_rn(make_float2(yq.x, yq.y), g0, t) : mul2_rn(make_float2(yq.x, yq.y), g0);
                            w = q ? fma2_rn(make_float2(zq.x, zq.y), g0, w) : mul2_rn(make_float2(zq.x, zq.y), g0);
                            t = fma2_rn(make_float2(yq.z, yq.w), g1, t);
                            w = fma2_rn(make_float2(zq.z, zq.w), g1, w);
                        }
                        s[c] = __fadd_rn(t.x, t.y);
                        u[c] = __fadd_rn(w.x, w.y);
                    }
                    __syncwarp();
                    const float sum = __fadd_rn(s[0], s[1]), sum2 = __fadd_rn(u[0], u[1]);
                    __stcg(part + j, first ? sum : __fadd_rn(part_prev, sum));
                    __stcg(part + j + 2u * MIX_TILE, first ? sum2 : __fadd_rn(part_prev2, sum2));
                }
                continue;
            }
            __syncwarp();
            const float* row = sm + (lane >> 1) * SM_ROW;
            if (MIX == KC_MIX_F32_TREE) {
                // Half h of the row: lanes 16h..16h+15, two lanes per float4.
                // Sum both channels over the half in a fixed tree, then swap
                // the channel this lane does not own with its neighbour: each
                // slot is (lanes 0-15) + (lanes 16-31), in that order.
                // (Two passes of four loads keep fewer registers live.)
                const float4* q4 = reinterpret_cast<const float4*>(row + h * SM_HALF);
                float rl[4], rr[4];
#pragma unroll
                for (int p = 0; p < 2; ++p) {
                    float4 q[4];
#pragma unroll
                    for (int c = 0; c < 4; ++c) q[c] = q4[4 * p + c];
#pragma unroll
                    for (int c = 0; c < 2; ++c) {
                        rl[2 * p + c] = __fadd_rn(__fadd_rn(q[2 * c].x, q[2 * c].z), __fadd_rn(q[2 * c + 1].x, q[2 * c + 1].z));
                        rr[2 * p + c] = __fadd_rn(__fadd_rn(q[2 * c].y, q[2 * c].w), __fadd_rn(q[2 * c + 1].y, q[2 * c + 1].w));
                    }
                }
                __syncwarp();
                const float sl = __fadd_rn(__fadd_rn(rl[0], rl[1]), __fadd_rn(rl[2], rl[3]));
                const float sr = __fadd_rn(__fadd_rn(rr[0], rr[1]), __fadd_rn(rr[2], rr[3]));
                const float mine = h ? sr : sl;
                const float theirs = __shfl_xor_sync(0xFFFFFFFFu, h ? sl : sr, 1);
                const float sum = __fadd_rn(theirs, mine);  // (half 0) + (half 1) either way
                __stcg(part + j, first ? sum : __fadd_rn(part_prev, sum));
            } else {
                // This lane's channel over all 32 lanes, in lane order.
                float qq[32];
#pragma unroll
                for (int c = 0; c < 32; ++c) qq[c] = row[(c >> 4) * SM_HALF + (c & 15) * 2 + h];
                __syncwarp();
                if (MIX == KC_MIX_F64) {
                    // The FP64 form: the slot's 32 f32 terms summed in double.
                    double r[8];
#pragma unroll
                    for (int c = 0; c < 8; ++c)
                        r[c] = ((double)qq[4 * c] + (double)qq[4 * c + 1]) + ((double)qq[4 * c + 2] + (double)qq[4 * c + 3]);
                    const double sum = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
                    part_d[j] = first ? sum : part_d[j] + sum;
                } else {
                    // Compensated: sequential two-sum over the slot with carries.
                    float s = qq[0], e = 0.0f, t, err;
#pragma unroll
                    for (int c = 1; c < 32; ++c) {
                        two_sum(s, qq[c], t, err);
                        s = t;
                        e = __fadd_rn(e, err);
                    }
                    if (first) {
                        part[j] = s;
                        part_c[j] = e;
                    } else {
                        two_sum(part[j], s, t, err);
                        part[j] = t;
                        part_c[j] = __fadd_rn(__fadd_rn(part_c[j], e), err);
                    }
                }
            }
        }
#pragma unroll
        for (int k = 0; k < V; ++k) {
            const uint32_t vi = b * per + k * 32u + lane;
            if (vi < n) store_voice(v[k], a, vi);
        }
    }
    // How much of the block ran on the hot paths: the host picks the next
    // block's tile length by it (the output is the same either way).
    if (lane == 0 && gw < nbatch) {
        const uint32_t mine = (nbatch - gw + tw - 1u) / tw;
        atomicAdd(&a.st->hot_tiles, hot_tiles);
        atomicAdd(&a.st->all_tiles, mine * (a.block_frames / MIX_TILE));
    }
}

// The render pass. Template arguments select the interpolation, whether the
// channel-controller path is compiled in (the reference builds two pipelines
// for the same reason, shaders/render.wgsl:36-43), strict rounding, the mix
// arithmetic, and voices per lane (a per-context setting, so the summation
// order -- and the output bits -- are a function of the config, the live
// count and the grid alone).
template <int INTERP, bool CHAN, bool STRICT, int MIX, int V, bool DOUBLE = false>
__global__ void __launch_bounds__(RENDER_WARPS * 32, V == 1 ? 3 : 2)
k_render(RenderArgs a) {
    extern __shared__ float4 smem4[];
    float* sm = reinterpret_cast<float*>(smem4) + (threadIdx.x >> 5) * SM_WARP;
    const uint32_t gw = blockIdx.x * RENDER_WARPS + (threadIdx.x >> 5);
    const uint32_t tw = gridDim.x * RENDER_WARPS;
    render_batches<INTERP, CHAN, STRICT, MIX, V, true, DOUBLE>(a, sm, gw, tw, a.st->live_render);
}

// Fold the warps' partial slices into the output block in a fixed order:
// warp k of the CTA sums slices k, k+8, ... for 32 consecutive samples, then
// warp 0 adds the eight in order. Also records max |out| for BlockStats::peak.
template <int MIX>
__device__ __forceinline__ void reduce_body(const float* __restrict__ partial,
                                                const float* __restrict__ partial_c,
                                                float* __restrict__ out, DevState* st,
                                                uint32_t samples, uint32_t cta) {
    __shared__ float red[8][32];
    __shared__ float redc[8][32];
    __shared__ double redd[8][32];
    const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
    const uint32_t j = cta * 32u + lane;
    const uint32_t nw = st->active_warps;
    if (MIX == KC_MIX_F64) {
        const double* pd = reinterpret_cast<const double*>(partial);
        double d = 0.0;
        if (j < samples)
            for (uint32_t k = w; k < nw; k += 8u) d += __ldcs(pd + (size_t)k * samples + j);
        redd[w][lane] = d;
        __syncthreads();
        if (w == 0 && j < samples) {
            double tot = redd[0][lane];
            for (int k = 1; k < 8; ++k) tot += redd[k][lane];
            const float f = (float)tot;
            out[j] = f;
            atomicMax(&st->peak_bits, __float_as_uint(fabsf(f)));
        }
        return;
    }
    float s = 0.0f, e = 0.0f;
    if (j < samples) {
        for (uint32_t k = w; k < nw; k += 8u) {
            const size_t o = (size_t)k * samples + j;
            if (MIX == KC_MIX_F32_TREE) {
                s = __fadd_rn(s, __ldcs(partial + o));
            } else {
                float t, err;
                two_sum(s, __ldcs(partial + o), t, err);
                s = t;
                e = __fadd_rn(__fadd_rn(e, __ldcs(partial_c + o)), err);
            }
        }
    }
    red[w][lane] = s;
    redc[w][lane] = e;
    __syncthreads();
    if (w == 0 && j < samples) {
        float tot = red[0][lane], c = redc[0][lane];
        for (int k = 1; k < 8; ++k) {
            if (MIX == KC_MIX_F32_TREE) {
                tot = __fadd_rn(tot, red[k][lane]);
            } else {
                float t, err;
                two_sum(tot, red[k][lane], t, err);
                tot = t;
                c = __fadd_rn(__fadd_rn(c, redc[k][lane]), err);
            }
        }
        if (MIX != KC_MIX_F32_TREE) tot = __fadd_rn(tot, c);
        out[j] = tot;
        // |x| of a finite float orders like its bit pattern.
        atomicMax(&st->peak_bits, __float_as_uint(fabsf(tot)));
    }
}

template <int MIX>
__global__ void __launch_bounds__(256) k_reduce(const float* __restrict__ partial,
                                                const float* __restrict__ partial_c,
                                                float* __restrict__ out, DevState* st,
                                                uint32_t samples) {
    reduce_body<MIX>(partial, partial_c, out, st, samples, blockIdx.x);
}

}  // namespace kc
