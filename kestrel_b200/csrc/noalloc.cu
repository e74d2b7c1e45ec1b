// noalloc.cu -- render one block of a caller-owned voice pool without
// allocating any device memory.
//
// Why it exists: cudaMalloc and cudaFree can synchronise the whole device and
// take milliseconds, and some hosts forbid them outright once they are
// running -- a real-time audio callback has a few milliseconds per buffer and
// cannot wait on an allocation, and hosts with their own device-memory arenas
// (or graphs built once over fixed buffers) hand every buffer in from outside.
// Those callers own all inputs and outputs; the only device memory this entry
// point needs beyond them is the render pass's scratch (the per-warp partial
// mix slices and a few control words), and that lives in the file-scope array
// below instead of coming from cudaMalloc.
//
// The array is a static __device__ object: every GPU that loads this library
// holds it (NOALLOC_SCRATCH_BYTES) until the process exits, and every call on
// a device shares it. Calls that overlap on the GPU -- two streams, or two
// host threads, rendering at once on the same device -- race on it and must be
// serialised by the caller.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "common.cuh"
#include "render.cuh"

// 32 MiB: a 256-byte head for the control words, then the partial-mix slices
// (one 2 * block_frames float slice per render warp, two with the two-sum
// mix). At block_frames 4096 that is 1023 warp slices: 32,736 voices with the
// f32 mix, 16,352 with the two-sum mix; smaller blocks fit proportionally more.
static constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(32) << 20;
static constexpr size_t NOALLOC_HEAD_BYTES = 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

static_assert(sizeof(kc::DevState) + sizeof(kc::BlockCtl) <= NOALLOC_HEAD_BYTES, "head too small");

namespace kc {
// Records the message kc_last_error() returns (defined beside it in synth.cu).
int set_last_error(int code, const std::string& msg);
}  // namespace kc

namespace {

int fail(int code, const std::string& msg) { return kc::set_last_error(code, msg); }

// Voices one call can render: one 32-voice warp batch per partial slice.
uint32_t noalloc_max_voices(const kc_config& c) {
    const size_t per_slice = (size_t)c.block_frames * 2 * sizeof(float) * (c.mix_mode ? 2 : 1);
    const size_t slices = (NOALLOC_SCRATCH_BYTES - NOALLOC_HEAD_BYTES) / per_slice;
    const size_t v = slices * 32;
    return v > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)v;
}

// The scratch array's device address per device ordinal. In host code the
// array's name is only a host-side stand-in, so the address is looked up once
// per device (with that device current) and handed to the kernels.
std::mutex g_scratch_mu;
void* g_scratch_ptr[64] = {};

int scratch_for_current_device(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(KC_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= 64) return fail(KC_ERR_INVALID, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            return fail(KC_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return KC_OK;
}

// Control words for this call: what a context's admission pass would have
// left in DevState, for a render of `n` voices with no steal and no spawn.
__global__ void k_noalloc_setup(kc::DevState* st, kc::BlockCtl* ctl, uint32_t n, uint32_t nbatch,
                                uint32_t chan_active) {
    st->live = n;
    st->live_old = n;
    st->need = 0;
    st->take = 0;
    st->live_render = n;
    st->live_new = n;
    st->error = 0;
    st->peak_bits = 0;
    st->active_warps = nbatch;
    ctl->want = 0;
    ctl->chan_active = chan_active;
}

// The render pass over the caller's pool: the same per-warp batching and
// transpose-reduce as the context's render kernel, one voice per lane, each
// warp owning exactly one 32-voice batch and one partial slice.
template <int INTERP, bool CHAN, bool STRICT, int MIX>
__global__ void __launch_bounds__(kc::RENDER_WARPS * 32, 3) k_noalloc_render(kc::RenderArgs a) {
    extern __shared__ float4 smem4[];
    float* sm = reinterpret_cast<float*>(smem4) + (threadIdx.x >> 5) * kc::SM_WARP;
    const uint32_t gw = blockIdx.x * kc::RENDER_WARPS + (threadIdx.x >> 5);
    const uint32_t tw = gridDim.x * kc::RENDER_WARPS;
    kc::render_batches<INTERP, CHAN, STRICT, MIX, 1, false>(a, sm, gw, tw, a.st->live_render);
}

// Fold the slices into the block in a fixed order (eight warps each sum a
// strided set of slices, then warp 0 adds the eight), as the context's fold
// does.
template <int MIX>
__global__ void __launch_bounds__(256) k_noalloc_fold(const float* __restrict__ partial,
                                                      const float* __restrict__ partial_c, float* __restrict__ out,
                                                      kc::DevState* st, uint32_t samples) {
    __shared__ float red[8][32];
    __shared__ float redc[8][32];
    const uint32_t lane = kc::lane_id(), w = threadIdx.x >> 5;
    const uint32_t j = blockIdx.x * 32u + lane;
    const uint32_t nw = st->active_warps;
    float s = 0.0f, e = 0.0f;
    if (j < samples) {
        for (uint32_t k = w; k < nw; k += 8u) {
            const size_t o = (size_t)k * samples + j;
            if (MIX == KC_MIX_F32_TREE) {
                s = __fadd_rn(s, partial[o]);
            } else {
                float t, err;
                kc::two_sum(s, partial[o], t, err);
                s = t;
                e = __fadd_rn(__fadd_rn(e, partial_c[o]), err);
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
                kc::two_sum(tot, red[k][lane], t, err);
                tot = t;
                c = __fadd_rn(__fadd_rn(c, redc[k][lane]), err);
            }
        }
        if (MIX != KC_MIX_F32_TREE) tot = __fadd_rn(tot, c);
        out[j] = tot;
        atomicMax(&st->peak_bits, __float_as_uint(fabsf(tot)));
    }
}

template <int I, bool C, bool S, int M>
void* render_fn() {
    return reinterpret_cast<void*>(&k_noalloc_render<I, C, S, M>);
}

template <int I, bool C>
void* render_sm(bool strict, uint32_t mix) {
    if (strict) return mix ? render_fn<I, C, true, 1>() : render_fn<I, C, true, 0>();
    return mix ? render_fn<I, C, false, 1>() : render_fn<I, C, false, 0>();
}

void* render_pick(uint32_t interp, bool chan, bool strict, uint32_t mix) {
    switch (interp) {
        case KC_INTERP_NEAREST:
            return chan ? render_sm<0, true>(strict, mix) : render_sm<0, false>(strict, mix);
        case KC_INTERP_LINEAR:
            return chan ? render_sm<1, true>(strict, mix) : render_sm<1, false>(strict, mix);
        default:
            return chan ? render_sm<2, true>(strict, mix) : render_sm<2, false>(strict, mix);
    }
}

}  // namespace

extern "C" {

int kc_render_block_noalloc(const kc_config* cfg, uint32_t* d_pool, uint32_t cap, uint32_t n_voices,
                            const int16_t* d_pcm, uint64_t pcm_len, const kc_region_params* d_params,
                            uint32_t params_len, uint32_t n_slots, const uint32_t* d_gates, const uint32_t* d_chan,
                            int bend, int gain, int variant, float* d_out, void* stream) {
    if (!cfg) return fail(KC_ERR_INVALID, "null config");
    const kc_config& c = *cfg;
    if (c.block_frames == 0 || c.block_frames % kc::MIX_TILE != 0 || c.block_frames > 65535)
        return fail(KC_ERR_INVALID, "block_frames must be a non-zero multiple of 16, at most 65535");
    if (c.gate_frames == 0 || c.gate_frames % kc::MIX_TILE != 0 || c.block_frames % c.gate_frames != 0)
        return fail(KC_ERR_INVALID, "gate_frames must be a multiple of 16 that divides block_frames");
    if (c.steal_fade_frames == 0 || c.steal_fade_frames >= c.block_frames)
        return fail(KC_ERR_INVALID, "steal_fade_frames must be in 1..block_frames-1");
    if (c.interpolation > 2 || c.decay_curve > 1 || c.release_curve > 1 || c.mix_mode > 2)
        return fail(KC_ERR_INVALID, "unknown enum value in config");
    if (c.mix_mode == KC_MIX_F64)
        return fail(KC_ERR_INVALID, "KC_MIX_F64 is not supported by kc_render_block_noalloc (its f64 slices would "
                                    "halve the voices the scratch holds); use KC_MIX_F32_TREE or KC_MIX_TWO_SUM");
    if (n_voices > cap) return fail(KC_ERR_INVALID, "n_voices exceeds the pool's field stride (cap)");
    if ((n_voices && !d_pool) || !d_gates || !d_chan || !d_out || !d_params || params_len == 0 || n_slots == 0)
        return fail(KC_ERR_INVALID, "null or empty argument");
    if (pcm_len && !d_pcm) return fail(KC_ERR_INVALID, "null sample pool");
    // The kernels read params records and channel rows as 16-byte vectors and
    // the pool, gate rows and output as 32-bit words.
    const auto misaligned = [](const void* p, uintptr_t a) { return ((uintptr_t)p & (a - 1)) != 0; };
    if (misaligned(d_params, 16) || misaligned(d_chan, 16))
        return fail(KC_ERR_INVALID, "d_params and d_chan must be 16-byte aligned");
    if (misaligned(d_pool, 4) || misaligned(d_gates, 4) || misaligned(d_out, 4) || misaligned(d_pcm, 2))
        return fail(KC_ERR_INVALID, "d_pool, d_gates and d_out must be 4-byte aligned, d_pcm 2-byte aligned");
    const uint32_t max_voices = noalloc_max_voices(c);
    if (n_voices > max_voices)
        return fail(KC_ERR_INVALID, "n_voices " + std::to_string(n_voices) +
                                        " exceeds the no-alloc scratch: at block_frames " +
                                        std::to_string(c.block_frames) + " it holds at most " +
                                        std::to_string(max_voices) + " voices");

    void* scratch = nullptr;
    if (int rc = scratch_for_current_device(&scratch)) return rc;
    auto* head = static_cast<unsigned char*>(scratch);
    auto* st = reinterpret_cast<kc::DevState*>(head);
    auto* ctl = reinterpret_cast<kc::BlockCtl*>(head + sizeof(kc::DevState));
    float* partial = reinterpret_cast<float*>(head + NOALLOC_HEAD_BYTES);
    const uint32_t samples = c.block_frames * 2;
    const uint32_t nbatch = (n_voices + 31u) / 32u;
    float* partial_c = c.mix_mode ? partial + (size_t)nbatch * samples : nullptr;

    cudaStream_t q = static_cast<cudaStream_t>(stream);
    const uint32_t chan_active = (bend ? 1u : 0u) | (gain ? 2u : 0u) | (variant ? 4u : 0u);
    k_noalloc_setup<<<1, 1, 0, q>>>(st, ctl, n_voices, nbatch, chan_active);

    kc::RenderArgs ra{};
    ra.pool = d_pool;
    ra.cap = cap;
    ra.pcm = d_pcm;
    ra.pcm_len = (uint32_t)(pcm_len > 0xFFFFFFFFull ? 0xFFFFFFFFull : pcm_len);
    ra.params = d_params;
    ra.params_per = params_len;
    ra.n_slots = n_slots;
    ra.gates = d_gates;
    ra.chan = d_chan;
    ra.ctl = ctl;
    ra.st = st;
    ra.partial = partial;
    ra.partial_c = partial_c;
    ra.block_frames = c.block_frames;
    ra.gate_frames = c.gate_frames;
    ra.fade = c.steal_fade_frames;
    ra.env_floor = c.env_floor;
    ra.exp_decay = c.decay_curve == KC_CURVE_EXPONENTIAL;
    ra.exp_release = c.release_curve == KC_CURVE_EXPONENTIAL;
    if (nbatch) {
        void* fn = render_pick(c.interpolation, chan_active != 0, c.strict_fp != 0, c.mix_mode);
        void* args[] = {&ra};
        const unsigned ctas = (nbatch + kc::RENDER_WARPS - 1) / kc::RENDER_WARPS;
        // 8 warp areas of SM_WARP (1,224) floats = 39,168 bytes: under the
        // 48 KiB every kernel may take without an opt-in attribute.
        const size_t smem = (size_t)kc::RENDER_WARPS * kc::SM_WARP * sizeof(float);
        cudaError_t e = cudaLaunchKernel(fn, dim3(ctas), dim3(kc::RENDER_WARPS * 32), args, smem, q);
        if (e != cudaSuccess) return fail(KC_ERR_CUDA, std::string("render launch: ") + cudaGetErrorString(e));
    }
    const unsigned fold_ctas = (samples + 31) / 32;
    if (c.mix_mode == KC_MIX_F32_TREE)
        k_noalloc_fold<0><<<fold_ctas, 256, 0, q>>>(partial, partial_c, d_out, st, samples);
    else
        k_noalloc_fold<1><<<fold_ctas, 256, 0, q>>>(partial, partial_c, d_out, st, samples);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(KC_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    return KC_OK;
}

}  // extern "C"
