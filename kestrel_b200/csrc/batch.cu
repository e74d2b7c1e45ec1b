// batch.cu -- many contexts, one launch sequence per audio block.
//
// A kc_batch renders one block of every context (job) in a list with a single
// sequence of launches that does not depend on the jobs: it is captured once
// as a CUDA graph and replayed every block. Each pass is persistent over a
// flattened item space. After admission, the plan kernel turns every job's
// device-resident counts into per-pass item counts and prefix sums; each pass
// then walks its items, finds the owning job by binary search, and runs the
// same pass body the single-context path runs (pool_ops.cuh, render.cuh) on
// that job's pool, tables and chunk numbering. The render is one persistent
// kernel over (job, slice) items handed out to warps by an atomic counter,
// the slices of the jobs with the most batches per slice first.
//
// Results are byte-identical to rendering each context alone with kc_render:
// a job's render slices are numbered exactly as its own grid numbers them
// (slice k takes batches k, k + W, ... for the context's W render warps) and
// the fold reads them in the same fixed order; the steal select, spawn,
// compaction and sort produce results that do not depend on how their work is
// chunked.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <unordered_set>
#include <vector>

#include "common.cuh"
#include "pool_ops.cuh"
#include "render.cuh"
#include "synth_impl.cuh"

namespace kc {
int set_last_error(int code, const std::string& msg);
}  // namespace kc

using namespace kc;

namespace {

constexpr uint32_t MAX_JOBS = 1024;       // one plan CTA scans them
constexpr uint32_t SEL_CHUNK = 8192;      // voices per select / mark item
constexpr uint32_t CMP_CHUNK = 4096;      // voices per compaction / sort item
constexpr uint32_t GATHER_CHUNK = 2048;   // voices per gather item

enum Kind : uint32_t { K_SEL, K_SPAWN, K_RENDER, K_REDUCE, K_CMP, K_SCAT, K_SORT, K_GATHER, N_KINDS };

// One job's pointers and settings for one block (host-built, uploaded).
struct JobDesc {
    PoolArgs pa;
    RenderArgs ra;
    SortLayout sort;
    BlockCtl* ctl;
    uint32_t* sel_hist;
    uint32_t* counts;
    uint32_t* total;
    uint32_t* keys[2];
    uint32_t* idx[2];
    const kc_spawn_cmd* cmds;
    float* out;
    float* stage_out;      // this job's rows of the packed readback
    DevState* stage_st;
    uint32_t want, chan_active;
    uint32_t samples;
    uint32_t sort_passes;  // 0: compaction scatter, no sort
    uint32_t sel_cap;      // the context's own grid for the grid-stride passes
    uint32_t cmp_cap;      // the context's own chunk count for compaction / sort
    uint32_t pad[2];
};

struct BatchHeader {
    uint32_t n_jobs;
    uint32_t pad[3];
};

// Device-written per block by the plan kernel.
struct BatchPlan {
    uint32_t render_next;
    uint32_t pad[3];
    uint32_t prefix[N_KINDS][MAX_JOBS + 1];
    uint32_t cmp_ctas[MAX_JOBS];
    uint32_t render_job[MAX_JOBS];  // render order -> job
};

// Last j in [0, n) with prefix[j] <= it (jobs without items share the next
// job's prefix and are skipped).
__device__ __forceinline__ uint32_t find_job(const uint32_t* prefix, uint32_t n, uint32_t it) {
    uint32_t lo = 0, hi = n;  // prefix[lo] <= it < prefix[hi]
    while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) >> 1;
        if (prefix[mid] <= it) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Walk the items of one kind: f(job, item within the job, job's item count).
// Every thread of the CTA takes the same items; the trailing barrier keeps a
// pass body's shared memory from being reused before all threads are done.
template <Kind K, class F>
__device__ __forceinline__ void for_items(const BatchHeader* hdr, const BatchPlan* plan, F&& f) {
    const uint32_t n = hdr->n_jobs;
    const uint32_t* pre = plan->prefix[K];
    const uint32_t total = pre[n];
    for (uint32_t it = blockIdx.x; it < total; it += gridDim.x) {
        const uint32_t j = find_job(pre, n, it);
        f(j, it - pre[j], pre[j + 1] - pre[j]);
        __syncthreads();
    }
}

__device__ __forceinline__ uint32_t cdiv(uint32_t a, uint32_t b) { return (a + b - 1u) / b; }

// ---- admission and plan ----------------------------------------------------

__global__ void __launch_bounds__(256) kb_admit(const BatchHeader* hdr, const JobDesc* jobs) {
    const uint32_t n = hdr->n_jobs;
    for (uint32_t j = blockIdx.x; j < n; j += gridDim.x) {
        const JobDesc& d = jobs[j];
        for (uint32_t i = threadIdx.x; i < SEL_ROUNDS * 256u; i += blockDim.x) d.sel_hist[i] = 0u;
        if (threadIdx.x == 0) admit_state(d.pa, d.ctl, d.want, d.chan_active);
    }
}

// Exclusive scan over the CTA (1024 threads), returning the total in *tot.
__device__ __forceinline__ uint32_t cta_scan(uint32_t v, uint32_t* wsum, uint32_t* tot) {
    const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
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
    const uint32_t incl = x + (w ? wsum[w - 1] : 0u);
    *tot = wsum[31];
    __syncthreads();
    return incl - v;
}

__global__ void __launch_bounds__(1024) kb_plan(const BatchHeader* hdr, const JobDesc* jobs, BatchPlan* plan) {
    __shared__ uint32_t wsum[32];
    __shared__ uint32_t cost[MAX_JOBS];
    const uint32_t n = hdr->n_jobs;
    const uint32_t j = threadIdx.x;
    uint32_t cnt[N_KINDS] = {};
    uint32_t aw = 0, c = 0;
    if (j < n) {
        const JobDesc& d = jobs[j];
        const DevState* st = d.pa.st;
        const uint32_t live_old = st->live_old, need = st->need, take = st->take, nr = st->live_render;
        cnt[K_SEL] = need ? min(max(cdiv(live_old, SEL_CHUNK), 1u), d.sel_cap) : 0u;
        cnt[K_SPAWN] = cdiv(take, 256u);
        cnt[K_REDUCE] = cdiv(d.samples, 32u);
        const uint32_t g = min(max(cdiv(nr, CMP_CHUNK), 1u), d.cmp_cap);
        plan->cmp_ctas[j] = g;
        cnt[K_CMP] = g;
        cnt[K_SCAT] = d.sort_passes ? 0u : g;
        cnt[K_SORT] = d.sort_passes ? g : 0u;
        cnt[K_GATHER] = d.sort_passes ? cdiv(nr, GATHER_CHUNK) : 0u;
        aw = st->active_warps;
        // Batches per slice: the render cost of each of this job's items.
        const uint32_t per = 32u * d.pa.voices_per_lane;
        c = aw ? cdiv(cdiv(nr, per), d.pa.render_warps) : 0u;
    }
    if (j < MAX_JOBS) cost[j] = j < n ? c : 0u;
    __syncthreads();
    // Render order: most batches per slice first, then job index.
    if (j < n) {
        uint32_t rank = 0;
        for (uint32_t i = 0; i < n; ++i) rank += cost[i] > c || (cost[i] == c && i < j);
        plan->render_job[rank] = j;
    }
    uint32_t tot = 0;
    for (uint32_t k = 0; k < N_KINDS; ++k) {
        if (k == K_RENDER) continue;
        const uint32_t e = cta_scan(j < n ? cnt[k] : 0u, wsum, &tot);
        if (j < n) plan->prefix[k][j] = e;
        if (j == 0) plan->prefix[k][n] = tot;
    }
    __syncthreads();  // render_job complete
    uint32_t aw_r = 0;
    if (j < n) aw_r = jobs[plan->render_job[j]].pa.st->active_warps;
    const uint32_t e = cta_scan(aw_r, wsum, &tot);
    if (j < n) plan->prefix[K_RENDER][j] = e;
    if (j == 0) {
        plan->prefix[K_RENDER][n] = tot;
        plan->render_next = 0u;
    }
}

// ---- steal, spawn --------------------------------------------------------------

__global__ void __launch_bounds__(256) kb_select_hist(const BatchHeader* hdr, const JobDesc* jobs,
                                                      const BatchPlan* plan, uint32_t round) {
    for_items<K_SEL>(hdr, plan, [&](uint32_t j, uint32_t c, uint32_t m) {
        select_hist_body(jobs[j].pa, jobs[j].sel_hist, round, c, m);
    });
}

__global__ void __launch_bounds__(256) kb_select_refine(const BatchHeader* hdr, const JobDesc* jobs,
                                                        uint32_t round) {
    const uint32_t n = hdr->n_jobs;
    for (uint32_t j = blockIdx.x; j < n; j += gridDim.x) {
        select_refine_body(jobs[j].pa, jobs[j].sel_hist, round);
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256) kb_mark(const BatchHeader* hdr, const JobDesc* jobs, const BatchPlan* plan) {
    for_items<K_SEL>(hdr, plan, [&](uint32_t j, uint32_t c, uint32_t m) { mark_stolen_body(jobs[j].pa, c, m); });
}

__global__ void __launch_bounds__(256) kb_spawn(const BatchHeader* hdr, const JobDesc* jobs, const BatchPlan* plan) {
    for_items<K_SPAWN>(hdr, plan, [&](uint32_t j, uint32_t c, uint32_t m) {
        spawn_body(jobs[j].pa, jobs[j].cmds, c, m);
    });
}

// ---- render, fold ----------------------------------------------------------------

template <int INTERP, bool STRICT, int MIX, int V, bool DOUBLE = false>
__global__ void __launch_bounds__(RENDER_WARPS * 32, V == 1 ? 3 : 2)
kb_render(const BatchHeader* hdr, const JobDesc* jobs, BatchPlan* plan) {
    extern __shared__ float4 smem4[];
    __shared__ RenderArgs ra_s[RENDER_WARPS];
    const uint32_t w = threadIdx.x >> 5, lane = lane_id();
    float* sm = reinterpret_cast<float*>(smem4) + w * SM_WARP;
    const uint32_t n = hdr->n_jobs;
    const uint32_t* pre = plan->prefix[K_RENDER];
    const uint32_t total = pre[n];
    RenderArgs& a = ra_s[w];
    for (;;) {
        uint32_t it = 0;
        if (lane == 0) it = atomicAdd(&plan->render_next, 1u);
        it = __shfl_sync(0xFFFFFFFFu, it, 0);
        if (it >= total) break;
        const uint32_t r = find_job(pre, n, it);
        const JobDesc& d = jobs[plan->render_job[r]];
        const uint32_t k = it - pre[r];
        static_assert(sizeof(RenderArgs) % 4 == 0, "RenderArgs copies as words");
        const uint32_t* src = reinterpret_cast<const uint32_t*>(&d.ra);
        uint32_t* dst = reinterpret_cast<uint32_t*>(&a);
        for (uint32_t i = lane; i < sizeof(RenderArgs) / 4; i += 32u) dst[i] = src[i];
        __syncwarp();
        const uint32_t tw = d.pa.render_warps;
        const uint32_t nv = a.st->live_render;
        if (a.ctl->chan_active) render_batches<INTERP, true, STRICT, MIX, V, true, DOUBLE>(a, sm, k, tw, nv);
        else render_batches<INTERP, false, STRICT, MIX, V, true, DOUBLE>(a, sm, k, tw, nv);
        __syncwarp();
    }
}

template <int MIX>
__global__ void __launch_bounds__(256) kb_reduce(const BatchHeader* hdr, const JobDesc* jobs,
                                                 const BatchPlan* plan) {
    for_items<K_REDUCE>(hdr, plan, [&](uint32_t j, uint32_t c, uint32_t) {
        const JobDesc& d = jobs[j];
        reduce_body<MIX>(d.ra.partial, d.ra.partial_c, d.out, d.pa.st, d.samples, c);
    });
}

// ---- compaction, sort ------------------------------------------------------------

__global__ void __launch_bounds__(256) kb_compact_count(const BatchHeader* hdr, const JobDesc* jobs,
                                                        const BatchPlan* plan) {
    for_items<K_CMP>(hdr, plan, [&](uint32_t j, uint32_t c, uint32_t m) {
        compact_count_body(jobs[j].pa, jobs[j].counts, c, m);
    });
}

__global__ void __launch_bounds__(1024) kb_scan_commit(const BatchHeader* hdr, const JobDesc* jobs,
                                                       const BatchPlan* plan) {
    const uint32_t n = hdr->n_jobs;
    for (uint32_t j = blockIdx.x; j < n; j += gridDim.x) {
        const JobDesc& d = jobs[j];
        scan_counts_body(d.counts, plan->cmp_ctas[j], d.total);
        __syncthreads();
        if (threadIdx.x == 0) commit_body(d.pa.st, d.total);
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256) kb_compact_scatter(const BatchHeader* hdr, const JobDesc* jobs,
                                                          const BatchPlan* plan) {
    for_items<K_SCAT>(hdr, plan, [&](uint32_t j, uint32_t c, uint32_t m) {
        compact_scatter_body(jobs[j].pa, jobs[j].counts, c, m);
    });
}

// Pass p reads keys[p & 1] (the pool on pass 0) and writes keys[(p + 1) & 1],
// the alternation the single-context path uses.
template <uint32_t RB>
__global__ void __launch_bounds__(256) kb_sort_count(const BatchHeader* hdr, const JobDesc* jobs,
                                                     const BatchPlan* plan, uint32_t p) {
    for_items<K_SORT>(hdr, plan, [&](uint32_t j, uint32_t c, uint32_t m) {
        const JobDesc& d = jobs[j];
        if (p >= d.sort_passes) return;
        // Pass 0 keeps the keys it computes in idx[0] (free until pass 1
        // writes it) for its scatter.
        sort_count_body<RB>(d.pa, d.sort, p ? d.keys[p & 1u] : nullptr, RB * p, d.counts, c, m, nullptr,
                            p ? nullptr : d.idx[0]);
    });
}

template <uint32_t RB>
__global__ void __launch_bounds__(1024) kb_sort_scan(const BatchHeader* hdr, const JobDesc* jobs,
                                                     const BatchPlan* plan, uint32_t p) {
    const uint32_t n = hdr->n_jobs;
    for (uint32_t j = blockIdx.x; j < n; j += gridDim.x) {
        const JobDesc& d = jobs[j];
        if (p < d.sort_passes) scan_counts_body(d.counts, (1u << RB) * plan->cmp_ctas[j], d.total + 1);
        __syncthreads();
    }
}

template <uint32_t RB>
__global__ void __launch_bounds__(256) kb_sort_scatter(const BatchHeader* hdr, const JobDesc* jobs,
                                                       const BatchPlan* plan, uint32_t p) {
    for_items<K_SORT>(hdr, plan, [&](uint32_t j, uint32_t c, uint32_t m) {
        const JobDesc& d = jobs[j];
        if (p >= d.sort_passes) return;
        const uint32_t cur = p & 1u;
        sort_scatter_body<RB>(d.pa, d.sort, p ? d.keys[cur] : d.idx[0], p ? d.idx[cur] : nullptr, d.keys[cur ^ 1u],
                              d.idx[cur ^ 1u], RB * p, d.counts, c, m);
    });
}

// The batch's sort passes at its digit width: enough passes for a 32-bit key;
// a job whose key is shorter skips the passes it does not need.
template <uint32_t RB>
void sort_passes(cudaStream_t q, uint32_t P, const BatchHeader* h, const JobDesc* J, const BatchPlan* pl) {
    for (uint32_t p = 0; p < (32u + RB - 1u) / RB; ++p) {
        kb_sort_count<RB><<<P, 256, 0, q>>>(h, J, pl, p);
        kb_sort_scan<RB><<<P, 1024, 0, q>>>(h, J, pl, p);
        kb_sort_scatter<RB><<<P, 256, 0, q>>>(h, J, pl, p);
    }
}

__global__ void __launch_bounds__(256) kb_sort_gather(const BatchHeader* hdr, const JobDesc* jobs,
                                                      const BatchPlan* plan) {
    for_items<K_GATHER>(hdr, plan, [&](uint32_t j, uint32_t c, uint32_t m) {
        const JobDesc& d = jobs[j];
        sort_gather_body(d.pa, d.idx[d.sort_passes & 1u], c, m);
    });
}

// ---- readback ------------------------------------------------------------------------
// Pack every job's block and state words into one buffer for one copy.
__global__ void __launch_bounds__(256) kb_collect(const BatchHeader* hdr, const JobDesc* jobs) {
    const uint32_t n = hdr->n_jobs;
    for (uint32_t j = blockIdx.x; j < n; j += gridDim.x) {
        const JobDesc& d = jobs[j];
        const float4* src = reinterpret_cast<const float4*>(d.out);
        float4* dst = reinterpret_cast<float4*>(d.stage_out);
        for (uint32_t i = threadIdx.x; i < d.samples / 4u; i += blockDim.x) dst[i] = src[i];
        if (threadIdx.x < sizeof(DevState) / 4) {
            reinterpret_cast<uint32_t*>(d.stage_st)[threadIdx.x] =
                reinterpret_cast<const uint32_t*>(d.pa.st)[threadIdx.x];
        }
    }
}

template <int I, bool S, int M, int V, bool D = false>
void* render_fn() {
    return reinterpret_cast<void*>(&kb_render<I, S, M, V, D>);
}

// The 32-frame unit tiles (`dbl`) exist for the linear interpolator, the
// f32 mix and one voice per lane; null elsewhere.
template <int I, bool S, int M>
void* render_v(uint32_t v, bool dbl) {
    if constexpr (I == KC_INTERP_LINEAR && M == KC_MIX_F32_TREE) {
        if (v == 2) return dbl ? nullptr : render_fn<I, S, M, 2>();
        if (dbl) return render_fn<I, S, M, 1, true>();
    }
    return dbl ? nullptr : render_fn<I, S, M, 1>();
}

template <int I, bool S>
void* render_m(uint32_t mix, uint32_t v, bool dbl) {
    if (mix == KC_MIX_TWO_SUM) return render_v<I, S, KC_MIX_TWO_SUM>(v, dbl);
    if (mix == KC_MIX_F64) return render_v<I, S, KC_MIX_F64>(v, dbl);
    return render_v<I, S, KC_MIX_F32_TREE>(v, dbl);
}

void* batch_render_fn(uint32_t interp, bool strict, uint32_t mix, uint32_t v, bool dbl = false) {
    switch (interp) {
        case KC_INTERP_NEAREST:
            return strict ? render_m<0, true>(mix, v, dbl) : render_m<0, false>(mix, v, dbl);
        case KC_INTERP_LINEAR:
            return strict ? render_m<1, true>(mix, v, dbl) : render_m<1, false>(mix, v, dbl);
        default:
            return strict ? render_m<2, true>(mix, v, dbl) : render_m<2, false>(mix, v, dbl);
    }
}

uint32_t max_steal_of(const kc_config& c) {
    const uint64_t n = (uint64_t)c.max_voices * c.max_steal_percent / 100;
    const uint32_t v = (uint32_t)n;
    return v > 1 ? v : 1;
}

}  // namespace

struct kc_batch {
    kc_batch_config cfg{};
    int device = 0;
    int sms = 148;
    cudaStream_t stream = nullptr;
    uint32_t vpl = 1;
    uint32_t radix = 8;
    void* render_fn = nullptr;
    void* render_fn2 = nullptr;    // 32-frame unit tiles (null where not built)
    bool hot_tiles = false;       // the last batch ran mostly on hot tiles
    size_t render_smem = 0;
    uint32_t render_ctas = 0;
    uint32_t pass_ctas = 0;

    // device
    BatchHeader* d_hdr = nullptr;  // followed by max_jobs JobDesc
    JobDesc* d_jobs = nullptr;
    BatchPlan* d_plan = nullptr;
    char* d_stage = nullptr;       // per job: samples floats, then DevState
    // host
    char* h_table = nullptr;       // pinned: header + descs
    char* h_stage = nullptr;       // pinned readback
    size_t job_stride = 0;         // bytes per job in the stage

    cudaGraph_t graph = nullptr, graph2 = nullptr;
    cudaGraphExec_t exec = nullptr, exec2 = nullptr;  // 16- and 32-frame unit tiles
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    float last_ms = 0.0f;
    uint64_t blocks = 0;
};

namespace {

int fail(int code, const std::string& msg) { return kc::set_last_error(code, msg); }

#define KB_CUDA(call)                                                                    \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return fail(KC_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

void free_batch(kc_batch* b) {
    if (!b) return;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->exec2) cudaGraphExecDestroy(b->exec2);
    if (b->graph2) cudaGraphDestroy(b->graph2);
    cudaFree(b->d_hdr);
    cudaFree(b->d_plan);
    cudaFree(b->d_stage);
    cudaFreeHost(b->h_table);
    cudaFreeHost(b->h_stage);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->stream) cudaStreamDestroy(b->stream);
}

// The block's launches, in the single-context order. Every launch reads the
// job count and its items from device memory, so the sequence is the same for
// every block and every job set.
int enqueue_passes(kc_batch* b, void* render_fn) {
    cudaStream_t q = b->stream;
    const uint32_t P = b->pass_ctas;
    const BatchHeader* h = b->d_hdr;
    const JobDesc* J = b->d_jobs;
    BatchPlan* pl = b->d_plan;
    kb_admit<<<P, 256, 0, q>>>(h, J);
    kb_plan<<<1, 1024, 0, q>>>(h, J, pl);
    for (uint32_t r = 0; r < SEL_ROUNDS; ++r) {
        kb_select_hist<<<P, 256, 0, q>>>(h, J, pl, r);
        kb_select_refine<<<P, 256, 0, q>>>(h, J, r);
    }
    kb_mark<<<P, 256, 0, q>>>(h, J, pl);
    kb_spawn<<<P, 256, 0, q>>>(h, J, pl);
    void* args[] = {(void*)&h, (void*)&J, (void*)&pl};
    KB_CUDA(cudaLaunchKernel(render_fn, dim3(b->render_ctas), dim3(RENDER_WARPS * 32), args, b->render_smem, q));
    if (b->cfg.mix_mode == KC_MIX_F32_TREE) kb_reduce<KC_MIX_F32_TREE><<<P, 256, 0, q>>>(h, J, pl);
    else if (b->cfg.mix_mode == KC_MIX_TWO_SUM) kb_reduce<KC_MIX_TWO_SUM><<<P, 256, 0, q>>>(h, J, pl);
    else kb_reduce<KC_MIX_F64><<<P, 256, 0, q>>>(h, J, pl);
    kb_compact_count<<<P, 256, 0, q>>>(h, J, pl);
    kb_scan_commit<<<P, 1024, 0, q>>>(h, J, pl);
    kb_compact_scatter<<<P, 256, 0, q>>>(h, J, pl);
    switch (b->radix) {
        case 4: sort_passes<4>(q, P, h, J, pl); break;
        case 5: sort_passes<5>(q, P, h, J, pl); break;
        case 6: sort_passes<6>(q, P, h, J, pl); break;
        case 7: sort_passes<7>(q, P, h, J, pl); break;
        case 9: sort_passes<9>(q, P, h, J, pl); break;
        case 10: sort_passes<10>(q, P, h, J, pl); break;
        default: sort_passes<8>(q, P, h, J, pl); break;
    }
    kb_sort_gather<<<P, 256, 0, q>>>(h, J, pl);
    kb_collect<<<P, 256, 0, q>>>(h, J);
    KB_CUDA(cudaGetLastError());
    return KC_OK;
}

bool same_variant(const kc_batch* b, const kc_synth* s) {
    return s->device == b->device && s->cfg.block_frames == b->cfg.block_frames &&
           s->cfg.interpolation == b->cfg.interpolation && (s->cfg.strict_fp != 0) == (b->cfg.strict_fp != 0) &&
           s->cfg.mix_mode == b->cfg.mix_mode && s->vpl == b->vpl && s->radix == b->radix;
}

}  // namespace

extern "C" {

int kc_batch_config_default(kc_batch_config* c) {
    if (!c) return fail(KC_ERR_INVALID, "null config");
    std::memset(c, 0, sizeof(*c));
    c->device = 0;
    c->max_jobs = 256;
    c->block_frames = 4096;
    c->interpolation = KC_INTERP_LINEAR;
    c->strict_fp = 1;
    c->mix_mode = KC_MIX_F32_TREE;
    c->voices_per_lane = 1;
    c->use_graph = 1;
    return KC_OK;
}

int kc_batch_create(const kc_batch_config* cfg, kc_batch** out) {
    if (!cfg || !out) return fail(KC_ERR_INVALID, "null argument");
    *out = nullptr;
    if (cfg->max_jobs == 0 || cfg->max_jobs > MAX_JOBS)
        return fail(KC_ERR_INVALID, "max_jobs must be in 1..=" + std::to_string(MAX_JOBS));
    if (cfg->block_frames == 0 || cfg->block_frames % MIX_TILE != 0 || cfg->block_frames > 65535)
        return fail(KC_ERR_INVALID, "block_frames must be a non-zero multiple of 16, at most 65535");
    if (cfg->interpolation > 2 || cfg->mix_mode > 2 || cfg->voices_per_lane > 2)
        return fail(KC_ERR_INVALID, "unknown enum value in batch config");
    if (cfg->sort_radix_bits && (cfg->sort_radix_bits < SORT_RADIX_MIN || cfg->sort_radix_bits > SORT_RADIX_MAX))
        return fail(KC_ERR_INVALID, "sort_radix_bits must be 0 or in 4..=10");
    kc_batch* b = new kc_batch();
    b->cfg = *cfg;
    b->device = (int)cfg->device;
    b->vpl = cfg->voices_per_lane == 2 ? 2u : 1u;
    b->radix = cfg->sort_radix_bits ? cfg->sort_radix_bits : SORT_RADIX_DEFAULT;
    auto bail = [&](int rc) {
        free_batch(b);
        delete b;
        return rc;
    };
#define KB_TRY(call)                                                                      \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return bail(fail(e_ == cudaErrorMemoryAllocation ? KC_ERR_OOM : KC_ERR_CUDA,  \
                             std::string(#call) + ": " + cudaGetErrorString(e_)));        \
    } while (0)
    KB_TRY(cudaSetDevice(b->device));
    KB_TRY(cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device));
    KB_TRY(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    b->render_fn = batch_render_fn(cfg->interpolation, cfg->strict_fp != 0, cfg->mix_mode, b->vpl);
    b->render_fn2 = batch_render_fn(cfg->interpolation, cfg->strict_fp != 0, cfg->mix_mode, b->vpl, true);
    if (b->render_fn2)
        KB_TRY(cudaFuncSetAttribute(b->render_fn2, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)((size_t)RENDER_WARPS * SM_WARP * sizeof(float))));
    b->render_smem = (size_t)RENDER_WARPS * SM_WARP * sizeof(float);
    KB_TRY(cudaFuncSetAttribute(b->render_fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->render_smem));
    int per_sm = 0;
    KB_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, b->render_fn, RENDER_WARPS * 32, b->render_smem));
    b->render_ctas = (uint32_t)(b->sms * std::max(per_sm, 1));
    b->pass_ctas = (uint32_t)b->sms * 4;

    const size_t table = sizeof(BatchHeader) + (size_t)cfg->max_jobs * sizeof(JobDesc);
    KB_TRY(cudaMalloc(&b->d_hdr, table));
    b->d_jobs = reinterpret_cast<JobDesc*>(reinterpret_cast<char*>(b->d_hdr) + sizeof(BatchHeader));
    KB_TRY(cudaMemset(b->d_hdr, 0, table));
    KB_TRY(cudaMalloc(&b->d_plan, sizeof(BatchPlan)));
    KB_TRY(cudaMemset(b->d_plan, 0, sizeof(BatchPlan)));
    b->job_stride = (((size_t)cfg->block_frames * 2 * 4 + sizeof(DevState)) + 255) & ~(size_t)255;
    KB_TRY(cudaMalloc(&b->d_stage, b->job_stride * cfg->max_jobs));
    KB_TRY(cudaMallocHost(&b->h_table, table));
    std::memset(b->h_table, 0, table);
    KB_TRY(cudaMallocHost(&b->h_stage, b->job_stride * cfg->max_jobs));
    KB_TRY(cudaEventCreate(&b->ev0));
    KB_TRY(cudaEventCreate(&b->ev1));
    if (cfg->use_graph) {
        for (int k = 0; k < 2; ++k) {
            void* fn = k ? b->render_fn2 : b->render_fn;
            if (!fn) continue;
            KB_TRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
            const int rc = enqueue_passes(b, fn);
            cudaGraph_t g = nullptr;
            const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
            if (rc) {
                if (g) cudaGraphDestroy(g);
                return bail(rc);
            }
            KB_TRY(e);
            (k ? b->graph2 : b->graph) = g;
            KB_TRY(cudaGraphInstantiate(k ? &b->exec2 : &b->exec, g, 0));
        }
    }
    KB_TRY(cudaStreamSynchronize(b->stream));
#undef KB_TRY
    *out = b;
    return KC_OK;
}

void kc_batch_destroy(kc_batch* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    free_batch(b);
    delete b;
}

int kc_batch_render(kc_batch* b, kc_synth* const* jobs, uint32_t n_jobs, float* const* outs) {
    if (!b || (n_jobs && (!jobs || !outs))) return fail(KC_ERR_INVALID, "null argument");
    if (n_jobs > b->cfg.max_jobs)
        return fail(KC_ERR_INVALID, "n_jobs " + std::to_string(n_jobs) + " exceeds the batch's max_jobs " +
                                        std::to_string(b->cfg.max_jobs));
    std::unordered_set<const kc_synth*> seen;
    for (uint32_t j = 0; j < n_jobs; ++j) {
        kc_synth* s = jobs[j];
        if (!s || !outs[j]) return fail(KC_ERR_INVALID, "null job or output at index " + std::to_string(j));
        if (!seen.insert(s).second) return fail(KC_ERR_INVALID, "job " + std::to_string(j) + " is listed twice");
        if (s->pending)
            return fail(KC_ERR_INVALID, "job " + std::to_string(j) + " has a block in flight (kc_render_begin)");
        if (!same_variant(b, s))
            return fail(KC_ERR_INVALID, "job " + std::to_string(j) +
                                            " differs from the batch in device, block_frames, interpolation, "
                                            "strict_fp, mix_mode, voices_per_lane or sort_radix_bits");
    }
    cudaSetDevice(b->device);
    cudaStream_t q = b->stream;
    BatchHeader* hh = reinterpret_cast<BatchHeader*>(b->h_table);
    JobDesc* hj = reinterpret_cast<JobDesc*>(b->h_table + sizeof(BatchHeader));
    hh->n_jobs = n_jobs;
    for (uint32_t j = 0; j < n_jobs; ++j) {
        kc_synth* s = jobs[j];
        const kc_config& c = s->cfg;
        // A context's own stream may still hold work from kc_render or
        // kc_enqueue_block_device; its pool is only touched here after that.
        KB_CUDA(cudaStreamSynchronize(s->stream));
        if (s->want > s->cmds_cap) {
            uint32_t nc = std::max<uint32_t>(s->cmds_cap, 1);
            while (nc < s->want) nc *= 2;
            cudaFree(s->cmds);
            s->cmds = nullptr;
            s->cmds_cap = 0;
            if (cudaMalloc(&s->cmds, (size_t)nc * sizeof(kc_spawn_cmd)) != cudaSuccess)
                return fail(KC_ERR_OOM, "device spawn buffer");
            s->cmds_cap = nc;
        }
        const size_t gate_words = (size_t)s->tiles * KC_GATE_SLOTS;
        const size_t chan_words = (size_t)s->tiles * KC_BEND_CHANNELS * KC_CHAN_FIELDS;
        KB_CUDA(cudaMemcpyAsync(s->gates, s->h_gates, gate_words * 4, cudaMemcpyHostToDevice, q));
        KB_CUDA(cudaMemcpyAsync(s->chan, s->h_chan, chan_words * 4, cudaMemcpyHostToDevice, q));
        if (s->want)
            KB_CUDA(cudaMemcpyAsync(s->cmds, s->h_cmds, (size_t)s->want * sizeof(kc_spawn_cmd),
                                    cudaMemcpyHostToDevice, q));
        JobDesc& d = hj[j];
        std::memset(&d, 0, sizeof(d));
        PoolArgs& pa = d.pa;
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
        RenderArgs& ra = d.ra;
        ra.pool = pa.pool;
        ra.cap = s->cap;
        ra.pcm = s->pcm;
        ra.pcmf = s->pcmf;
        ra.pcmp = s->pcmp;
        ra.pcm_len = (uint32_t)std::min<uint64_t>(s->pcm_len, 0xFFFFFFFFull);
        ra.params = s->params;
        ra.params_per = s->params_per;
        ra.n_slots = s->n_slots;
        ra.gates = s->gates;
        ra.chan = s->chan;
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
        d.sort = block_sort_layout(s, s->bend ? s->chan : nullptr);
        d.ctl = s->ctl;
        d.sel_hist = s->sel_hist;
        d.counts = s->counts;
        d.total = s->total;
        for (int i = 0; i < 2; ++i) {
            d.keys[i] = s->keys[i];
            d.idx[i] = s->idx[i];
        }
        d.cmds = s->cmds;
        d.out = s->out;
        d.stage_out = reinterpret_cast<float*>(b->d_stage + b->job_stride * j);
        d.stage_st = reinterpret_cast<DevState*>(b->d_stage + b->job_stride * j + (size_t)c.block_frames * 8);
        d.want = s->want;
        d.chan_active = (s->bend ? 1u : 0u) | (s->gain ? 2u : 0u) | (s->variant ? 4u : 0u);
        d.samples = c.block_frames * 2;
        d.sort_passes = sort_this_block(s) ? (s->sort.bits + s->radix - 1) / s->radix : 0u;
        ++s->blocks;
        d.sel_cap = s->pool_ctas;
        d.cmp_cap = s->compact_ctas;
    }
    const size_t table = sizeof(BatchHeader) + (size_t)n_jobs * sizeof(JobDesc);
    KB_CUDA(cudaMemcpyAsync(b->d_hdr, b->h_table, table, cudaMemcpyHostToDevice, q));
    KB_CUDA(cudaEventRecord(b->ev0, q));
    // Both tile lengths leave the same bits; the last batch's unit-path
    // share picks the faster one.
    const bool dbl = b->hot_tiles && b->render_fn2;
    if (b->exec && (!dbl || b->exec2)) KB_CUDA(cudaGraphLaunch(dbl ? b->exec2 : b->exec, q));
    else if (int rc = enqueue_passes(b, dbl ? b->render_fn2 : b->render_fn)) return rc;
    KB_CUDA(cudaEventRecord(b->ev1, q));
    if (n_jobs) KB_CUDA(cudaMemcpyAsync(b->h_stage, b->d_stage, b->job_stride * n_jobs, cudaMemcpyDeviceToHost, q));
    KB_CUDA(cudaStreamSynchronize(q));
    cudaEventElapsedTime(&b->last_ms, b->ev0, b->ev1);
    b->blocks += 1;
    int rc = KC_OK;
    uint64_t unit = 0, all = 0;
    for (uint32_t j = 0; j < n_jobs; ++j) {
        kc_synth* s = jobs[j];
        const char* row = b->h_stage + b->job_stride * j;
        const size_t samples = (size_t)s->cfg.block_frames * 2;
        std::memcpy(outs[j], row, samples * 4);
        DevState st;
        std::memcpy(&st, row + samples * 4, sizeof(st));
        *s->h_st = st;
        s->parity ^= 1;
        s->want = 0;
        s->stats.active_voices = st.live;
        s->stats.stolen = st.stolen;
        s->stats.dropped = st.dropped;
        std::memcpy(&s->stats.peak, &st.peak_bits, 4);
        unit += st.hot_tiles;
        all += st.all_tiles;
        if (st.all_tiles) s->hot_tiles = (uint64_t)st.hot_tiles * 2u >= st.all_tiles;
        if (st.error && rc == KC_OK)
            rc = fail(KC_ERR_DEVICE, "job " + std::to_string(j) + ": device error word " + std::to_string(st.error));
    }
    if (all) b->hot_tiles = unit * 2u >= all;
    return rc;
}

int kc_batch_last_ms(kc_batch* b, float* ms) {
    if (!b || !ms) return fail(KC_ERR_INVALID, "null argument");
    *ms = b->last_ms;
    return KC_OK;
}

}  // extern "C"
