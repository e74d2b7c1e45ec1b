// resample.cu -- the load-time sample-rate conversion on the device.
//
// SincBank::process (src/resample.rs:51-107): every output sample j of a
// source at ratio r is a 32-tap dot product of the source around
// t = j / r with one of 512 phases of a windowed-sinc table. On the host this
// is most of a soundfont's load time (a bank of 128 x 32,768-frame samples
// takes 0.2 s on one core, and the reference converts multi-gigabyte banks the
// same way); here one thread computes one output sample of any source of a
// batch, so a bank converts in one launch.
//
// Bit-exact with the host restatement: the phase arithmetic is the same f64
// multiply / floor / subtract (explicitly rounded, never contracted), the 32
// products are summed in f32 in tap order with separately rounded multiplies
// and adds (as Rust's `acc += c * v as f32` does), and the f32 sinc tables
// are built by the caller with the host's own sin/cos and passed in, so no
// device transcendental is involved.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <unordered_map>
#include <vector>

#include "common.cuh"

namespace kc {
int set_last_error(int code, const std::string& msg);
}  // namespace kc

namespace {

constexpr uint32_t TAPS = 32, PHASES = 512;

struct SourceDesc {
    uint64_t src_off;   // into the concatenated sources
    uint64_t dst_off;   // into the concatenated outputs
    uint32_t src_len;
    uint32_t dst_len;
    uint32_t table;     // index of its sinc table
    uint32_t pad;
    double inv_ratio;   // 1 / ratio, computed on the host
};

// Last s with dst_off[s] <= g (the output ranges are contiguous and ascending).
__device__ __forceinline__ uint32_t find_source(const SourceDesc* d, uint32_t n, uint64_t g) {
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) >> 1;
        if (d[mid].dst_off <= g) lo = mid;
        else hi = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(256) k_resample(const SourceDesc* __restrict__ desc, uint32_t n_src,
                                                  const int16_t* __restrict__ src, const float* __restrict__ tables,
                                                  int16_t* __restrict__ dst, uint64_t total) {
    for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total;
         g += (uint64_t)gridDim.x * blockDim.x) {
        const SourceDesc d = desc[find_source(desc, n_src, g)];
        const uint64_t j = g - d.dst_off;
        const int16_t* s = src + d.src_off;
        const int64_t n = d.src_len;
        const double t = __dmul_rn((double)j, d.inv_ratio);
        const double fl = floor(t);
        const int64_t i = (int64_t)fl;
        const double frac = __dsub_rn(t, (double)i);
        uint64_t p = (uint64_t)__dmul_rn(frac, (double)PHASES);
        if (p > PHASES - 1) p = PHASES - 1;
        const float* c = tables + (size_t)d.table * PHASES * TAPS + p * TAPS;
        const int64_t base = i - (int64_t)(TAPS / 2) + 1;
        float acc = 0.0f;
        if (base >= 0 && base + (int64_t)TAPS <= n) {
#pragma unroll
            for (uint32_t k = 0; k < TAPS; ++k) acc = __fadd_rn(acc, __fmul_rn(__ldg(c + k), (float)s[base + k]));
        } else {
#pragma unroll
            for (uint32_t k = 0; k < TAPS; ++k) {
                int64_t idx = base + (int64_t)k;
                idx = idx < 0 ? 0 : (idx > n - 1 ? n - 1 : idx);
                acc = __fadd_rn(acc, __fmul_rn(__ldg(c + k), (float)s[idx]));
            }
        }
        // acc.clamp(-32768.0, 32767.0) as i16: the sum of finite products is
        // finite, so the clamp is two comparisons and the cast truncates.
        acc = acc < -32768.0f ? -32768.0f : (acc > 32767.0f ? 32767.0f : acc);
        dst[g] = (int16_t)__float2int_rz(acc);
    }
}

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

}  // namespace

extern "C" int kc_resample_i16_batch(void* device, uint32_t n, const int16_t* const* src, const uint32_t* src_len,
                                     const double* ratio, const float* const* table, int16_t* const* dst,
                                     const uint32_t* dst_len) {
    if (n == 0) return KC_OK;
    if (!src || !src_len || !ratio || !table || !dst || !dst_len)
        return kc::set_last_error(KC_ERR_INVALID, "resample: null argument");
    const int dev = device ? *static_cast<const int*>(device) : 0;
    // Sources, outputs and tables, concatenated; identical table pointers
    // share one copy.
    std::vector<SourceDesc> desc(n);
    std::unordered_map<const float*, uint32_t> table_ix;
    std::vector<const float*> tables;
    uint64_t src_total = 0, dst_total = 0;
    for (uint32_t s = 0; s < n; ++s) {
        if (src_len[s] == 0 || (!src[s] && src_len[s]) || !dst[s] || !table[s] || !(ratio[s] > 0.0))
            return kc::set_last_error(KC_ERR_INVALID, "resample: source " + std::to_string(s) + " is empty or invalid");
        const double want = std::max(std::round((double)src_len[s] * ratio[s]), 1.0);
        if ((double)dst_len[s] != want)
            return kc::set_last_error(KC_ERR_INVALID, "resample: output " + std::to_string(s) +
                                                          " must hold max(round(len * ratio), 1) samples");
        auto it = table_ix.find(table[s]);
        if (it == table_ix.end()) {
            it = table_ix.emplace(table[s], (uint32_t)tables.size()).first;
            tables.push_back(table[s]);
        }
        desc[s] = SourceDesc{src_total, dst_total, src_len[s], dst_len[s], it->second, 0, 1.0 / ratio[s]};
        src_total += src_len[s];
        dst_total += dst_len[s];
    }
    std::vector<int16_t> h_src(src_total), h_dst(dst_total);
    for (uint32_t s = 0; s < n; ++s)
        std::copy(src[s], src[s] + src_len[s], h_src.begin() + (ptrdiff_t)desc[s].src_off);
    std::vector<float> h_tab(tables.size() * PHASES * TAPS);
    for (size_t t = 0; t < tables.size(); ++t)
        std::copy(tables[t], tables[t] + PHASES * TAPS, h_tab.begin() + (ptrdiff_t)(t * PHASES * TAPS));

    cudaError_t e = cudaSetDevice(dev);
    cudaStream_t q = nullptr;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking);
    DevBuf d_desc, d_src, d_tab, d_dst;
    if (e == cudaSuccess) e = cudaMalloc(&d_desc.p, desc.size() * sizeof(SourceDesc));
    if (e == cudaSuccess) e = cudaMalloc(&d_src.p, h_src.size() * 2);
    if (e == cudaSuccess) e = cudaMalloc(&d_tab.p, h_tab.size() * 4);
    if (e == cudaSuccess) e = cudaMalloc(&d_dst.p, h_dst.size() * 2);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_desc.p, desc.data(), desc.size() * sizeof(SourceDesc), cudaMemcpyHostToDevice, q);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_src.p, h_src.data(), h_src.size() * 2, cudaMemcpyHostToDevice, q);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_tab.p, h_tab.data(), h_tab.size() * 4, cudaMemcpyHostToDevice, q);
    if (e == cudaSuccess) {
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const uint64_t blocks = std::min<uint64_t>((dst_total + 255) / 256, (uint64_t)sms * 16);
        k_resample<<<(unsigned)blocks, 256, 0, q>>>(static_cast<const SourceDesc*>(d_desc.p), n,
                                                     static_cast<const int16_t*>(d_src.p),
                                                     static_cast<const float*>(d_tab.p),
                                                     static_cast<int16_t*>(d_dst.p), dst_total);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_dst.data(), d_dst.p, h_dst.size() * 2, cudaMemcpyDeviceToHost, q);
    if (e == cudaSuccess) e = cudaStreamSynchronize(q);
    if (q) cudaStreamDestroy(q);
    if (e != cudaSuccess) return kc::set_last_error(KC_ERR_CUDA, std::string("resample: ") + cudaGetErrorString(e));
    for (uint32_t s = 0; s < n; ++s)
        std::copy(h_dst.begin() + (ptrdiff_t)desc[s].dst_off, h_dst.begin() + (ptrdiff_t)(desc[s].dst_off + dst_len[s]),
                  dst[s]);
    return KC_OK;
}
