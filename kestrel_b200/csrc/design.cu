// design.cu -- FP64 biquad coefficient design on the device.
//
// The reference designs every region's lowpass in f32 (biquad_lowpass,
// src/bank.rs:956-979). At low cutoff that loses most of the precision of
// (1 - cos w0): at 20 Hz and 48 kHz, cos w0 = 1 - 3.4e-6, and the f32 ulp
// near 1 is 6e-8, so b0 and b1 carry about 2% error and the DC gain drifts by
// a fraction of a dB; at high Q the poles sit within w0 / 2Q of the unit
// circle, where that error also moves the resonance. Designing in FP64 and
// rounding once to f32 leaves each coefficient within half an f32 ulp of the
// exact design. The numerator is then matched to the rounded denominator: in
// exact arithmetic 1 + a1 + a2 = 2 (1 - cos w0) / a0 = 4 b0 / gain, so b0 is
// taken as gain (1 + a1' + a2') / 4 from the f32-rounded a1', a2' (the sum is
// exact in double) and b1 = 2 b0. The stored f32 filter then has the design's
// DC gain to within one rounding of b0 (about -140 dB), where rounding each
// coefficient on its own leaves the cancellation in 1 + a1' + a2' (0.06 dB at
// 20 Hz). What no FP64 design removes is the f32 quantisation of a1 itself,
// which moves a resonant pole at low cutoff by a fraction of its bandwidth.
// This is the only FP64 arithmetic on the device; the render recursion stays
// f32.
#include <cuda_runtime.h>

#include <string>

#include "common.cuh"

namespace kc {
int set_last_error(int code, const std::string& msg);
}  // namespace kc

namespace {

// The reference's design statement for statement (normalised against the
// default Q so an unresonant filter stays at unity gain), in double, with
// 1 - cos w0 written as 2 sin^2(w0 / 2) so it does not cancel.
__global__ void k_design_lowpass_f64(const float* __restrict__ fc_hz, const float* __restrict__ q_cb, uint32_t n,
                                     double sr, float4* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double q_db = (double)q_cb[i] / 10.0 - 3.01;
    double q = pow(10.0, q_db / 20.0);
    if (q < 0.001) q = 0.001;
    const double gain = sqrt(0.70710678118654752440 / q);
    double r = (double)fc_hz[i] / sr;
    r = r < 1.0e-5 ? 1.0e-5 : (r > 0.49 ? 0.49 : r);
    const double w0 = 2.0 * 3.14159265358979323846 * r;
    const double sh = sin(0.5 * w0);
    const double one_minus_cos = 2.0 * sh * sh;
    const double cos_w0 = cos(w0);
    const double alpha = sin(w0) / (2.0 * q);
    const double a0 = 1.0 + alpha;
    const float a1 = (float)(-2.0 * cos_w0 / a0);
    const float a2 = (float)((1.0 - alpha) / a0);
    // Numerator matched to the rounded poles (DC gain exactly `gain` but for
    // b0's own rounding); b1 = 2 b0 is exact in f32.
    const float b0 = (float)(gain * ((1.0 + (double)a1) + (double)a2) * 0.25);
    out[i] = make_float4(b0, 2.0f * b0, a1, a2);
}

}  // namespace

extern "C" int kc_design_lowpass_f64(const float* fc_hz, const float* q_cb, uint32_t n, float sample_rate,
                                     float* coefs, int device) {
    if (!coefs || (n && (!fc_hz || !q_cb))) return kc::set_last_error(KC_ERR_INVALID, "null argument");
    if (!(sample_rate > 0.0f)) return kc::set_last_error(KC_ERR_INVALID, "sample_rate must be positive");
    if (n == 0) return KC_OK;
    cudaError_t e = cudaSetDevice(device);
    float *d_fc = nullptr, *d_q = nullptr;
    float4* d_out = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&d_fc, (size_t)n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&d_q, (size_t)n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&d_out, (size_t)n * 16);
    if (e == cudaSuccess) e = cudaMemcpy(d_fc, fc_hz, (size_t)n * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_q, q_cb, (size_t)n * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_design_lowpass_f64<<<(n + 255) / 256, 256>>>(d_fc, d_q, n, (double)sample_rate, d_out);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(coefs, d_out, (size_t)n * 16, cudaMemcpyDeviceToHost);
    cudaFree(d_fc);
    cudaFree(d_q);
    cudaFree(d_out);
    if (e != cudaSuccess) return kc::set_last_error(KC_ERR_CUDA, std::string("design: ") + cudaGetErrorString(e));
    return KC_OK;
}
