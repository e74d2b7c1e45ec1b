// rust.h -- Rust numeric semantics the host restatement relies on.
//
// Rust's float `min`/`max` return the non-NaN operand, `clamp` keeps NaN, and
// float-to-int `as` casts saturate with NaN mapping to zero; C++ casts of
// out-of-range floats are undefined, so every such cast goes through here.
#pragma once

#include <array>
#include <cmath>
#include <cstdint>
#include <limits>

namespace kh {

inline float rmax(float a, float b) { return std::fmax(a, b); }
inline float rmin(float a, float b) { return std::fmin(a, b); }
inline double rmaxd(double a, double b) { return std::fmax(a, b); }
inline double rmind(double a, double b) { return std::fmin(a, b); }
inline float rclamp(float v, float lo, float hi) {
    if (v < lo) v = lo;
    if (v > hi) v = hi;
    return v;
}
inline double rclampd(double v, double lo, double hi) {
    if (v < lo) v = lo;
    if (v > hi) v = hi;
    return v;
}

template <class I, class F>
inline I sat_cast(F v) {
    if (std::isnan(v)) return 0;
    if (v <= (F)std::numeric_limits<I>::min()) return std::numeric_limits<I>::min();
    if (v >= (F)std::numeric_limits<I>::max()) return std::numeric_limits<I>::max();
    return (I)v;
}

// f32::round / f64::round: half away from zero (std::round does the same).
inline float rroundf(float v) { return std::round(v); }

// Fixed::from_f64 (src/fixed.rs:24-38).
inline uint64_t fixed_from_f64(double v) {
    const double scaled = v * 4294967296.0;
    if (std::isnan(scaled) || scaled <= 0.0) return 0;
    if (scaled >= 18446744073709551616.0) return UINT64_MAX;
    return (uint64_t)scaled;
}

// bend_factor (src/fixed.rs:101-113).
inline uint32_t bend_factor(double semitones) {
    if (!std::isfinite(semitones)) return 1u << 24;
    const double f = std::exp2(semitones / 12.0) * (double)(1u << 24);
    if (f <= 0.0) return 1;
    if (f >= 4294967295.0) return 0xFFFFFFFFu;
    return (uint32_t)std::round(f);
}

}  // namespace kh
