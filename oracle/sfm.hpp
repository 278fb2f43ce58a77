// oracle/sfm.hpp -- CPU restatement of the reference's SfM initialisation
// (TEST INFRASTRUCTURE ONLY): parse_points3d_bin (src/pipeline/sfm.rs:142-183),
// gaussians_from_sfm (:365-404) and estimate_initial_scales (:408-450).
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

#include "fmath.hpp"

namespace orc {
namespace sfm {

// Rust's slice::binary_search_by in the size-halving form of the toolchains
// that build edition 2024: no early exit on Equal, base moves right whenever
// the probe is not Greater, so among equal keys the LAST one is found.
// Returns the found index (Ok) or the insertion point (Err) with *ok set.
inline size_t rust_binary_search(const double* xs, size_t n, double t, bool* ok) {
    if (n == 0) { *ok = false; return 0; }
    size_t base = 0, size = n;
    while (size > 1) {
        const size_t half = size / 2;
        const size_t mid = base + half;
        if (!(xs[mid] > t)) base = mid;  // Less or Equal (no NaN reaches here)
        size -= half;
    }
    if (xs[base] == t) { *ok = true; return base; }
    *ok = false;
    return base + (xs[base] < t ? 1 : 0);
}

// sfm.rs:408-450: mean distance to the K = 3 nearest of a 50-wide window of
// the x-sorted points around the point's own x.
inline void estimate_initial_scales(const double* xyz, size_t n, float* scales) {
    std::vector<size_t> order(n);
    std::iota(order.begin(), order.end(), size_t(0));
    // sort_by(partial_cmp) is stable; -0.0 and 0.0 compare equal
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return xyz[3 * a] < xyz[3 * b]; });
    std::vector<double> sx(n);
    for (size_t p = 0; p < n; ++p) sx[p] = xyz[3 * order[p]];
    const size_t window = std::min<size_t>(50, n);
    std::vector<double> dists;
    for (size_t i = 0; i < n; ++i) {
        const double* q = xyz + 3 * i;
        bool ok;
        size_t found = rust_binary_search(sx.data(), n, q[0], &ok);
        if (!ok) found = 0;  // unwrap_or(0)
        const size_t start = found - std::min(found, window / 2);
        const size_t end = std::min(start + window, n);
        dists.clear();
        for (size_t p = start; p < end; ++p) {
            const size_t j = order[p];
            if (j == i) continue;
            const double* o = xyz + 3 * j;
            const double dx = o[0] - q[0], dy = o[1] - q[1], dz = o[2] - q[2];
            dists.push_back(std::sqrt(dx * dx + dy * dy + dz * dz));
        }
        std::stable_sort(dists.begin(), dists.end());
        if (dists.empty()) {
            scales[i] = 0.01f;
        } else {
            const size_t k = std::min<size_t>(3, dists.size());
            double s = -0.0;  // f64 Sum's neutral element
            for (size_t m = 0; m < k; ++m) s += dists[m];
            scales[i] = (float)(s / (double)k);
        }
    }
}

// f32::powf(x, 2.2) for x = u / 255 in [0, 1]: exp(y ln x) in double, rounded once.
inline float pow22(float x) {
    if (x == 0.0f) return 0.0f;
    return (float)fm::exp_core_d((double)2.2f * fm::log_pos_d((double)x));
}

// sfm.rs:365-404: Gaussian3D records (59 f32: position, opacity_logit,
// rotation wxyz, log_scale, sh[48] channel-major) from points and colours.
inline void gaussians_from_sfm(const double* xyz, const uint8_t* rgb, size_t n, float* out) {
    if (n == 0) return;
    std::vector<float> scales(n);
    estimate_initial_scales(xyz, n, scales.data());
    const float SH_C0_INV = 1.0f / 0.28209479177387814f;
    const float p = 0.1f;
    const float opacity_logit = fm::log_cr(p / (1.0f - p));  // math::logit(0.1)
    for (size_t i = 0; i < n; ++i) {
        float* g = out + i * 59;
        std::memset(g, 0, 59 * sizeof(float));
        g[0] = (float)xyz[3 * i];
        g[1] = (float)xyz[3 * i + 1];
        g[2] = (float)xyz[3 * i + 2];
        g[3] = opacity_logit;
        g[4] = 1.0f;
        for (int c = 0; c < 3; ++c) {
            const float x = (float)rgb[3 * i + c] / 255.0f;
            g[11 + 16 * c] = (pow22(x) - 0.5f) * SH_C0_INV;
        }
        const float s = fm::log_cr(std::fmax(scales[i], 1e-4f));
        g[8] = g[9] = g[10] = s;
    }
}

// sfm.rs:147-183: COLMAP points3D.bin (little-endian). Returns 0, or -1 when
// the data ends before a record does.
struct Point {
    uint64_t id;
    double xyz[3];
    uint8_t rgb[3];
    double error;
    uint64_t track_length;
};

inline int parse_points3d_bin(const uint8_t* d, size_t size, std::vector<Point>& pts) {
    size_t at = 0;
    auto take = [&](void* dst, size_t k) {
        if (size - at < k) return false;
        std::memcpy(dst, d + at, k);
        at += k;
        return true;
    };
    uint64_t count = 0;
    if (!take(&count, 8)) return -1;
    pts.clear();
    for (uint64_t r = 0; r < count; ++r) {
        Point p{};
        if (!take(&p.id, 8) || !take(p.xyz, 24) || !take(p.rgb, 3) || !take(&p.error, 8) || !take(&p.track_length, 8))
            return -1;
        if (p.track_length > (size - at) / 8) return -1;
        at += p.track_length * 8;
        pts.push_back(p);
    }
    return 0;
}

}  // namespace sfm
}  // namespace orc
