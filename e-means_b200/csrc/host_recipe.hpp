// Host-side training plan and random streams of e-means: the batch/step
// scaling laws and the cosine schedule (unchanged from the reference, which
// keeps them on the host) and the xoshiro256++ generator whose streams fix the
// initial centroids, the per-epoch row orders and the revival draws.
#pragma once
#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/emb200.h"

namespace emb {

// Constants of src/lib.rs:31-43 (which ships faiss's e-means constants).
constexpr double kAlphaMinFactor = 0.1;
constexpr size_t kCheckUnusedEvery = 5;
constexpr float kInitUsage = 1.0f / 65536.0f;
constexpr float kSplitEpsilon = 1e-4f;
constexpr float kUnusedThreshold = 0.1f;
constexpr size_t kNoRevivalMaxD = 2;
constexpr size_t kAutoQualityMaxD = 16;
constexpr double kBatchThroughput[4] = {0.035134, 0.134749, 0.876473, 0.813344};
constexpr double kBatchQuality[4] = {0.00439175, 0.134749, 0.876473, 0.813344};
constexpr double kAlphaLaw[5] = {0.8244, -0.4617, 0.9003, -0.4498, -0.1057};

struct Recipe {
    size_t batch_size;
    double alpha0;
    std::vector<size_t> epoch_rows;
    size_t total_steps;
    float unused_threshold;
};

// Nearest power of two in ratio (src/lib.rs:165-172).
inline size_t round_power_of_two(double v) {
    if (v <= 1.0) return 1;
    double low = std::pow(2.0, (int)std::floor(std::log2(v)));
    double high = 2.0 * low;
    return (size_t)((v / low < high / v) ? low : high);
}

// Step law alpha0 = c k^a b^b n^c T^d, clamped (src/lib.rs:174-178).
inline double step_law(size_t n, size_t k, double nepochs, size_t batch) {
    double a = kAlphaLaw[0] * std::pow((double)k, kAlphaLaw[1]) * std::pow((double)batch, kAlphaLaw[2]) *
               std::pow((double)n, kAlphaLaw[3]) * std::pow(nepochs, kAlphaLaw[4]);
    return a < 1e-4 ? 1e-4 : (a > 1.0 ? 1.0 : a);
}

// Rows per pass: whole epochs, a fractional pass before the last (src/lib.rs:180-192).
inline std::vector<size_t> epoch_rows_of(size_t n, double nepochs) {
    size_t whole = (size_t)std::floor(nepochs);
    size_t rem = (size_t)std::nearbyint((nepochs - (double)whole) * (double)n);  // ties to even
    if (whole == 0) return {rem};
    std::vector<size_t> v(whole - 1, n);
    if (rem > 0) v.push_back(rem);
    v.push_back(n);
    return v;
}

// Cosine schedule with a floor of 0.1 alpha0 (src/lib.rs:194-198).
inline double scheduled_alpha(double alpha0, size_t step, size_t total) {
    double frac = (double)(step < total ? step : total) / (double)(total > 1 ? total : 1);
    double cosine = 0.5 * (1.0 + std::cos(M_PI * frac));
    return alpha0 * (kAlphaMinFactor + (1.0 - kAlphaMinFactor) * cosine);
}

// resolve_recipe (src/lib.rs:201-225).
inline Recipe resolve_recipe(size_t n, size_t d, size_t k, const emb200_config& cfg) {
    int law = cfg.batch_law;
    if (law == 0) law = d <= kAutoQualityMaxD ? 2 : 1;
    size_t batch;
    if (cfg.batch_size > 0) {
        batch = cfg.batch_size < 1 ? 1 : (cfg.batch_size > n ? n : cfg.batch_size);
    } else {
        const double* c = law == 1 ? kBatchThroughput : kBatchQuality;
        double raw = c[0] * std::pow((double)k, c[1]) * std::pow((double)n, c[2]) * std::pow(cfg.nepochs, c[3]);
        size_t b = round_power_of_two(raw);
        size_t cap = law == 1 ? round_power_of_two((double)n / 2.0) : n / 2;
        b = b < cap ? b : cap;
        b = b < n ? b : n;
        batch = b < 1 ? 1 : b;
    }
    Recipe r;
    r.batch_size = batch;
    r.alpha0 = cfg.alpha0 > 0 ? cfg.alpha0 : step_law(n, k, cfg.nepochs, batch);
    r.epoch_rows = epoch_rows_of(n, cfg.nepochs);
    r.total_steps = 0;
    for (size_t e : r.epoch_rows) r.total_steps += (e + batch - 1) / batch;
    r.unused_threshold = cfg.unused_threshold >= 0 ? cfg.unused_threshold
                                                   : (d <= kNoRevivalMaxD ? 0.0f : kUnusedThreshold);
    return r;
}

// xoshiro256++ seeded through splitmix64 (src/lib.rs:227-274).
struct Xoshiro {
    uint64_t s[4];
    explicit Xoshiro(uint64_t seed) {
        uint64_t z = seed;
        for (auto& w : s) {
            z += 0x9E3779B97F4A7C15ull;
            uint64_t v = z;
            v = (v ^ (v >> 30)) * 0xBF58476D1CE4E5B9ull;
            v = (v ^ (v >> 27)) * 0x94D049BB133111EBull;
            w = v ^ (v >> 31);
        }
    }
    static uint64_t rotl(uint64_t v, int r) { return (v << r) | (v >> (64 - r)); }
    uint64_t next() {
        uint64_t out = rotl(s[0] + s[3], 23) + s[0];
        uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return out;
    }
    // Unbiased integer in [0, bound): Lemire's multiply-and-reject.
    uint64_t below(uint64_t bound) {
        const uint64_t floor_rej = (0 - bound) % bound;
        for (;;) {
            unsigned __int128 p = (unsigned __int128)next() * bound;
            if ((uint64_t)p >= floor_rej) return (uint64_t)(p >> 64);
        }
    }
    // Uniform in (0, 1) from the top 53 bits.
    double open01() { return ((double)(next() >> 11) + 0.5) / 9007199254740992.0; }
    // Fisher-Yates from the top index down.
    void permutation(size_t n, uint32_t* p) {
        for (size_t i = 0; i < n; i++) p[i] = (uint32_t)i;
        for (size_t i = n; i-- > 1;) {
            size_t j = (size_t)below((uint64_t)i + 1);
            uint32_t t = p[i];
            p[i] = p[j];
            p[j] = t;
        }
    }
};

}  // namespace emb
