// CPU oracle for the e-means hot path.
//
// TEST INFRASTRUCTURE ONLY. This file restates, in C++, the algorithm of the
// Rust crate andrewluetgers/e-means (crate `emeans`) so that the B200 engine can
// be checked against it on identical inputs. Only tests/, the smoke check and
// the CPU-baseline leg of bench.py may load it; the engine never links or calls
// it. Each function cites the reference source it follows (paths inside the
// reference project).
//
// Floating-point semantics follow the Rust code exactly: Rust never contracts
// a*b+c into an FMA, so this file is compiled with -ffp-contract=off, and the
// only fused multiply-adds are the explicit `_mm512_fmadd_ps` / `_mm256_fmadd_ps`
// of the SIMD kernels, restated with fmaf() in the scalar emulations.
//
// Parity is pinned by the reference's own known-answer tests (recipe values
// printed by faiss 1.16.0, the Lloyd step, the quantizer round trip, integer
// exactness, brute-force tolerance): see tests/test_oracle.py.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cfloat>
#include <cstring>
#include <vector>
#include <immintrin.h>
#include <omp.h>

extern "C" {

// ---------------------------------------------------------------- constants
// src/lib.rs:31-43
static const double ALPHA_MIN_FACTOR = 0.1;
static const size_t CHECK_UNUSED_EVERY = 5;
static const float INIT_USAGE = 1.0f / 65536.0f;
static const float SPLIT_EPSILON = 1e-4f;
static const float UNUSED_THRESHOLD = 0.1f;
static const size_t NO_REVIVAL_MAX_D = 2;
static const size_t AUTO_QUALITY_MAX_D = 16;
static const double BATCH_THROUGHPUT[4] = {0.035134, 0.134749, 0.876473, 0.813344};
static const double BATCH_QUALITY[4] = {0.00439175, 0.134749, 0.876473, 0.813344};
static const double ALPHA_LAW[5] = {0.8244, -0.4617, 0.9003, -0.4498, -0.1057};
static const size_t ASSIGN_CHUNK = 65536;

// Config mirror of src/lib.rs:104-124. Optional fields use a sentinel:
// batch_size 0 = None, alpha0 <= 0 = None, unused_threshold < 0 = None.
typedef struct {
    double nepochs;
    int batch_law;  // 0 Auto, 1 Throughput, 2 Quality (src/lib.rs:94-101)
    uint64_t batch_size;
    double alpha0;
    float unused_threshold;
    float balance;
    uint64_t seed;
} orc_config;

typedef struct {
    uint64_t batch_size;
    double alpha0;
    uint64_t n_epochs;
    uint64_t total_steps;
    float unused_threshold;
} orc_recipe;

// ---------------------------------------------------------------- recipe
// src/lib.rs:165-172
static size_t round_power_of_two(double v) {
    if (v <= 1.0) return 1;
    double low = std::pow(2.0, (int)std::floor(std::log2(v)));
    double high = 2.0 * low;
    return (size_t)((v / low < high / v) ? low : high);
}

// src/lib.rs:174-178
static double step_law(size_t n, size_t k, double nepochs, size_t batch) {
    double a = ALPHA_LAW[0] * std::pow((double)k, ALPHA_LAW[1]) * std::pow((double)batch, ALPHA_LAW[2]) *
               std::pow((double)n, ALPHA_LAW[3]) * std::pow(nepochs, ALPHA_LAW[4]);
    return std::min(std::max(a, 1e-4), 1.0);
}

// src/lib.rs:180-192 (round_ties_even == nearbyint in the default rounding mode)
static std::vector<size_t> epoch_rows_of(size_t n, double nepochs) {
    size_t whole = (size_t)std::floor(nepochs);
    size_t rem = (size_t)std::nearbyint((nepochs - (double)whole) * (double)n);
    if (whole == 0) return {rem};
    std::vector<size_t> v(whole - 1, n);
    if (rem > 0) v.push_back(rem);
    v.push_back(n);
    return v;
}

// src/lib.rs:194-198
double orc_scheduled_alpha(double alpha0, size_t step, size_t total) {
    double frac = (double)std::min(step, total) / (double)std::max(total, (size_t)1);
    double cosine = 0.5 * (1.0 + std::cos(M_PI * frac));
    return alpha0 * (ALPHA_MIN_FACTOR + (1.0 - ALPHA_MIN_FACTOR) * cosine);
}

// src/lib.rs:201-225. Writes up to max_epochs entries of epoch_rows.
int orc_resolve_recipe(size_t n, size_t d, size_t k, const orc_config* cfg, orc_recipe* out, uint64_t* epoch_rows,
                       size_t max_epochs) {
    int law = cfg->batch_law;
    if (law == 0) law = (d <= AUTO_QUALITY_MAX_D) ? 2 : 1;
    size_t batch;
    if (cfg->batch_size > 0) {
        batch = std::min(std::max((size_t)cfg->batch_size, (size_t)1), n);
    } else {
        const double* c = (law == 1) ? BATCH_THROUGHPUT : BATCH_QUALITY;
        double raw = c[0] * std::pow((double)k, c[1]) * std::pow((double)n, c[2]) * std::pow(cfg->nepochs, c[3]);
        size_t b = round_power_of_two(raw);
        size_t cap = (law == 1) ? round_power_of_two((double)n / 2.0) : n / 2;
        batch = std::max(std::min(std::min(b, cap), n), (size_t)1);
    }
    double alpha0 = cfg->alpha0 > 0 ? cfg->alpha0 : step_law(n, k, cfg->nepochs, batch);
    std::vector<size_t> er = epoch_rows_of(n, cfg->nepochs);
    size_t total = 0;
    for (size_t r : er) total += (r + batch - 1) / batch;
    out->batch_size = batch;
    out->alpha0 = alpha0;
    out->n_epochs = er.size();
    out->total_steps = total;
    out->unused_threshold = cfg->unused_threshold >= 0 ? cfg->unused_threshold
                                                       : (d <= NO_REVIVAL_MAX_D ? 0.0f : UNUSED_THRESHOLD);
    for (size_t i = 0; i < er.size() && i < max_epochs; i++) epoch_rows[i] = er[i];
    return 0;
}

// ---------------------------------------------------------------- RNG
// src/lib.rs:227-274: xoshiro256++ seeded through splitmix64.
struct Rng {
    uint64_t s[4];
    explicit Rng(uint64_t seed) {
        uint64_t z = seed;
        for (int i = 0; i < 4; i++) {
            z += 0x9E3779B97F4A7C15ull;
            uint64_t x = z;
            x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
            x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
            s[i] = x ^ (x >> 31);
        }
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next_u64() {
        uint64_t r = rotl(s[0] + s[3], 23) + s[0];
        uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    uint64_t below(uint64_t bound) {  // Lemire, src/lib.rs:255-262
        for (;;) {
            unsigned __int128 m = (unsigned __int128)next_u64() * bound;
            if ((uint64_t)m >= (0 - bound) % bound) return (uint64_t)(m >> 64);
        }
    }
    double open01() { return ((double)(next_u64() >> 11) + 0.5) / (double)(1ull << 53); }
    void permutation(size_t n, uint32_t* p) {  // src/lib.rs:267-273
        for (size_t i = 0; i < n; i++) p[i] = (uint32_t)i;
        for (size_t i = n; i-- > 1;) std::swap(p[i], p[below((uint64_t)i + 1)]);
    }
};

void orc_rng_u64(uint64_t seed, size_t m, uint64_t* out) {
    Rng r(seed);
    for (size_t i = 0; i < m; i++) out[i] = r.next_u64();
}
void orc_rng_open01(uint64_t seed, size_t m, double* out) {
    Rng r(seed);
    for (size_t i = 0; i < m; i++) out[i] = r.open01();
}
void orc_rng_permutation(uint64_t seed, size_t n, uint32_t* out) { Rng(seed).permutation(n, out); }

// ---------------------------------------------------------------- FP32 kernels
// Kernel variants of src/cpu.rs: 0 = AVX-512 (dots_avx512 :200-231),
// 1 = AVX2+FMA (dots_avx2 :233-266), 2 = portable (dots_portable :182-198).
// Each has a SIMD implementation (used when the CPU has it) and a scalar
// emulation with the same rounding; tests check the two agree bit for bit.

// sqnorm, src/cpu.rs:169-180: 16 accumulators, then sequential sums.
static float sqnorm(const float* v, size_t d) {
    float acc[16] = {0};
    size_t body = d / 16 * 16;
    for (size_t i = 0; i < body; i += 16)
        for (int l = 0; l < 16; l++) acc[l] = acc[l] + v[i + l] * v[i + l];
    float s = -0.0f;
    for (int l = 0; l < 16; l++) s = s + acc[l];
    float t = -0.0f;
    for (size_t i = body; i < d; i++) t = t + v[i] * v[i];
    return s + t;
}

// Tree of _mm512_reduce_add_ps: lanes (l, l+8), (l, l+4), (l, l+2), (0, 1).
static inline float tree16(const float* a) {
    float t8[8], t4[4], t2[2];
    for (int l = 0; l < 8; l++) t8[l] = a[l] + a[l + 8];
    for (int l = 0; l < 4; l++) t4[l] = t8[l] + t8[l + 4];
    for (int l = 0; l < 2; l++) t2[l] = t4[l] + t4[l + 2];
    return t2[0] + t2[1];
}
// Tree of the AVX2 horizontal sum (src/cpu.rs:254-257): (l, l+4), (l, l+2), (0, 1).
static inline float tree8(const float* a) {
    float t4[4], t2[2];
    for (int l = 0; l < 4; l++) t4[l] = a[l] + a[l + 4];
    for (int l = 0; l < 2; l++) t2[l] = t4[l] + t4[l + 2];
    return t2[0] + t2[1];
}

// Scalar emulation of one dot product under each kernel's rounding.
static float dot_emul(int kernel, const float* q, const float* c, size_t d) {
    if (kernel == 0) {
        float acc[16] = {0};
        size_t i = 0;
        for (; i + 16 <= d; i += 16)
            for (int l = 0; l < 16; l++) acc[l] = fmaf(q[i + l], c[i + l], acc[l]);
        if (i < d)
            for (int l = 0; l < 16; l++) {
                float a = (i + l < d) ? q[i + l] : 0.0f, b = (i + l < d) ? c[i + l] : 0.0f;
                acc[l] = fmaf(a, b, acc[l]);
            }
        return tree16(acc);
    } else if (kernel == 1) {
        size_t body = d & ~(size_t)7;
        float acc[8] = {0};
        for (size_t i = 0; i < body; i += 8)
            for (int l = 0; l < 8; l++) acc[l] = fmaf(q[i + l], c[i + l], acc[l]);
        float r = tree8(acc);
        for (size_t i = body; i < d; i++) r = r + q[i] * c[i];
        return r;
    } else {
        float acc[8] = {0};
        size_t body = d / 8 * 8;
        float tail = -0.0f;
        for (size_t i = body; i < d; i++) tail = tail + q[i] * c[i];
        for (size_t i = 0; i < body; i += 8)
            for (int l = 0; l < 8; l++) acc[l] = acc[l] + q[i + l] * c[i + l];
        float s = -0.0f;
        for (int l = 0; l < 8; l++) s = s + acc[l];
        return s + tail;
    }
}

// 4x4 block of dot products, src/cpu.rs:200-231, with AVX-512 intrinsics.
__attribute__((target("avx512f"))) static void dots_avx512(const float* const* q, const float* const* c, size_t d,
                                                            float* out) {
    __m512 acc[16];
    for (int t = 0; t < 16; t++) acc[t] = _mm512_setzero_ps();
    size_t i = 0;
    while (i + 16 <= d) {
        __m512 qv[4], cv[4];
        for (int t = 0; t < 4; t++) qv[t] = _mm512_loadu_ps(q[t] + i);
        for (int t = 0; t < 4; t++) cv[t] = _mm512_loadu_ps(c[t] + i);
        for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) acc[4 * a + b] = _mm512_fmadd_ps(qv[a], cv[b], acc[4 * a + b]);
        i += 16;
    }
    if (i < d) {
        __mmask16 mask = (__mmask16)((1u << (d - i)) - 1);
        __m512 qv[4], cv[4];
        for (int t = 0; t < 4; t++) qv[t] = _mm512_maskz_loadu_ps(mask, q[t] + i);
        for (int t = 0; t < 4; t++) cv[t] = _mm512_maskz_loadu_ps(mask, c[t] + i);
        for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) acc[4 * a + b] = _mm512_fmadd_ps(qv[a], cv[b], acc[4 * a + b]);
    }
    for (int t = 0; t < 16; t++) {
        alignas(64) float lanes[16];
        _mm512_store_ps(lanes, acc[t]);
        out[t] = tree16(lanes);
    }
}

// src/cpu.rs:233-266 with AVX2+FMA intrinsics.
__attribute__((target("avx2,fma"))) static void dots_avx2(const float* const* q, const float* const* c, size_t d,
                                                          float* out) {
    size_t body = d & ~(size_t)7;
    for (int half = 0; half < 2; half++) {
        const float* q0 = q[2 * half];
        const float* q1 = q[2 * half + 1];
        __m256 acc[8];
        for (int t = 0; t < 8; t++) acc[t] = _mm256_setzero_ps();
        for (size_t i = 0; i < body; i += 8) {
            __m256 a0 = _mm256_loadu_ps(q0 + i), a1 = _mm256_loadu_ps(q1 + i);
            for (int b = 0; b < 4; b++) {
                __m256 cv = _mm256_loadu_ps(c[b] + i);
                acc[b] = _mm256_fmadd_ps(a0, cv, acc[b]);
                acc[4 + b] = _mm256_fmadd_ps(a1, cv, acc[4 + b]);
            }
        }
        for (int t = 0; t < 8; t++) {
            alignas(32) float lanes[8];
            _mm256_store_ps(lanes, acc[t]);
            const float* qrow = t < 4 ? q0 : q1;
            float r = tree8(lanes);
            for (size_t i = body; i < d; i++) r = r + qrow[i] * c[t % 4][i];
            out[8 * half + t] = r;
        }
    }
}

static void dots_scalar(int kernel, const float* const* q, const float* const* c, size_t d, float* out) {
    for (int a = 0; a < 4; a++)
        for (int b = 0; b < 4; b++) out[4 * a + b] = dot_emul(kernel, q[a], c[b], d);
}

static bool cpu_has(int kernel) {
    if (kernel == 0) return __builtin_cpu_supports("avx512f");
    if (kernel == 1) return __builtin_cpu_supports("avx2") && __builtin_cpu_supports("fma");
    return true;
}

int orc_cpu_has_kernel(int kernel) { return cpu_has(kernel) ? 1 : 0; }

// CpuAssigner state (src/cpu.rs:41-104).
struct CpuAssigner {
    int kernel;     // 0 avx512, 1 avx2, 2 portable
    bool emulate;   // scalar emulation instead of intrinsics
    size_t k = 0, d = 0;
    std::vector<float> centroids, norms;
    void set_centroids(const float* c, size_t k_, size_t d_) {  // src/cpu.rs:84-93
        k = k_;
        d = d_;
        centroids.assign(c, c + k * d);
        norms.resize(k);
        for (size_t j = 0; j < k; j++) norms[j] = sqnorm(&centroids[j * d], d);
    }
    void set_bias(const float* b) {  // src/cpu.rs:95-99
        for (size_t j = 0; j < k; j++) norms[j] = norms[j] + b[j];
    }
    // src/cpu.rs:108-167. x holds m rows already widened to f32.
    void assign(const float* x, size_t m, uint32_t* labels, float* dist, int threads) {
        size_t block = std::min(std::max((size_t)(256 * 1024) / (4 * d), (size_t)4), (size_t)4096) & ~(size_t)3;
        size_t nblocks = (m + block - 1) / block;
        bool simd = !emulate && cpu_has(kernel) && kernel != 2;
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
        for (size_t bi = 0; bi < nblocks; bi++) {
            size_t r0 = bi * block, nq = std::min(block, m - r0);
            const float* xb = x + r0 * d;
            float* best = dist + r0;
            uint32_t* lab = labels + r0;
            for (size_t i = 0; i < nq; i++) {
                best[i] = INFINITY;
                lab[i] = 0;
            }
            float out[16];
            for (size_t c0 = 0; c0 < k; c0 += block) {
                size_t c1 = std::min(c0 + block, k);
                for (size_t q0 = 0; q0 < nq; q0 += 4) {
                    size_t qn = std::min(nq - q0, (size_t)4);
                    const float* qp[4];
                    for (size_t i = 0; i < 4; i++) qp[i] = xb + (q0 + std::min(i, qn - 1)) * d;
                    for (size_t j0 = c0; j0 < c1; j0 += 4) {
                        size_t cn = std::min(c1 - j0, (size_t)4);
                        const float* cp[4];
                        for (size_t i = 0; i < 4; i++) cp[i] = &centroids[(j0 + std::min(i, cn - 1)) * d];
                        if (simd && kernel == 0)
                            dots_avx512(qp, cp, d, out);
                        else if (simd && kernel == 1)
                            dots_avx2(qp, cp, d, out);
                        else
                            dots_scalar(kernel, qp, cp, d, out);
                        for (size_t qi = 0; qi < qn; qi++) {
                            float b = best[q0 + qi];
                            uint32_t l = lab[q0 + qi];
                            for (size_t ci = 0; ci < cn; ci++) {
                                float s = norms[j0 + ci] - 2.0f * out[4 * qi + ci];
                                if (s < b) {
                                    b = s;
                                    l = (uint32_t)(j0 + ci);
                                }
                            }
                            best[q0 + qi] = b;
                            lab[q0 + qi] = l;
                        }
                    }
                }
            }
            for (size_t i = 0; i < nq; i++) {
                float v = best[i] + sqnorm(xb + i * d, d);
                best[i] = std::fmax(v, 0.0f);  // f32::max(v, 0.0)
            }
        }
    }
};

// Widen rows of dtype (0 f32, 1 i8, 2 u8) to f32 (src/lib.rs:62-71, Scalar::to_f32).
static void widen(int dtype, const void* x, size_t count, float* out) {
    if (dtype == 0) {
        std::memcpy(out, x, count * sizeof(float));
    } else if (dtype == 1) {
        const int8_t* p = (const int8_t*)x;
        for (size_t i = 0; i < count; i++) out[i] = (float)p[i];
    } else {
        const uint8_t* p = (const uint8_t*)x;
        for (size_t i = 0; i < count; i++) out[i] = (float)p[i];
    }
}

// One-shot CpuAssigner: set_centroids, optional set_bias, assign.
// kernel: 0 avx512, 1 avx2, 2 portable; +8 forces the scalar emulation.
int orc_cpu_assign(int kernel, int dtype, const void* x, size_t m, size_t d, const float* c, size_t k,
                   const float* bias, uint32_t* labels, float* dist, int threads) {
    CpuAssigner a;
    a.kernel = kernel & 7;
    a.emulate = (kernel & 8) != 0;
    if (!a.emulate && !cpu_has(a.kernel)) return -1;
    a.set_centroids(c, k, d);
    if (bias) a.set_bias(bias);
    std::vector<float> xf(m * d);
    widen(dtype, x, m * d, xf.data());
    a.assign(xf.data(), m, labels, dist, threads);
    return 0;
}

// Raw per-pair score used by a kernel (tests): norm_j - 2 * dot under kernel rounding.
float orc_score(int kernel, const float* x, const float* c, size_t d) {
    return sqnorm(c, d) - 2.0f * dot_emul(kernel, x, c, d);
}
float orc_sqnorm(const float* v, size_t d) { return sqnorm(v, d); }

// ---------------------------------------------------------------- int8 kernels
// CpuI8Assigner, src/cpu_i8.rs:34-191. Both the VNNI and portable kernels
// compute exact integers, so one portable restatement covers both.
struct I8Assigner {
    int bits = 8;  // 8 or 16 (CentroidBits::I8 / I16)
    size_t k = 0, d = 0;
    uint32_t shift = 0;
    std::vector<int8_t> c8;
    std::vector<int16_t> c16;
    std::vector<int64_t> offset;
    int64_t mult = 2;
    static int8_t round_i8(float c) {  // c.round().clamp(-128, 127) as i8
        if (std::isnan(c)) return 0;
        float r = std::round(c);
        return (int8_t)std::min(std::max(r, -128.0f), 127.0f);
    }
    int set_centroids(const float* c, size_t k_, size_t d_) {  // src/cpu_i8.rs:73-110
        if (d_ > 32768) return -1;
        k = k_;
        d = d_;
        if (bits == 8) {
            shift = 0;
            c8.resize(k * d);
            for (size_t i = 0; i < k * d; i++) c8[i] = round_i8(c[i]);
            offset.resize(k);
            for (size_t j = 0; j < k; j++) {
                int64_t s = 0;
                for (size_t t = 0; t < d; t++) {
                    int64_t v = c8[j * d + t];
                    s += v * v + 256 * v;
                }
                offset[j] = s;
            }
            mult = 2;
        } else {
            shift = 0;
            for (int s = 7; s >= 0; s--)
                if (((uint64_t)d << (14 + s)) < (1ull << 31)) {
                    shift = (uint32_t)s;
                    break;
                }
            float scale = (float)(1u << shift);
            c16.resize(k * d);
            for (size_t i = 0; i < k * d; i++) {
                float v = c[i] * scale;
                if (std::isnan(v)) {
                    c16[i] = 0;
                    continue;
                }
                float r = std::min(std::max(std::round(v), -32768.0f), 32767.0f);
                c16[i] = (int16_t)r;
            }
            offset.resize(k);
            for (size_t j = 0; j < k; j++) {
                int64_t s = 0;
                for (size_t t = 0; t < d; t++) {
                    int64_t v = c16[j * d + t];
                    s += v * v;
                }
                offset[j] = s;
            }
            mult = (int64_t)2 << shift;
        }
        return 0;
    }
    void set_bias(const float* b) {  // src/cpu_i8.rs:112-117
        double unit = (double)(1ull << (2 * shift));
        for (size_t j = 0; j < k; j++) {
            double v = std::round((double)b[j] * unit);
            int64_t iv;
            if (std::isnan(v)) iv = 0;
            else if (v >= 9.2233720368547758e18) iv = INT64_MAX;
            else if (v <= -9.2233720368547758e18) iv = INT64_MIN;
            else iv = (int64_t)v;
            offset[j] += iv;
        }
    }
    void assign(const int8_t* x, size_t m, uint32_t* labels, float* dist, int threads) {  // :130-191
        double inv_unit = 1.0 / (double)(1ull << (2 * shift));
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads)
        for (size_t i = 0; i < m; i++) {
            const int8_t* r = x + i * d;
            int64_t best = INT64_MAX;
            uint32_t lab = 0;
            for (size_t j = 0; j < k; j++) {
                int32_t dot = 0;
                if (bits == 8) {
                    const int8_t* cj = &c8[j * d];
                    for (size_t t = 0; t < d; t++) dot += ((int32_t)r[t] + 128) * (int32_t)cj[t];
                } else {
                    const int16_t* cj = &c16[j * d];
                    for (size_t t = 0; t < d; t++) dot += (int32_t)r[t] * (int32_t)cj[t];
                }
                int64_t s = offset[j] - mult * (int64_t)dot;
                if (s < best) {
                    best = s;
                    lab = (uint32_t)j;
                }
            }
            int64_t norm = 0;
            for (size_t t = 0; t < d; t++) norm += (int64_t)r[t] * r[t];
            double v = std::fmax((double)norm + (double)best * inv_unit, 0.0);
            labels[i] = lab;
            dist[i] = (float)v;
        }
    }
};

int orc_i8_assign(int bits, const int8_t* x, size_t m, size_t d, const float* c, size_t k, const float* bias,
                  uint32_t* labels, float* dist, int threads) {
    I8Assigner a;
    a.bits = bits;
    if (a.set_centroids(c, k, d) != 0) return -1;
    if (bias) a.set_bias(bias);
    a.assign(x, m, labels, dist, threads);
    return 0;
}

// ---------------------------------------------------------------- FP64 brute force
// Exact nearest centroid in f64, lowest index on ties (the yardstick of label agreement).
void orc_bruteforce_f64(int dtype, const void* x, size_t m, size_t d, const float* c, size_t k, uint32_t* labels,
                        double* dist, int threads) {
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads)
    for (size_t i = 0; i < m; i++) {
        std::vector<double> r(d);
        for (size_t t = 0; t < d; t++) {
            if (dtype == 0) r[t] = ((const float*)x)[i * d + t];
            else if (dtype == 1) r[t] = ((const int8_t*)x)[i * d + t];
            else r[t] = ((const uint8_t*)x)[i * d + t];
        }
        double best = INFINITY;
        uint32_t lab = 0;
        for (size_t j = 0; j < k; j++) {
            double s = 0;
            const float* cj = c + j * d;
            for (size_t t = 0; t < d; t++) {
                double df = r[t] - (double)cj[t];
                s += df * df;
            }
            if (s < best) {
                best = s;
                lab = (uint32_t)j;
            }
        }
        labels[i] = lab;
        dist[i] = best;
    }
}

// ---------------------------------------------------------------- training
// State::apply, src/lib.rs:287-309.
static void state_apply(size_t k, size_t d, float* centroids, float* usage, const uint32_t* touched, size_t ntouched,
                        const uint32_t* counts, const float* sums, float alpha) {
    bool replace = alpha == 1.0f;
    if (!replace) {
        float decay = 1.0f - alpha;
        for (size_t j = 0; j < k; j++) usage[j] = usage[j] * decay;
    }
    for (size_t t = 0; t < ntouched; t++) {
        size_t j = touched[t];
        float n = (float)counts[j];
        float retained = replace ? 0.0f : usage[j];
        float mass = retained + alpha * n;
        float weight = alpha * n / mass;
        float* c = centroids + j * d;
        const float* s = sums + j * d;
        if (weight == 1.0f) {
            for (size_t i = 0; i < d; i++) c[i] = s[i] / n;
        } else {
            for (size_t i = 0; i < d; i++) c[i] = c[i] + weight * (s[i] / n - c[i]);
        }
        usage[j] = mass;
    }
}

void orc_state_apply(size_t k, size_t d, float* centroids, float* usage, const uint32_t* touched, size_t ntouched,
                     const uint32_t* counts, const float* sums, float alpha) {
    state_apply(k, d, centroids, usage, touched, ntouched, counts, sums, alpha);
}

// State::revive, src/lib.rs:314-344. Returns the number of splits.
static size_t state_revive(size_t k, size_t d, float* centroids, float* usage, float tau, Rng& rng) {
    float total = -0.0f;
    for (size_t j = 0; j < k; j++) total = total + usage[j];
    float threshold = total * tau / (float)k;
    std::vector<size_t> unused;
    for (size_t j = 0; j < k; j++)
        if (usage[j] < threshold) unused.push_back(j);
    if (unused.empty()) return 0;
    std::vector<std::pair<double, size_t>> donors;
    for (size_t j = 0; j < k; j++)
        if (usage[j] >= threshold && usage[j] > 0.0f)
            donors.push_back({std::log((double)usage[j]) - std::log(-std::log(rng.open01())), j});
    size_t nsplit = std::min(unused.size(), donors.size());
    std::sort(donors.begin(), donors.end(),
              [](const std::pair<double, size_t>& a, const std::pair<double, size_t>& b) { return a.first > b.first; });
    for (size_t p = 0; p < nsplit; p++) {
        size_t src = donors[p].second, dst = unused[p];
        float half = usage[src] / 2.0f;
        for (size_t i = 0; i < d; i++) {
            float offset = (i % 2 == 0) ? SPLIT_EPSILON : -SPLIT_EPSILON;
            float c = centroids[src * d + i];
            centroids[src * d + i] = c * (1.0f - offset);
            centroids[dst * d + i] = c * (1.0f + offset);
        }
        bool same = true;
        for (size_t i = 0; i < d; i++)
            if (centroids[src * d + i] != centroids[dst * d + i]) {
                same = false;
                break;
            }
        if (same) centroids[dst * d] = std::nextafter(centroids[dst * d], INFINITY);
        usage[src] = half;
        usage[dst] = half;
    }
    return nsplit;
}

size_t orc_state_revive(size_t k, size_t d, float* centroids, float* usage, float tau, uint64_t rng_seed) {
    Rng rng(rng_seed);
    return state_revive(k, d, centroids, usage, tau, rng);
}

// train, src/lib.rs:348-491. assigner: 0 = CpuAssigner (kernel as in
// orc_cpu_assign), 1 = CpuI8Assigner(I8), 2 = CpuI8Assigner(I16); the int8
// assigners need dtype 1 (i8 rows).
// Outputs: centroids k*d, labels n, objective (n_epochs), *n_splits.
int orc_train(int dtype, const void* x, size_t n, size_t d, size_t k, const orc_config* cfg, int assigner, int kernel,
              int threads, float* out_centroids, uint32_t* out_labels, double* out_objective, uint64_t* out_n_splits) {
    if (d == 0 || k == 0) return -1;
    if (n < k) return -2;
    if (n > 0xFFFFFFFFull) return -3;
    if (!(cfg->nepochs > 0.0)) return -4;
    if (assigner != 0 && dtype != 1) return -5;
    orc_recipe rec;
    std::vector<uint64_t> er_buf((size_t)std::floor(cfg->nepochs) + 2);
    orc_resolve_recipe(n, d, k, cfg, &rec, er_buf.data(), er_buf.size());
    std::vector<size_t> er(er_buf.begin(), er_buf.begin() + rec.n_epochs);
    size_t batch = rec.batch_size;
    size_t esz = dtype == 0 ? 4 : 1;
    const uint8_t* xb = (const uint8_t*)x;

    std::vector<float> centroids(k * d), usage(k, INIT_USAGE);
    {
        std::vector<uint32_t> init(n);
        Rng(cfg->seed).permutation(n, init.data());
        for (size_t j = 0; j < k; j++) widen(dtype, xb + (size_t)init[j] * d * esz, d, &centroids[j * d]);
    }
    Rng split_rng(cfg->seed ^ 0x5EED5EED5EED5EEDull);
    size_t n_splits = 0;

    CpuAssigner fa;
    fa.kernel = kernel & 7;
    fa.emulate = (kernel & 8) != 0;
    if (assigner == 0 && !fa.emulate && !cpu_has(fa.kernel)) return -6;
    I8Assigner ia;
    ia.bits = assigner == 2 ? 16 : 8;

    size_t chunk = std::min(ASSIGN_CHUNK, batch);
    std::vector<float> rows(chunk * d);
    std::vector<int8_t> rows8(assigner != 0 ? chunk * d : 0);
    std::vector<uint32_t> chunk_labels(chunk);
    std::vector<float> chunk_dist(chunk);
    std::vector<uint32_t> counts(k, 0);
    std::vector<float> sums(k * d, 0.0f);
    std::vector<uint32_t> touched;
    std::vector<uint32_t> labels(n, 0xFFFFFFFFu);
    std::vector<double> objective;
    std::vector<uint64_t> pass_counts(k, 0);
    std::vector<float> pass_sums;
    std::vector<float> bias(cfg->balance > 0.0f ? k : 0, 0.0f);
    double mean_sqdist = 0.0;
    size_t step = 0;
    size_t last = er.size() - 1;
    std::vector<uint32_t> order(n);

    for (size_t epoch = 0; epoch < er.size(); epoch++) {
        size_t epoch_n = er[epoch];
        Rng(cfg->seed * 1000003ull + (uint64_t)epoch + 1).permutation(n, order.data());
        bool is_last = epoch == last;
        if (is_last) {
            std::fill(pass_counts.begin(), pass_counts.end(), 0);
            pass_sums.assign(k * d, 0.0f);
        }
        double epoch_obj = 0.0;
        for (size_t b0 = 0; b0 < epoch_n; b0 += batch) {
            size_t bn = std::min(batch, epoch_n - b0);
            const uint32_t* ids = order.data() + b0;
            if (assigner == 0) fa.set_centroids(centroids.data(), k, d);
            else if (ia.set_centroids(centroids.data(), k, d) != 0) return -7;
            bool penalized = cfg->balance > 0.0f && mean_sqdist > 0.0;
            if (penalized) {
                double mm = -0.0;
                for (size_t j = 0; j < k; j++) mm += (double)usage[j];
                double mean_mass = mm / (double)k;
                float scale = (float)((double)cfg->balance * mean_sqdist / mean_mass);
                for (size_t j = 0; j < k; j++) bias[j] = scale * usage[j];
                if (assigner == 0) fa.set_bias(bias.data());
                else ia.set_bias(bias.data());
            }
            double batch_obj = 0.0;
            for (size_t p0 = 0; p0 < bn; p0 += chunk) {
                size_t m = std::min(chunk, bn - p0);
                const uint32_t* part = ids + p0;
                for (size_t r = 0; r < m; r++) {
                    const uint8_t* src = xb + (size_t)part[r] * d * esz;
                    widen(dtype, src, d, &rows[r * d]);
                    if (assigner != 0) std::memcpy(&rows8[r * d], src, d);
                }
                if (assigner == 0) fa.assign(rows.data(), m, chunk_labels.data(), chunk_dist.data(), threads);
                else ia.assign(rows8.data(), m, chunk_labels.data(), chunk_dist.data(), threads);
                if (penalized)
                    for (size_t r = 0; r < m; r++)
                        chunk_dist[r] = std::fmax(chunk_dist[r] - bias[chunk_labels[r]], 0.0f);
                for (size_t r = 0; r < m; r++) {
                    size_t l = chunk_labels[r];
                    if (counts[l] == 0) touched.push_back((uint32_t)l);
                    counts[l] += 1;
                    float* s = &sums[l * d];
                    const float* v = &rows[r * d];
                    for (size_t t = 0; t < d; t++) s[t] = s[t] + v[t];
                    if (is_last) labels[part[r]] = (uint32_t)l;
                }
                double cs = -0.0;
                for (size_t r = 0; r < m; r++) cs += (double)chunk_dist[r];
                batch_obj += cs;
            }
            epoch_obj += batch_obj;
            mean_sqdist = batch_obj / (double)bn;
            if (is_last)
                for (uint32_t j : touched) {
                    pass_counts[j] += counts[j];
                    for (size_t t = 0; t < d; t++) pass_sums[j * d + t] = pass_sums[j * d + t] + sums[j * d + t];
                }
            float alpha = (float)orc_scheduled_alpha(rec.alpha0, step, rec.total_steps);
            state_apply(k, d, centroids.data(), usage.data(), touched.data(), touched.size(), counts.data(),
                        sums.data(), alpha);
            for (uint32_t j : touched) {
                counts[j] = 0;
                std::fill(&sums[(size_t)j * d], &sums[(size_t)j * d] + d, 0.0f);
            }
            touched.clear();
            if ((step + 1) % CHECK_UNUSED_EVERY == 0 && rec.unused_threshold > 0.0f)
                n_splits += state_revive(k, d, centroids.data(), usage.data(), rec.unused_threshold, split_rng);
            step++;
        }
        objective.push_back(epoch_obj);
    }
    // Closing mean, src/lib.rs:483-489.
    for (size_t j = 0; j < k; j++)
        if (pass_counts[j] > 0) {
            float inv = 1.0f / (float)pass_counts[j];
            for (size_t t = 0; t < d; t++) centroids[j * d + t] = pass_sums[j * d + t] * inv;
        }
    std::memcpy(out_centroids, centroids.data(), k * d * sizeof(float));
    std::memcpy(out_labels, labels.data(), n * sizeof(uint32_t));
    for (size_t e = 0; e < objective.size(); e++) out_objective[e] = objective[e];
    *out_n_splits = n_splits;
    return 0;
}

// balance_stats, src/lib.rs:497-504.
void orc_balance_stats(const uint32_t* labels, size_t n, size_t k, double* out3) {
    std::vector<uint64_t> counts(k, 0);
    for (size_t i = 0; i < n; i++) counts[labels[i]]++;
    double sq = 0;
    uint64_t mx = 0, empty = 0;
    for (size_t j = 0; j < k; j++) {
        sq += (double)(counts[j] * counts[j]);
        mx = std::max(mx, counts[j]);
        empty += counts[j] == 0;
    }
    double nn = (double)n;
    out3[0] = (double)k * sq / (nn * nn);
    out3[1] = (double)mx * (double)k / nn;
    out3[2] = (double)empty;
}

// ---------------------------------------------------------------- quantizer
// Int8Quantizer::fit, src/quantize.rs:45-62.
void orc_quantizer_fit(const float* sample, size_t n, size_t d, float target_peak, double quantile, int power_of_two,
                       float* shift, float* scale_out) {
    std::vector<double> mean(d, 0.0);
    for (size_t i = 0; i < n; i++)
        for (size_t t = 0; t < d; t++) mean[t] += (double)sample[i * d + t];
    for (size_t t = 0; t < d; t++) shift[t] = (float)(mean[t] / (double)n);
    std::vector<float> mags(n * d);
    for (size_t i = 0; i < n; i++)
        for (size_t t = 0; t < d; t++) mags[i * d + t] = std::fabs(sample[i * d + t] - shift[t]);
    // ((len - 1) as f64 * quantile.clamp(0, 1)).round() as usize: NaN -> 0
    double q = std::isnan(quantile) ? 0.0 : std::min(std::max(quantile, 0.0), 1.0);
    size_t idx = (size_t)std::round((double)(mags.size() - 1) * q);
    // select_nth_unstable_by(idx, f32::total_cmp): order by the sign-folded bit pattern
    auto total_key = [](float v) {
        int32_t b;
        std::memcpy(&b, &v, 4);
        return b ^ (int32_t)((uint32_t)(b >> 31) >> 1);
    };
    std::nth_element(mags.begin(), mags.begin() + idx, mags.end(),
                     [&](float a, float b) { return total_key(a) < total_key(b); });
    float peak = mags[idx];
    float scale = peak > 0.0f ? target_peak / peak : 1.0f;
    if (power_of_two) {
        // 2f32.powi(scale.log2().floor() as i32): saturating cast, NaN -> 0
        float l = std::floor(std::log2(scale));
        int e = std::isnan(l) ? 0 : l >= 2147483647.0f ? INT32_MAX : l <= -2147483648.0f ? INT32_MIN : (int)l;
        // powi forms 2^|e| by repeated squaring (inf from 2^128 on), then 1 / 2^|e| for e < 0
        if (e >= 128) scale = INFINITY;
        else if (e >= 0) scale = std::ldexp(1.0f, e);
        else if (e > -128) scale = 1.0f / std::ldexp(1.0f, -e);
        else scale = 0.0f;
    }
    *scale_out = scale;
}

// Int8Quantizer::encode, src/quantize.rs:65-73.
void orc_quantizer_encode(const float* x, size_t n, size_t d, const float* shift, float scale, int8_t* out) {
    for (size_t i = 0; i < n; i++)
        for (size_t t = 0; t < d; t++) {
            float v = (x[i * d + t] - shift[t]) * scale;
            if (std::isnan(v)) {
                out[i * d + t] = 0;
                continue;
            }
            float r = std::min(std::max(std::round(v), -128.0f), 127.0f);
            out[i * d + t] = (int8_t)r;
        }
}

// Int8Quantizer::clipped_fraction numerator, src/quantize.rs:87-95: values whose
// scaled centred value lies outside [-128.5, 127.5) (NaN included).
uint64_t orc_quantizer_clipped(const float* x, size_t n, size_t d, const float* shift, float scale) {
    uint64_t c = 0;
    for (size_t i = 0; i < n; i++)
        for (size_t t = 0; t < d; t++) {
            float v = (x[i * d + t] - shift[t]) * scale;
            if (!(v >= -128.5f && v < 127.5f)) c++;
        }
    return c;
}

// Int8Quantizer::decode, src/quantize.rs:76-79.
void orc_quantizer_decode(const float* codes, size_t n, size_t d, const float* shift, float scale, float* out) {
    float inv = 1.0f / scale;
    for (size_t i = 0; i < n; i++)
        for (size_t t = 0; t < d; t++) out[i * d + t] = codes[i * d + t] * inv + shift[t];
}

// ---------------------------------------------------------------- report
// report(), src/report.rs:83-241. Cluster fields in declaration order
// (src/report.rs:37-56).
struct OrcClusterStats {
    uint32_t size;
    float rms, median, mad, p90, p99, max, looseness;
    uint32_t nearest_centroid;
    float nearest_dist, isolation;
    uint32_t family;
};

static int32_t rep_total_key(float v) {  // f32::total_cmp as a signed integer order
    int32_t b;
    std::memcpy(&b, &v, 4);
    return b ^ (int32_t)((uint32_t)(b >> 31) >> 1);
}
static bool rep_less(float a, float b) { return rep_total_key(a) < rep_total_key(b); }

// quantile, src/report.rs:83-88
static float rep_quantile(const float* sorted, size_t len, double q) {
    if (len == 0) return 0.0f;
    return sorted[(size_t)std::round((double)(len - 1) * q)];
}

// median_mad, src/report.rs:91-96
static void rep_median_mad(const float* sorted, size_t len, float* med, float* mad) {
    *med = rep_quantile(sorted, len, 0.5);
    std::vector<float> dev(len);
    for (size_t i = 0; i < len; i++) dev[i] = std::fabs(sorted[i] - *med);
    std::sort(dev.begin(), dev.end(), rep_less);
    *mad = rep_quantile(dev.data(), len, 0.5);
}

// sqdist, src/report.rs:104-114: 16 lane accumulators over whole 16-chunks,
// a sequential tail, then the lanes summed in order and the tail added.
static float rep_sqdist(const float* a, const float* b, size_t d) {
    float acc[16] = {0};
    const size_t d16 = d / 16 * 16;
    float tail = 0.0f;
    for (size_t t = d16; t < d; t++) tail += (a[t] - b[t]) * (a[t] - b[t]);
    for (size_t c = 0; c < d16; c += 16)
        for (int i = 0; i < 16; i++) acc[i] += (a[c + i] - b[c + i]) * (a[c + i] - b[c + i]);
    float s = 0.0f;
    for (int i = 0; i < 16; i++) s += acc[i];
    return s + tail;
}

static float rep_max_ignoring_nan(float a, float b) { return std::isnan(a) ? b : std::isnan(b) ? a : (a > b ? a : b); }

// Equal-size clusters are ordered by index (the reference's sort_unstable_by_key
// leaves that order to its sort algorithm), and equal-size families by the order
// they were formed in.
void orc_report(const uint32_t* labels, const float* sq, size_t n, const float* c, size_t k, size_t d,
                float family_radius, size_t min_local_size, OrcClusterStats* clusters, float* local_z,
                float* global_z, float* medians, uint32_t* n_families, uint32_t* fam_leader, uint64_t* fam_size,
                double* fam_share, uint32_t* fam_offsets, uint32_t* fam_members) {
    std::vector<float> dist(n);
    for (size_t i = 0; i < n; i++) dist[i] = std::sqrt(rep_max_ignoring_nan(sq[i], 0.0f));
    std::vector<size_t> start(k + 1, 0);
    for (size_t i = 0; i < n; i++) start[labels[i] + 1]++;
    for (size_t j = 0; j < k; j++) start[j + 1] += start[j];
    std::vector<size_t> cursor(start.begin(), start.end() - 1);
    std::vector<float> grouped(n);
    for (size_t i = 0; i < n; i++) grouped[cursor[labels[i]]++] = dist[i];

    std::vector<float> all(dist);
    std::sort(all.begin(), all.end(), rep_less);
    float g_med, g_mad;
    rep_median_mad(all.data(), n, &g_med, &g_mad);
    const float g_scale = rep_max_ignoring_nan(1.4826f * g_mad, FLT_MIN);

    for (size_t j = 0; j < k; j++) {
        OrcClusterStats cs{};
        const size_t len = start[j + 1] - start[j];
        if (len) {
            std::vector<float> m(grouped.begin() + start[j], grouped.begin() + start[j + 1]);
            std::sort(m.begin(), m.end(), rep_less);
            rep_median_mad(m.data(), len, &cs.median, &cs.mad);
            double ss = 0.0;
            for (float v : m) ss += (double)v * (double)v;
            cs.size = (uint32_t)len;
            cs.rms = (float)std::sqrt(ss / (double)len);
            cs.p90 = rep_quantile(m.data(), len, 0.9);
            cs.p99 = rep_quantile(m.data(), len, 0.99);
            cs.max = m.back();
        }
        clusters[j] = cs;
    }

    // nearest other live centroid, src/report.rs:170-183
    std::vector<uint32_t> nj(k);
    std::vector<float> nd(k);
#pragma omp parallel for schedule(dynamic, 16)
    for (long i = 0; i < (long)k; i++) {
        uint32_t bj = (uint32_t)i;
        float bs = INFINITY;
        for (size_t j = 0; j < k; j++) {
            if (j == (size_t)i || clusters[j].size == 0) continue;
            const float s = rep_sqdist(c + i * d, c + j * d, d);
            if (s < bs) {
                bs = s;
                bj = (uint32_t)j;
            }
        }
        nj[i] = bj;
        nd[i] = std::sqrt(bs);
    }
    std::vector<float> rl, nl;
    for (size_t j = 0; j < k; j++)
        if (clusters[j].size) {
            rl.push_back(clusters[j].rms);
            nl.push_back(nd[j]);
        }
    std::sort(rl.begin(), rl.end(), rep_less);
    std::sort(nl.begin(), nl.end(), rep_less);
    const float median_rms = rep_quantile(rl.data(), rl.size(), 0.5);
    const float median_nearest = rep_quantile(nl.data(), nl.size(), 0.5);
    for (size_t j = 0; j < k; j++) {
        clusters[j].nearest_centroid = nj[j];
        clusters[j].nearest_dist = nd[j];
        clusters[j].looseness = clusters[j].rms / rep_max_ignoring_nan(median_rms, FLT_MIN);
        clusters[j].isolation = nd[j] / rep_max_ignoring_nan(median_nearest, FLT_MIN);
    }

    // families, src/report.rs:198-223
    const float radius = family_radius * median_nearest;
    std::vector<size_t> order;
    for (size_t j = 0; j < k; j++)
        if (clusters[j].size) order.push_back(j);
    std::stable_sort(order.begin(), order.end(),
                     [&](size_t a, size_t b) { return clusters[a].size > clusters[b].size; });
    std::vector<uint32_t> family_of(k, UINT32_MAX);
    std::vector<uint32_t> lead_of;
    std::vector<uint64_t> size_of;
    std::vector<std::vector<uint32_t>> members;
    for (size_t lead : order) {
        if (family_of[lead] != UINT32_MAX) continue;
        std::vector<uint32_t> joins;
        for (size_t j : order)
            if (family_of[j] == UINT32_MAX &&
                (j == lead || std::sqrt(rep_sqdist(c + lead * d, c + j * d, d)) <= radius))
                joins.push_back((uint32_t)j);
        uint64_t size = 0;
        for (uint32_t j : joins) {
            family_of[j] = (uint32_t)lead_of.size();
            size += clusters[j].size;
        }
        lead_of.push_back((uint32_t)lead);
        size_of.push_back(size);
        members.push_back(joins);
    }
    std::vector<size_t> rank(lead_of.size());
    for (size_t f = 0; f < rank.size(); f++) rank[f] = f;
    std::stable_sort(rank.begin(), rank.end(), [&](size_t a, size_t b) { return size_of[a] > size_of[b]; });
    size_t off = 0;
    fam_offsets[0] = 0;
    for (size_t f = 0; f < rank.size(); f++) {
        const size_t g = rank[f];
        fam_leader[f] = lead_of[g];
        fam_size[f] = size_of[g];
        fam_share[f] = (double)size_of[g] / (double)n;
        for (uint32_t j : members[g]) {
            fam_members[off++] = j;
            clusters[j].family = (uint32_t)f;
        }
        fam_offsets[f + 1] = (uint32_t)off;
    }
    *n_families = (uint32_t)rank.size();

    for (size_t i = 0; i < n; i++) {
        const float gz = (dist[i] - g_med) / g_scale;
        global_z[i] = gz;
        const OrcClusterStats& cs = clusters[labels[i]];
        local_z[i] = ((size_t)cs.size < min_local_size || cs.mad <= 0.0f) ? gz : (dist[i] - cs.median) / (1.4826f * cs.mad);
    }
    medians[0] = g_med;
    medians[1] = median_rms;
    medians[2] = median_nearest;
}

}  // extern "C"
