// Int8 quantizer on the device: the fit (per-dimension mean shift and the
// peak of the centred magnitudes) and the encode / clipped count / decode of
// Int8Quantizer (src/quantize.rs:45-96), bit-exact with the reference.
//
// Exactness notes, per step of Int8Quantizer::fit (src/quantize.rs:45-62):
//  * mean: the reference adds the rows in order into one f64 accumulator per
//    dimension (`:48-51`). f64 addition is not associative, so a tree reduction
//    could differ in the last bit; k_quant_colsum keeps the row order, one
//    accumulator per dimension, and streams rows into shared memory by cp.async
//    several stages ahead so that the chain of dependent adds sets its pace.
//  * peak: `select_nth_unstable_by(idx, f32::total_cmp)` over |x - shift|
//    (`:53-56`). Every magnitude has a clear sign bit, so total_cmp is the
//    unsigned order of the bit patterns (NaNs above +inf); the select is a
//    three-pass radix select on those bit patterns (11 + 10 + 10 bits), or one
//    max / min reduction when idx is the last / first rank.
//  * encode: `((v - s) * scale).round().clamp(-128, 127) as i8` (`:65-73`):
//    two separately rounded f32 operations, round half away from zero, and the
//    saturating cast that sends NaN to 0.
#pragma once
#include <cstdint>

#include "common.cuh"

namespace emb {

constexpr int kQsumRows = 256;     // rows per shared-memory stage of the column sums
constexpr int kQsumStages = 4;     // stages in flight (cp.async groups)
constexpr int kQsumThreads = 256;  // all threads copy; warp 0 sums
constexpr int kQThreads = 512;     // element-wise passes
constexpr int kQBins0 = 2048;      // bits 30..20 of a magnitude (bit 31 is always clear)
constexpr int kQBins = 1024;       // bits 19..10, then bits 9..0

struct QuantSelect {
    unsigned long long rank;  // rank still to find inside the current prefix
    unsigned int prefix;      // bit pattern chosen so far (the peak after the last pass)
    unsigned int pad;
    unsigned long long hist[kQBins0];
};

__device__ __forceinline__ void qs_cp_async16(float* smem, const float* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void qs_cp_async4(float* smem, const float* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void qs_cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void qs_cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Per-dimension f64 sums in row order, then shift = (f32)(sum / n)
// (src/quantize.rs:48-52). One CTA per 32 consecutive dimensions; lane t of
// warp 0 owns dimension c0 + t and adds its values in row order. Rows arrive
// in 256-row stages by cp.async, kQsumStages - 1 stages ahead of the sums (16-
// byte copies when d % 4 == 0, else 4-byte copies). Dynamic shared memory:
// kQsumStages x kQsumRows x 32 floats.
__global__ void __launch_bounds__(kQsumThreads) k_quant_colsum(const float* __restrict__ x, size_t n, size_t d,
                                                               float* __restrict__ shift) {
    extern __shared__ __align__(16) float qs_stage[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const size_t c0 = (size_t)blockIdx.x * 32;
    const size_t nchunks = (n + kQsumRows - 1) / kQsumRows;
    const bool vec = (d & 3) == 0;
    auto issue = [&](size_t chunk) {
        if (chunk < nchunks) {
            const size_t r0 = chunk * kQsumRows;
            float* dst = qs_stage + (chunk % kQsumStages) * (kQsumRows * 32);
            if (vec) {  // 8 x 16 bytes per row slice
                for (int e = tid; e < kQsumRows * 8; e += kQsumThreads) {
                    const int r = e >> 3, q = e & 7;
                    const size_t row = r0 + r, col = c0 + 4 * q;
                    if (row < n && col < d) qs_cp_async16(dst + r * 32 + 4 * q, x + row * d + col);
                }
            } else {
                for (int e = tid; e < kQsumRows * 32; e += kQsumThreads) {
                    const int r = e >> 5, t = e & 31;
                    const size_t row = r0 + r, col = c0 + t;
                    if (row < n && col < d) qs_cp_async4(dst + r * 32 + t, x + row * d + col);
                }
            }
        }
        qs_cp_commit();  // an empty group past the end keeps the group count uniform
    };
#pragma unroll
    for (int s = 0; s < kQsumStages - 1; s++) issue(s);
    double acc = 0.0;
    for (size_t c = 0; c < nchunks; c++) {
        issue(c + kQsumStages - 1);
        qs_cp_wait<kQsumStages - 1>();  // this thread's copies of chunk c have landed
        __syncthreads();                  // everyone's have
        if (warp == 0) {
            const float* src = qs_stage + (c % kQsumStages) * (kQsumRows * 32);
            const int rows = (int)min((size_t)kQsumRows, n - c * kQsumRows);
            int r = 0;
            for (; r + 16 <= rows; r += 16) {  // loads ahead of the dependent adds
                float v[16];
#pragma unroll
                for (int i = 0; i < 16; i++) v[i] = src[(r + i) * 32 + lane];
#pragma unroll
                for (int i = 0; i < 16; i++) acc = __dadd_rn(acc, (double)v[i]);
            }
            for (; r < rows; r++) acc = __dadd_rn(acc, (double)src[r * 32 + lane]);
        }
        __syncthreads();  // the stage is free before it is refilled
    }
    qs_cp_wait<0>();
    if (warp == 0 && c0 + lane < d) shift[c0 + lane] = __double2float_rn(__ddiv_rn(acc, (double)n));
}

// The element-wise passes visit elements e = 4 * t + j * S (t the global thread
// index, S = 4 x threads in the grid). The host sizes the grid so that S is a
// multiple of d: a thread's four dimensions, and so its four shifts, never change.
__device__ __forceinline__ unsigned int quant_mag_bits(float v, float s) {
    return __float_as_uint(fabsf(__fsub_rn(v, s)));
}

// pass 0: histogram of bits 30..20; pass 1: of bits 19..10 among magnitudes whose
// bits 30..20 are sel->prefix; pass 2: of bits 9..0 among those matching bits 30..10.
template <int PASS>
__global__ void __launch_bounds__(kQThreads) k_quant_hist(const float* __restrict__ x, size_t N, size_t d,
                                                          const float* __restrict__ shift, QuantSelect* sel) {
    constexpr int NB = PASS == 0 ? kQBins0 : kQBins;
    __shared__ unsigned int h[NB];
    for (int i = threadIdx.x; i < NB; i += blockDim.x) h[i] = 0;
    const unsigned int prefix = PASS == 0 ? 0u : sel->prefix;
    __syncthreads();
    auto count = [&](unsigned int bits) {
        if (PASS == 0) {
            atomicAdd(&h[bits >> 20], 1u);
        } else if (PASS == 1) {
            if ((bits >> 20) == prefix) atomicAdd(&h[(bits >> 10) & 1023u], 1u);
        } else {
            if ((bits >> 10) == prefix) atomicAdd(&h[bits & 1023u], 1u);
        }
    };
    const size_t nthr = (size_t)gridDim.x * blockDim.x;
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t N4 = N / 4, S4 = nthr;
    if (t < N4) {
        float s[4];
#pragma unroll
        for (int i = 0; i < 4; i++) s[i] = shift[(4 * t + i) % d];
        const float4* x4 = reinterpret_cast<const float4*>(x);
        for (size_t g = t; g < N4; g += S4) {
            const float4 v = __ldg(x4 + g);
            count(quant_mag_bits(v.x, s[0]));
            count(quant_mag_bits(v.y, s[1]));
            count(quant_mag_bits(v.z, s[2]));
            count(quant_mag_bits(v.w, s[3]));
        }
    }
    if (t < N - 4 * N4) {  // the last N % 4 elements
        const size_t e = 4 * N4 + t;
        count(quant_mag_bits(x[e], shift[e % d]));
    }
    __syncthreads();
    for (int i = threadIdx.x; i < NB; i += blockDim.x)
        if (h[i]) atomicAdd(&sel->hist[i], (unsigned long long)h[i]);
}

// One warp: find the bin holding rank `rank` (pass 0: the rank passed in; later
// passes: sel->rank), extend the prefix by it, keep the rank within that bin and
// clear the histogram for the next pass.
__global__ void k_quant_pick(QuantSelect* sel, int pass, unsigned long long rank0) {
    const int lane = threadIdx.x;
    const int nb = pass == 0 ? kQBins0 : kQBins, per = nb / 32;
    unsigned long long rank = pass == 0 ? rank0 : sel->rank;
    unsigned long long mine = 0;
    for (int i = 0; i < per; i++) mine += sel->hist[lane * per + i];
    unsigned long long incl = mine;
    for (int o = 1; o < 32; o <<= 1) {
        unsigned long long v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    const unsigned long long excl = incl - mine;
    const unsigned int hit = __ballot_sync(0xffffffffu, incl > rank);
    const int owner = hit ? __ffs(hit) - 1 : 31;
    int bin = nb - 1;
    unsigned long long below = 0;
    if (lane == owner) {
        unsigned long long cum = excl;
        bin = lane * per + per - 1;
        for (int i = 0; i < per; i++) {
            const unsigned long long c = sel->hist[lane * per + i];
            if (cum + c > rank) {
                bin = lane * per + i;
                break;
            }
            cum += c;
        }
        below = cum;
    }
    bin = __shfl_sync(0xffffffffu, bin, owner);
    below = __shfl_sync(0xffffffffu, below, owner);
    __syncwarp();
    for (int i = lane; i < nb; i += 32) sel->hist[i] = 0;
    if (lane == 0) {
        sel->prefix = pass == 0 ? (unsigned int)bin : (sel->prefix << 10) | (unsigned int)bin;
        sel->rank = rank - below;
    }
}

// The largest (MAX) or smallest magnitude's bit pattern into sel->prefix, which
// the host initialises to 0 (MAX) or 0xffffffff (MIN).
template <bool MAX>
__global__ void __launch_bounds__(kQThreads) k_quant_extreme(const float* __restrict__ x, size_t N, size_t d,
                                                             const float* __restrict__ shift, QuantSelect* sel) {
    unsigned int best = MAX ? 0u : 0xffffffffu;
    auto take = [&](unsigned int b) { best = MAX ? max(best, b) : min(best, b); };
    const size_t nthr = (size_t)gridDim.x * blockDim.x;
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t N4 = N / 4;
    if (t < N4) {
        float s[4];
#pragma unroll
        for (int i = 0; i < 4; i++) s[i] = shift[(4 * t + i) % d];
        const float4* x4 = reinterpret_cast<const float4*>(x);
        for (size_t g = t; g < N4; g += nthr) {
            const float4 v = __ldg(x4 + g);
            take(quant_mag_bits(v.x, s[0]));
            take(quant_mag_bits(v.y, s[1]));
            take(quant_mag_bits(v.z, s[2]));
            take(quant_mag_bits(v.w, s[3]));
        }
    }
    if (t < N - 4 * N4) {
        const size_t e = 4 * N4 + t;
        take(quant_mag_bits(x[e], shift[e % d]));
    }
    for (int o = 16; o; o >>= 1) {
        const unsigned int v = __shfl_xor_sync(0xffffffffu, best, o);
        best = MAX ? max(best, v) : min(best, v);
    }
    if ((threadIdx.x & 31) == 0) {
        if (MAX) atomicMax(&sel->prefix, best);
        else atomicMin(&sel->prefix, best);
    }
}

// One code, and whether the value clips: src/quantize.rs:69 and :91.
__device__ __forceinline__ int quant_code(float v, float s, float scale, unsigned int& clipped) {
    const float y = __fmul_rn(__fsub_rn(v, s), scale);
    clipped += !(y >= -128.5f && y < 127.5f);
    if (y != y) return 0;  // NaN: the saturating cast gives 0
    return (int)fminf(fmaxf(roundf(y), -128.f), 127.f);
}

// Encode 16 elements per thread and step (four float4 loads, one 16-byte store);
// the host sizes the grid so that 16 x threads in the grid is a multiple of d.
// codes may be null (count only); clipped may be null (codes only).
__global__ void __launch_bounds__(kQThreads) k_quant_encode(const float* __restrict__ x, size_t N, size_t d,
                                                            const float* __restrict__ shift, float scale,
                                                            int8_t* __restrict__ codes,
                                                            unsigned long long* __restrict__ clipped) {
    const size_t nthr = (size_t)gridDim.x * blockDim.x;
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t N16 = N / 16;
    unsigned int clip = 0;
    if (t < N16) {
        float s[16];
#pragma unroll
        for (int i = 0; i < 16; i++) s[i] = shift[(16 * t + i) % d];
        const float4* x4 = reinterpret_cast<const float4*>(x);
        for (size_t g = t; g < N16; g += nthr) {
            float v[16];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const float4 f = __ldcs(x4 + 4 * g + q);
                v[4 * q] = f.x;
                v[4 * q + 1] = f.y;
                v[4 * q + 2] = f.z;
                v[4 * q + 3] = f.w;
            }
            uint32_t w[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                uint32_t packed = 0;
#pragma unroll
                for (int i = 0; i < 4; i++)
                    packed |= (uint32_t)(quant_code(v[4 * q + i], s[4 * q + i], scale, clip) & 0xff) << (8 * i);
                w[q] = packed;
            }
            if (codes) __stcs(reinterpret_cast<uint4*>(codes) + g, make_uint4(w[0], w[1], w[2], w[3]));
        }
    }
    if (t < N - 16 * N16) {
        const size_t e = 16 * N16 + t;
        const int c = quant_code(x[e], shift[e % d], scale, clip);
        if (codes) codes[e] = (int8_t)c;
    }
    if (clipped) {
        for (int o = 16; o; o >>= 1) clip += __shfl_xor_sync(0xffffffffu, clip, o);
        if ((threadIdx.x & 31) == 0 && clip) atomicAdd(clipped, (unsigned long long)clip);
    }
}

// Int8Quantizer::decode, src/quantize.rs:76-79: v * (1 / scale) + s, two
// separately rounded operations (inv is the host's correctly rounded 1 / scale).
__global__ void k_quant_decode(const float* __restrict__ codes, size_t N, size_t d, const float* __restrict__ shift,
                               float inv, float* __restrict__ out) {
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < N; e += (size_t)gridDim.x * blockDim.x)
        out[e] = __fadd_rn(__fmul_rn(codes[e], inv), shift[e % d]);
}

}  // namespace emb
