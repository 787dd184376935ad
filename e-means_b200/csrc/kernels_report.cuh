// report() on the device (src/report.rs:121-241): per-cluster distance
// statistics, corpus medians, nearest other centroid, prototype families and
// the per-row z-scores, bit-exact with the reference's f32 / f64 arithmetic.
//
// Building blocks:
//  * an LSD radix sort of 64-bit keys (8-bit digits, stable scatter by warp
//    match + per-warp digit counts). Rows are sorted by (label, distance) keys
//    whose low word is the distance's f32::total_cmp order, so each cluster's
//    distances come out ascending exactly as the reference's per-cluster
//    sort_unstable_by(total_cmp) leaves them (equal floats are interchangeable);
//  * a radix select on 32-bit order keys (12 + 10 + 10 bits) for the corpus
//    median and MAD and the medians over clusters;
//  * k_rep_pairs: the exact O(k^2 d) pair pass in the reference's sqdist
//    rounding (src/report.rs:104-114), as a nearest-other-centroid search or as
//    the adjacency bitset of the families' radius test;
//  * k_rep_families: the greedy family pass (src/report.rs:198-216) in one CTA.
#pragma once
#include <cfloat>
#include <cstdint>

#include "common.cuh"

namespace emb {

constexpr int kRsThreads = 512;
constexpr int kRsRounds = 8;
constexpr int kRsTile = kRsThreads * kRsRounds;  // keys per block and pass
constexpr int kRsWarps = kRsThreads / 32;
constexpr int kSelBins0 = 4096;                  // bits 31..20 of an order key

// f32::total_cmp as an unsigned order, and back.
__device__ __forceinline__ uint32_t ord_f32(float v) {
    const uint32_t b = __float_as_uint(v);
    return b ^ ((b >> 31) ? 0xffffffffu : 0x80000000u);
}
__device__ __forceinline__ float unord_f32(uint32_t u) {
    return __uint_as_float(u ^ ((u >> 31) ? 0x80000000u : 0xffffffffu));
}

// `((len - 1) as f64 * q).round() as usize` (src/report.rs:87).
__device__ __forceinline__ size_t rep_qidx(size_t len, double q) {
    return (size_t)round(__dmul_rn((double)(len - 1), q));
}

// ---- radix sort ------------------------------------------------------------

// Digit counts of each block's tile: hist[digit * nblocks + block].
__global__ void __launch_bounds__(kRsThreads) k_rs_upsweep(const unsigned long long* __restrict__ keys, size_t n,
                                                           int shift, uint32_t* __restrict__ hist, uint32_t nblocks) {
    __shared__ uint32_t cnt[256];
    if (threadIdx.x < 256) cnt[threadIdx.x] = 0;
    __syncthreads();
    const size_t base = (size_t)blockIdx.x * kRsTile;
#pragma unroll
    for (int r = 0; r < kRsRounds; r++) {
        const size_t i = base + (size_t)r * kRsThreads + threadIdx.x;
        if (i < n) atomicAdd(&cnt[(uint32_t)(keys[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    if (threadIdx.x < 256) hist[(size_t)threadIdx.x * nblocks + blockIdx.x] = cnt[threadIdx.x];
}

// One block per digit: exclusive scan of the digit's row of block counts in
// place; the row's total into row_total[digit].
__global__ void __launch_bounds__(1024) k_rs_scan(uint32_t* __restrict__ hist, uint32_t nblocks,
                                                  uint32_t* __restrict__ row_total) {
    __shared__ uint32_t ws[32];
    uint32_t* row = hist + (size_t)blockIdx.x * nblocks;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t carry = 0;
    for (uint32_t c0 = 0; c0 < nblocks; c0 += 1024) {
        const uint32_t i = c0 + threadIdx.x;
        const uint32_t v = i < nblocks ? row[i] : 0u;
        uint32_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) ws[warp] = x;
        __syncthreads();
        if (warp == 0) {
            uint32_t w = ws[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            ws[lane] = w;
        }
        __syncthreads();
        if (i < nblocks) row[i] = carry + (warp ? ws[warp - 1] : 0u) + x - v;
        carry += ws[31];
        __syncthreads();
    }
    if (threadIdx.x == 0) row_total[blockIdx.x] = carry;
}

// Stable scatter of one tile by the digit at `shift`. Keys are taken in index
// order (round-major, then thread): a key's place is its digit's base for the
// block, plus the keys of that digit in earlier rounds, earlier warps of this
// round and lower lanes of its warp.
__global__ void __launch_bounds__(kRsThreads) k_rs_downsweep(const unsigned long long* __restrict__ in,
                                                             unsigned long long* __restrict__ out, size_t n, int shift,
                                                             const uint32_t* __restrict__ hist,
                                                             const uint32_t* __restrict__ row_total, uint32_t nblocks) {
    __shared__ uint32_t base[256];
    __shared__ uint32_t tot[256];
    __shared__ uint32_t wc[kRsWarps][256];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid < 256) tot[tid] = row_total[tid];
    __syncthreads();
    if (warp == 0) {  // digit bases: exclusive scan of the 256 digit totals
        uint32_t v[8], s = 0;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            v[i] = tot[lane * 8 + i];
            s += v[i];
        }
        uint32_t x = s;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        uint32_t e = x - s;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            base[lane * 8 + i] = e;
            e += v[i];
        }
    }
    __syncthreads();
    if (tid < 256) base[tid] += hist[(size_t)tid * nblocks + blockIdx.x];
    const size_t tile = (size_t)blockIdx.x * kRsTile;
    const unsigned lower = (1u << lane) - 1u;
    for (int r = 0; r < kRsRounds; r++) {
        for (int i = tid; i < kRsWarps * 256; i += kRsThreads) (&wc[0][0])[i] = 0;
        __syncthreads();
        const size_t idx = tile + (size_t)r * kRsThreads + tid;
        const bool valid = idx < n;
        const unsigned long long key = valid ? in[idx] : 0ull;
        const uint32_t digit = valid ? ((uint32_t)(key >> shift) & 255u) : 256u + (uint32_t)lane;
        const unsigned peers = __match_any_sync(0xffffffffu, digit);
        const uint32_t wrank = __popc(peers & lower);
        if (valid && wrank == 0) wc[warp][digit] = __popc(peers);
        __syncthreads();
        if (tid < 256) {
            uint32_t run = 0;
#pragma unroll
            for (int w = 0; w < kRsWarps; w++) {
                const uint32_t c = wc[w][tid];
                wc[w][tid] = run;
                run += c;
            }
            tot[tid] = run;
        }
        __syncthreads();
        if (valid) out[base[digit] + wc[warp][digit] + wrank] = key;
        __syncthreads();
        if (tid < 256) base[tid] += tot[tid];
    }
}

// ---- radix select on 32-bit order keys --------------------------------------

struct RepSelect {
    unsigned long long rank;
    uint32_t prefix;  // after the last pick: the selected key
    uint32_t pad;
    unsigned long long hist[kSelBins0];
};

// pass 0: bits 31..20; pass 1: bits 19..10 of keys whose bits 31..20 match;
// pass 2: bits 9..0 of keys whose bits 31..10 match.
template <int PASS>
__global__ void __launch_bounds__(512) k_sel_hist(const uint32_t* __restrict__ keys, size_t n, RepSelect* sel) {
    constexpr int NB = PASS == 0 ? kSelBins0 : 1024;
    __shared__ uint32_t h[NB];
    for (int i = threadIdx.x; i < NB; i += blockDim.x) h[i] = 0;
    const uint32_t prefix = PASS == 0 ? 0u : sel->prefix;
    __syncthreads();
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t u = keys[i];
        if (PASS == 0) atomicAdd(&h[u >> 20], 1u);
        else if (PASS == 1) {
            if ((u >> 20) == prefix) atomicAdd(&h[(u >> 10) & 1023u], 1u);
        } else if ((u >> 10) == prefix) {
            atomicAdd(&h[u & 1023u], 1u);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < NB; i += blockDim.x)
        if (h[i]) atomicAdd(&sel->hist[i], (unsigned long long)h[i]);
}

// One warp: the bin holding the rank (pass 0: rank0, or *rank_dev when given),
// the prefix extended by it, the rank kept within the bin, the histogram cleared.
__global__ void k_sel_pick(RepSelect* sel, int pass, unsigned long long rank0) {
    const int lane = threadIdx.x;
    const int nb = pass == 0 ? kSelBins0 : 1024, per = nb / 32;
    const unsigned long long rank = pass == 0 ? rank0 : sel->rank;
    unsigned long long mine = 0;
    for (int i = 0; i < per; i++) mine += sel->hist[lane * per + i];
    unsigned long long incl = mine;
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    const unsigned int hit = __ballot_sync(0xffffffffu, incl > rank);
    const int owner = hit ? __ffs(hit) - 1 : 31;
    int bin = nb - 1;
    unsigned long long below = 0;
    if (lane == owner) {
        unsigned long long cum = incl - mine;
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
        sel->prefix = pass == 0 ? (uint32_t)bin : (sel->prefix << 10) | (uint32_t)bin;
        sel->rank = rank > below ? rank - below : 0;
    }
}

// ---- report kernels ---------------------------------------------------------

// dist = sqrt(max(sq, 0)) (src/report.rs:124; max ignores NaN, and -0 becomes
// +0 as the oracle's restatement has it); sort keys
// (label, order of dist) and order keys of dist. Labels >= k are counted in bad.
__global__ void k_rep_prep(const uint32_t* __restrict__ labels, const float* __restrict__ sq, size_t n, uint32_t k,
                           float* __restrict__ dist, unsigned long long* __restrict__ keys, uint32_t* __restrict__ gkeys,
                           unsigned int* __restrict__ bad) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        uint32_t l = labels[i];
        if (l >= k) {
            atomicAdd(bad, 1u);
            l = 0;
        }
        const float s = sq[i];
        const float v = __fsqrt_rn(s > 0.0f ? s : 0.0f);  // NaN and -0 give +0
        dist[i] = v;
        const uint32_t o = ord_f32(v);
        keys[i] = ((unsigned long long)l << 32) | o;
        gkeys[i] = o;
    }
}

// start[j] = first sorted position of label j (start[k] = n): every boundary
// between labels a < b fills start[a+1..b].
__global__ void k_rep_starts(const unsigned long long* __restrict__ sorted, size_t n, uint32_t k,
                             uint32_t* __restrict__ start) {
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p <= n; p += (size_t)gridDim.x * blockDim.x) {
        const long long a = p > 0 ? (long long)(sorted[p - 1] >> 32) : -1;
        const long long b = p < n ? (long long)(sorted[p] >> 32) : (long long)k;
        for (long long j = a + 1; j <= b; j++) start[j] = (uint32_t)p;
    }
}

// Per cluster (src/report.rs:145-166): size, median, p90, p99, max, and rms
// = sqrt(sum of v*v in f64, ascending order, / len) as f32.
__global__ void k_rep_stats(const unsigned long long* __restrict__ sorted, const uint32_t* __restrict__ start,
                            uint32_t k, float* __restrict__ med, float* __restrict__ p90, float* __restrict__ p99,
                            float* __restrict__ mx, float* __restrict__ rms) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= k) return;
    const size_t s = start[j], len = start[j + 1] - s;
    if (len == 0) {
        med[j] = p90[j] = p99[j] = mx[j] = rms[j] = 0.0f;
        return;
    }
    auto val = [&](size_t p) { return unord_f32((uint32_t)sorted[s + p]); };
    med[j] = val(rep_qidx(len, 0.5));
    p90[j] = val(rep_qidx(len, 0.9));
    p99[j] = val(rep_qidx(len, 0.99));
    mx[j] = val(len - 1);
    double ss = 0.0;
    for (size_t p = 0; p < len; p++) {
        const double v = (double)val(p);
        ss = __dadd_rn(ss, __dmul_rn(v, v));
    }
    rms[j] = __double2float_rn(__dsqrt_rn(__ddiv_rn(ss, (double)len)));
}

// (label, order of |v - median|) for every sorted member (src/report.rs:93).
__global__ void k_rep_devkeys(const unsigned long long* __restrict__ sorted, size_t n, const float* __restrict__ med,
                              unsigned long long* __restrict__ dkeys) {
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        const unsigned long long key = sorted[p];
        const uint32_t j = (uint32_t)(key >> 32);
        const float dev = fabsf(__fsub_rn(unord_f32((uint32_t)key), med[j]));
        dkeys[p] = ((unsigned long long)j << 32) | ord_f32(dev);
    }
}

__global__ void k_rep_mad(const unsigned long long* __restrict__ dsorted, const uint32_t* __restrict__ start, uint32_t k,
                          float* __restrict__ mad) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= k) return;
    const size_t s = start[j], len = start[j + 1] - s;
    mad[j] = len ? unord_f32((uint32_t)dsorted[s + rep_qidx(len, 0.5)]) : 0.0f;
}

// Order keys of |dist - median| with the median taken from a finished select.
__global__ void k_rep_gdev(const float* __restrict__ dist, size_t n, const RepSelect* __restrict__ sel,
                           uint32_t* __restrict__ keys) {
    const float m = unord_f32(sel->prefix);
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        keys[i] = ord_f32(fabsf(__fsub_rn(dist[i], m)));
}

// Scalars of the report kept on the device.
struct RepScalars {
    float g_med, g_mad, g_scale, median_rms, median_nearest, radius;
    uint32_t live, pad;
};

// Order keys of the live clusters' values (dead clusters: the largest key) and
// the live count.
__global__ void k_rep_live_keys(const uint32_t* __restrict__ start, uint32_t k, const float* __restrict__ v,
                                bool take_sqrt, uint32_t* __restrict__ keys, RepScalars* sc) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    bool live = false;
    if (j < k) {
        live = start[j + 1] > start[j];
        const float x = take_sqrt ? __fsqrt_rn(v[j]) : v[j];
        keys[j] = live ? ord_f32(x) : 0xffffffffu;
    }
    const unsigned b = __ballot_sync(0xffffffffu, live);
    if ((threadIdx.x & 31) == 0 && b && sc) atomicAdd(&sc->live, (uint32_t)__popc(b));
}

// Scalars from finished selects: which = 0 -> g_med, 1 -> g_mad (and g_scale),
// 2 -> median_rms, 3 -> median_nearest (and the families' radius). `empty`:
// the median of nothing, 0 (src/report.rs:84-86).
__global__ void k_rep_take(const RepSelect* __restrict__ sel, RepScalars* sc, int which, bool empty,
                           float family_radius) {
    const float v = empty ? 0.0f : unord_f32(sel->prefix);
    if (which == 0) sc->g_med = v;
    if (which == 1) {
        sc->g_mad = v;
        sc->g_scale = fmaxf(__fmul_rn(1.4826f, v), FLT_MIN);
    }
    if (which == 2) sc->median_rms = v;
    if (which == 3) {
        sc->median_nearest = v;
        sc->radius = __fmul_rn(family_radius, v);
    }
}

// Per-row z-scores (src/report.rs:225-238).
__global__ void k_rep_z(const uint32_t* __restrict__ labels, const float* __restrict__ dist, size_t n,
                        const uint32_t* __restrict__ start, const float* __restrict__ med,
                        const float* __restrict__ mad, const RepScalars* __restrict__ sc, unsigned long long min_local,
                        float* __restrict__ local_z, float* __restrict__ global_z) {
    const float gm = sc->g_med, gs = sc->g_scale;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float v = dist[i];
        const float gz = __fdiv_rn(__fsub_rn(v, gm), gs);
        global_z[i] = gz;
        const uint32_t l = labels[i];
        const unsigned long long size = start[l + 1] - start[l];
        const float m = mad[l];
        local_z[i] = (size < min_local || m <= 0.0f) ? gz : __fdiv_rn(__fsub_rn(v, med[l]), __fmul_rn(1.4826f, m));
    }
}

// ---- exact pair pass ---------------------------------------------------------

constexpr int kPairT = 32;         // rows and columns per tile
constexpr int kPairThreads = 256;  // each thread: rows {r, r+16} x columns {c, c+16} of the tile
constexpr int kPairDC = 64;        // dimensions per staged chunk
constexpr int kPairLd = kPairDC + 4;  // row pitch of a staged chunk (16-byte rows for cp.async)
constexpr int kPairStage = 2 * kPairT * kPairLd;  // floats of one stage (row tile chunk + column tile chunk)

constexpr size_t pair_smem_bytes() {
    return sizeof(float) * (2 * kPairStage + 2 * kPairT * 16) + kPairT * (sizeof(unsigned long long) + sizeof(uint32_t));
}

__device__ __forceinline__ void pair_cp16(float* smem, const float* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void pair_cp4(float* smem, const float* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}

// Exact squared distances of centroid pairs in the reference's sqdist rounding
// (src/report.rs:104-114): lane l of 16 accumulates (c_i[t] - c_j[t])^2 over
// t = l, l + 16, ... below d16 = d - d % 16 (separate subtract, multiply and
// add), the lanes are summed in order, then the tail (t >= d16, summed in
// order) is added. A thread keeps all 16 lane accumulators of its 4 pairs, so
// the ordered lane sum stays in registers. The result is the same for (i, j)
// and (j, i) (x - y and y - x square alike), so only tiles J >= I are
// computed; CTA b takes row tiles b and T-1-b, which balances the triangle.
// Dimension chunks of both tiles are double-buffered by cp.async.
//   NEAREST (ADJ = false): near_key[i] = min over live j != i with s < inf of
//   (bits of s, j), by 64-bit atomicMin (first j of the least s, as the
//   reference's strict < scan); the host initialises it to all ones.
//   ADJ: bit j of row i of the adjacency is set when both are live, j != i and
//   sqrt(s) <= radius; every word of every row is written.
template <bool ADJ>
__global__ void __launch_bounds__(kPairThreads, 2) k_rep_pairs(const float* __restrict__ c, uint32_t k, uint32_t d,
                                                               const uint32_t* __restrict__ start,
                                                               unsigned long long* __restrict__ near_key,
                                                               const RepScalars* __restrict__ sc,
                                                               uint32_t* __restrict__ adj, uint32_t words) {
    extern __shared__ __align__(16) float pair_sm[];
    float* stage = pair_sm;                  // 2 stages x (row chunk, column chunk)
    float* xt = stage + 2 * kPairStage;      // row tile tails [32][16]
    float* yt = xt + kPairT * 16;            // column tile tails
    unsigned long long* colkey = reinterpret_cast<unsigned long long*>(yt + kPairT * 16);
    uint32_t* colbits = reinterpret_cast<uint32_t*>(colkey + kPairT);
    const int tid = threadIdx.x, tr = tid >> 4, tc = tid & 15;  // rows tr, tr+16; columns tc, tc+16
    const uint32_t T = (k + kPairT - 1) / kPairT;
    const uint32_t d16 = d / 16 * 16, dt = d - d16;
    const uint32_t nchunk = (d16 + kPairDC - 1) / kPairDC;
    const bool vec = (d & 3) == 0;
    const float radius = ADJ ? sc->radius : 0.0f;
    const uint32_t b = blockIdx.x, I0 = b, I1 = T - 1 - b;
    const uint32_t n0 = (T - I0) * nchunk, n1 = I1 > I0 ? (T - I1) * nchunk : 0;
    auto coords = [&](uint32_t it, uint32_t& I, uint32_t& J, uint32_t& dc0) {
        const uint32_t base = it < n0 ? 0 : n0;
        I = it < n0 ? I0 : I1;
        const uint32_t r = it - base;
        J = I + r / nchunk;
        dc0 = (r % nchunk) * kPairDC;
    };
    auto issue = [&](uint32_t it) {
        if (it < n0 + n1) {
            uint32_t I, J, dc0;
            coords(it, I, J, dc0);
            float* xs = stage + (it & 1) * kPairStage;
            float* ys = xs + kPairT * kPairLd;
            if (vec) {
                for (int e = tid; e < 2 * kPairT * (kPairDC / 4); e += kPairThreads) {
                    const int side = e / (kPairT * (kPairDC / 4)), f = e % (kPairT * (kPairDC / 4));
                    const int r = f / (kPairDC / 4), q = f % (kPairDC / 4);
                    const uint32_t ci = (side ? J : I) * kPairT + r, dim = dc0 + 4 * q;
                    if (ci < k && dim < d16) pair_cp16((side ? ys : xs) + r * kPairLd + 4 * q, c + (size_t)ci * d + dim);
                }
            } else {
                for (int e = tid; e < 2 * kPairT * kPairDC; e += kPairThreads) {
                    const int side = e / (kPairT * kPairDC), f = e % (kPairT * kPairDC);
                    const int r = f / kPairDC, t = f % kPairDC;
                    const uint32_t ci = (side ? J : I) * kPairT + r, dim = dc0 + t;
                    if (ci < k && dim < d16) pair_cp4((side ? ys : xs) + r * kPairLd + t, c + (size_t)ci * d + dim);
                }
            }
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };
    if (tid < kPairT) {
        colkey[tid] = ~0ull;
        colbits[tid] = 0u;
    }
    uint32_t it = 0;
    issue(0);
    for (int sd = 0; sd < 2; sd++) {
        const uint32_t I = sd ? I1 : I0;
        if (sd == 1 && I1 <= I0) break;
        const uint32_t i0 = I * kPairT;
        const uint32_t ia = i0 + tr, ib = i0 + tr + 16;
        const bool live_a = ia < k && start[ia + 1] > start[ia];
        const bool live_b = ib < k && start[ib + 1] > start[ib];
        unsigned long long best_a = ~0ull, best_b = ~0ull;
        __syncthreads();  // the previous row tile's tails are no longer read
        for (int e = tid; e < kPairT * 16; e += kPairThreads) {
            const int r = e >> 4, t = e & 15;
            xt[e] = (i0 + r < k && t < (int)dt) ? c[(size_t)(i0 + r) * d + d16 + t] : 0.0f;
        }
        for (uint32_t J = I; J < T; J++) {
            const uint32_t j0 = J * kPairT;
            float acc[2][2][16];
#pragma unroll
            for (int a = 0; a < 2; a++)
#pragma unroll
                for (int bb = 0; bb < 2; bb++)
#pragma unroll
                    for (int l = 0; l < 16; l++) acc[a][bb][l] = 0.0f;
            for (uint32_t ch = 0; ch < nchunk; ch++, it++) {
                issue(it + 1);
                asm volatile("cp.async.wait_group 1;\n" ::: "memory");
                __syncthreads();
                const float* xs = stage + (it & 1) * kPairStage;
                const float* ys = xs + kPairT * kPairLd;
                const int nq = (int)min((uint32_t)(kPairDC / 16), (d16 - ch * kPairDC) / 16);
                for (int q = 0; q < nq; q++) {
#pragma unroll
                    for (int g4 = 0; g4 < 4; g4++) {
                        const int off = q * 16 + g4 * 4;
                        const float4 x0 = *reinterpret_cast<const float4*>(xs + tr * kPairLd + off);
                        const float4 x1 = *reinterpret_cast<const float4*>(xs + (tr + 16) * kPairLd + off);
                        const float4 y0 = *reinterpret_cast<const float4*>(ys + tc * kPairLd + off);
                        const float4 y1 = *reinterpret_cast<const float4*>(ys + (tc + 16) * kPairLd + off);
                        const float xv[2][4] = {{x0.x, x0.y, x0.z, x0.w}, {x1.x, x1.y, x1.z, x1.w}};
                        const float yv[2][4] = {{y0.x, y0.y, y0.z, y0.w}, {y1.x, y1.y, y1.z, y1.w}};
#pragma unroll
                        for (int a = 0; a < 2; a++)
#pragma unroll
                            for (int bb = 0; bb < 2; bb++)
#pragma unroll
                                for (int i = 0; i < 4; i++) {
                                    const float u = __fsub_rn(xv[a][i], yv[bb][i]);
                                    acc[a][bb][g4 * 4 + i] = __fadd_rn(acc[a][bb][g4 * 4 + i], __fmul_rn(u, u));
                                }
                    }
                }
                __syncthreads();  // this stage is refilled by the issue two items on
            }
            for (int e = tid; e < kPairT * 16; e += kPairThreads) {
                const int r = e >> 4, t = e & 15;
                yt[e] = (j0 + r < k && t < (int)dt) ? c[(size_t)(j0 + r) * d + d16 + t] : 0.0f;
            }
            __syncthreads();
            const bool offdiag = J != I;
            uint32_t bits_a = 0, bits_b = 0;
#pragma unroll
            for (int a = 0; a < 2; a++) {
                const int row = tr + 16 * a;
                const uint32_t i = i0 + row;
                const bool live_i = a ? live_b : live_a;
#pragma unroll
                for (int bb = 0; bb < 2; bb++) {
                    const int col = tc + 16 * bb;
                    float s = acc[a][bb][0];
#pragma unroll
                    for (int l = 1; l < 16; l++) s = __fadd_rn(s, acc[a][bb][l]);
                    float tail = 0.0f;
                    for (uint32_t t = 0; t < dt; t++) {
                        const float u = __fsub_rn(xt[row * 16 + t], yt[col * 16 + t]);
                        tail = __fadd_rn(tail, __fmul_rn(u, u));
                    }
                    s = __fadd_rn(s, tail);
                    const uint32_t j = j0 + col;
                    const bool live_j = j < k && start[j + 1] > start[j];
                    if (ADJ) {
                        const bool hit = live_i && live_j && j != i && __fsqrt_rn(s) <= radius;
                        if (hit) (a ? bits_b : bits_a) |= 1u << col;
                        if (hit && offdiag) atomicOr(&colbits[col], 1u << row);
                    } else if (s < INFINITY && i < k && j < k && j != i) {
                        if (live_j) {
                            const unsigned long long key = ((unsigned long long)__float_as_uint(s) << 32) | j;
                            unsigned long long& best = a ? best_b : best_a;
                            best = key < best ? key : best;
                        }
                        if (live_i && offdiag)
                            atomicMin(&colkey[col], ((unsigned long long)__float_as_uint(s) << 32) | i);
                    }
                }
            }
            if (ADJ) {  // the 16 lanes of a half-warp hold one row pair: OR their bits
#pragma unroll
                for (int o = 1; o < 16; o <<= 1) {
                    bits_a |= __shfl_xor_sync(0xffffffffu, bits_a, o);
                    bits_b |= __shfl_xor_sync(0xffffffffu, bits_b, o);
                }
                if (tc == 0) {
                    if (ia < k) adj[(size_t)ia * words + J] = bits_a;
                    if (ib < k) adj[(size_t)ib * words + J] = bits_b;
                }
            }
            __syncthreads();
            if (offdiag && tid < kPairT && j0 + tid < k) {  // the column tile's rows, over this row tile
                if (ADJ) adj[(size_t)(j0 + tid) * words + I] = colbits[tid];
                else if (colkey[tid] != ~0ull) atomicMin(&near_key[j0 + tid], colkey[tid]);
            }
            if (tid < kPairT) {
                colkey[tid] = ~0ull;
                colbits[tid] = 0u;
            }
        }
        if (!ADJ) {
#pragma unroll
            for (int o = 1; o < 16; o <<= 1) {
                const unsigned long long va = __shfl_xor_sync(0xffffffffu, best_a, o);
                const unsigned long long vb = __shfl_xor_sync(0xffffffffu, best_b, o);
                best_a = va < best_a ? va : best_a;
                best_b = vb < best_b ? vb : best_b;
            }
            if (tc == 0) {
                if (ia < k && best_a != ~0ull) atomicMin(&near_key[ia], best_a);
                if (ib < k && best_b != ~0ull) atomicMin(&near_key[ib], best_b);
            }
        }
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// near_key -> (nearest centroid, squared distance), or (i, inf) without one.
__global__ void k_rep_near_finish(const unsigned long long* __restrict__ near_key, uint32_t k,
                                  uint32_t* __restrict__ near_j, float* __restrict__ near_s) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= k) return;
    const unsigned long long key = near_key[i];
    near_j[i] = key == ~0ull ? i : (uint32_t)key;
    near_s[i] = key == ~0ull ? INFINITY : __uint_as_float((uint32_t)(key >> 32));
}

// ---- families ----------------------------------------------------------------

// Sort keys of the clusters by size, largest first, then by index; dead
// clusters last.
__global__ void k_rep_order_keys(const uint32_t* __restrict__ start, uint32_t k, unsigned long long* __restrict__ keys) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < k) keys[j] = ((unsigned long long)(0xffffffffu - (start[j + 1] - start[j])) << 32) | j;
}

// Greedy families (src/report.rs:198-216) in one CTA: the first unassigned
// cluster in size order leads a new family of every unassigned live cluster
// within the radius (the adjacency row) and itself. The assigned bitset lives in
// shared memory; with TABLES, so do the size order and the cluster sizes, which
// leaves one global read (the leader's adjacency row) on each leader's path.
// Dynamic shared memory: words x 4 bytes, plus 2 x k x 4 bytes with TABLES.
template <bool TABLES>
__global__ void __launch_bounds__(1024) k_rep_families(const unsigned long long* __restrict__ order, uint32_t live,
                                                       uint32_t k, const uint32_t* __restrict__ adj, uint32_t words,
                                                       const uint32_t* __restrict__ start,
                                                       uint32_t* __restrict__ fam_of, uint32_t* __restrict__ fam_lead,
                                                       unsigned long long* __restrict__ fam_size,
                                                       uint32_t* __restrict__ nfam) {
    extern __shared__ __align__(16) uint32_t fam_sm[];
    uint32_t* assigned = fam_sm;                       // [words]
    uint32_t* ord = fam_sm + words;                    // TABLES: [live] cluster ids in size order
    uint32_t* size = ord + (TABLES ? k : 0);           // TABLES: [k] cluster sizes
    __shared__ uint32_t s_q;
    __shared__ unsigned long long s_part[32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (uint32_t w = tid; w < words; w += 1024) assigned[w] = 0u;
    if (TABLES) {
        for (uint32_t q = tid; q < live; q += 1024) ord[q] = (uint32_t)order[q];
        for (uint32_t j = tid; j < k; j += 1024) size[j] = start[j + 1] - start[j];
    }
    auto order_at = [&](uint32_t q) { return TABLES ? ord[q] : (uint32_t)order[q]; };
    auto size_of = [&](uint32_t j) { return TABLES ? size[j] : start[j + 1] - start[j]; };
    uint32_t p = 0, F = 0;
    for (;;) {
        if (tid == 0) s_q = 0xffffffffu;
        __syncthreads();
        for (uint32_t b0 = p; b0 < live; b0 += 1024) {
            const uint32_t q = b0 + tid;
            if (q < live) {
                const uint32_t j = order_at(q);
                if (!((assigned[j >> 5] >> (j & 31)) & 1u)) atomicMin(&s_q, q);
            }
            __syncthreads();
            const bool found = s_q != 0xffffffffu;
            __syncthreads();
            if (found) break;
        }
        const uint32_t q = s_q;
        if (q == 0xffffffffu) break;
        const uint32_t lead = order_at(q);
        p = q + 1;
        const uint32_t* arow = adj + (size_t)lead * words;
        unsigned long long sz = 0;
        for (uint32_t w = tid; w < words; w += 1024) {
            uint32_t m = arow[w] | (w == (lead >> 5) ? (1u << (lead & 31)) : 0u);
            m &= ~assigned[w];
            if (m) {
                assigned[w] |= m;
                while (m) {
                    const int b = __ffs(m) - 1;
                    m &= m - 1;
                    const uint32_t j = w * 32 + b;
                    fam_of[j] = F;
                    sz += size_of(j);
                }
            }
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) sz += __shfl_xor_sync(0xffffffffu, sz, o);
        if (lane == 0) s_part[warp] = sz;
        __syncthreads();
        if (tid == 0) {
            unsigned long long t = 0;
            for (int w = 0; w < 32; w++) t += s_part[w];
            fam_lead[F] = lead;
            fam_size[F] = t;
        }
        F++;
        __syncthreads();
    }
    if (tid == 0) *nfam = F;
}

// ---- families as the lexicographically first maximal independent set --------
//
// The greedy pass above makes cluster v a leader exactly when no cluster before
// it in size order that is adjacent to it is a leader; every other live cluster
// joins the earliest adjacent leader (the first leader to reach it). The same
// result, computed in parallel rounds over compact lists of earlier neighbours
// (by size-order position): an undecided position becomes FOLLOWER as soon as an
// earlier neighbour is a LEADER, and LEADER once all earlier neighbours are
// decided followers. Each round decides at least the earliest undecided position.

constexpr uint8_t kFamUndecided = 0, kFamLeader = 1, kFamFollower = 2;

// pos[cluster] = its position in size order (live clusters only).
__global__ void k_rep_pos(const unsigned long long* __restrict__ order, uint32_t live, uint32_t* __restrict__ pos) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < live) pos[(uint32_t)order[q]] = q;
}

// One warp per live position q: the earlier neighbours of cluster order[q] in its
// adjacency row. FILL = false counts them into ecount[q]; FILL = true writes their
// positions from eoff[q] on.
template <bool FILL>
__global__ void k_rep_nbrs(const unsigned long long* __restrict__ order, uint32_t live,
                           const uint32_t* __restrict__ adj, uint32_t words, const uint32_t* __restrict__ pos,
                           uint32_t* __restrict__ ecount, const uint32_t* __restrict__ eoff,
                           uint32_t* __restrict__ nbr) {
    const uint32_t q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (q >= live) return;
    const uint32_t v = (uint32_t)order[q];
    const uint32_t* row = adj + (size_t)v * words;
    uint32_t base = FILL ? eoff[q] : 0u, total = 0;
    for (uint32_t w0 = 0; w0 < words; w0 += 32) {
        const uint32_t w = w0 + lane;
        uint32_t m = w < words ? row[w] : 0u;
        uint32_t cnt = 0, keep = 0;
        for (uint32_t mm = m; mm;) {
            const int b = __ffs(mm) - 1;
            mm &= mm - 1;
            if (pos[w * 32 + b] < q) {
                cnt++;
                keep |= 1u << b;
            }
        }
        if (FILL) {
            uint32_t pre = cnt;  // inclusive prefix of the counts over lanes
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, pre, o);
                if (lane >= o) pre += y;
            }
            uint32_t at = base + pre - cnt;
            for (uint32_t mm = keep; mm;) {
                const int b = __ffs(mm) - 1;
                mm &= mm - 1;
                nbr[at++] = pos[w * 32 + b];
            }
            base += __shfl_sync(0xffffffffu, pre, 31);
        } else {
            total += cnt;
        }
    }
    if (!FILL) {
#pragma unroll
        for (int o = 16; o; o >>= 1) total += __shfl_xor_sync(0xffffffffu, total, o);
        if (lane == 0) ecount[q] = total;
    }
}

// One CTA: the rounds above on a status byte per position in shared memory
// (dynamic: live bytes), then each position's family: its own (leader) or that
// of its earliest leader neighbour. Families are numbered by their leaders'
// positions, which is the greedy pass's order of formation. fam_size must be
// zero on entry.
__global__ void __launch_bounds__(1024) k_rep_lfmis(const unsigned long long* __restrict__ order, uint32_t live,
                                                    const uint32_t* __restrict__ eoff,
                                                    const uint32_t* __restrict__ nbr,
                                                    const uint32_t* __restrict__ start,
                                                    uint32_t* __restrict__ fidx, uint32_t* __restrict__ fam_of,
                                                    uint32_t* __restrict__ fam_lead,
                                                    unsigned long long* __restrict__ fam_size,
                                                    uint32_t* __restrict__ nfam) {
    extern __shared__ uint8_t status[];
    __shared__ uint32_t ws[32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (uint32_t q = tid; q < live; q += 1024) status[q] = kFamUndecided;
    __syncthreads();
    for (uint32_t round = 0; round <= live; round++) {
        int open = 0;
        for (uint32_t q = tid; q < live; q += 1024) {
            if (status[q] != kFamUndecided) continue;
            bool leader_seen = false, all_decided = true;
            for (uint32_t e = eoff[q]; e < eoff[q + 1]; e++) {
                const uint8_t st = status[nbr[e]];
                if (st == kFamLeader) {
                    leader_seen = true;
                    break;
                }
                if (st == kFamUndecided) all_decided = false;
            }
            if (leader_seen) status[q] = kFamFollower;
            else if (all_decided) status[q] = kFamLeader;
            else open = 1;
        }
        if (!__syncthreads_or(open)) break;
    }
    // (every round decides the earliest undecided position, so none is left here)
    for (uint32_t q = tid; q < live; q += 1024)
        if (status[q] == kFamUndecided) status[q] = kFamLeader;
    __syncthreads();
    // family number of each leader: leaders before it in position order
    uint32_t carry = 0;
    for (uint32_t b0 = 0; b0 < live; b0 += 1024) {
        const uint32_t q = b0 + tid;
        const uint32_t isl = q < live && status[q] == kFamLeader ? 1u : 0u;
        const unsigned bal = __ballot_sync(0xffffffffu, isl);
        if (lane == 0) ws[warp] = __popc(bal);
        __syncthreads();
        uint32_t before = carry;
        for (int w = 0; w < warp; w++) before += ws[w];
        before += __popc(bal & ((1u << lane) - 1u));
        if (isl) fidx[q] = before;
        uint32_t tot = 0;
        for (int w = 0; w < 32; w++) tot += ws[w];
        carry += tot;
        __syncthreads();
    }
    if (tid == 0) *nfam = carry;
    __syncthreads();
    for (uint32_t q = tid; q < live; q += 1024) {
        uint32_t lq = q;
        if (status[q] != kFamLeader) {
            lq = 0xffffffffu;
            for (uint32_t e = eoff[q]; e < eoff[q + 1]; e++) {
                const uint32_t u = nbr[e];
                if (status[u] == kFamLeader && u < lq) lq = u;
            }
        }
        const uint32_t f = fidx[lq];
        const uint32_t v = (uint32_t)order[q];
        fam_of[v] = f;
        atomicAdd(&fam_size[f], (unsigned long long)(start[v + 1] - start[v]));
        if (lq == q) fam_lead[f] = v;
    }
}

// Families renumbered by size, largest first (formation order among equals).
__global__ void k_rep_family_keys(const unsigned long long* __restrict__ fam_size, uint32_t F,
                                  unsigned long long* __restrict__ keys) {
    const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f < F) keys[f] = ((unsigned long long)(0xffffffffu - (uint32_t)fam_size[f]) << 32) | f;
}

__global__ void k_rep_family_rank(const unsigned long long* __restrict__ sorted, uint32_t F,
                                  const uint32_t* __restrict__ fam_lead, const unsigned long long* __restrict__ fam_size,
                                  unsigned long long n, uint32_t* __restrict__ rank_of, uint32_t* __restrict__ out_lead,
                                  unsigned long long* __restrict__ out_size, double* __restrict__ out_share) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= F) return;
    const uint32_t f = (uint32_t)sorted[r];
    rank_of[f] = r;
    out_lead[r] = fam_lead[f];
    out_size[r] = fam_size[f];
    out_share[r] = __ddiv_rn((double)fam_size[f], (double)n);
}

// Member keys (family rank, position in size order): sorted, they list each
// family's members in size order, as the reference's order-preserving collect.
__global__ void k_rep_member_keys(const unsigned long long* __restrict__ order, uint32_t live,
                                  const uint32_t* __restrict__ fam_of, const uint32_t* __restrict__ rank_of,
                                  unsigned long long* __restrict__ keys) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < live) keys[q] = ((unsigned long long)rank_of[fam_of[(uint32_t)order[q]]] << 32) | q;
}

__global__ void k_rep_members(const unsigned long long* __restrict__ sorted, uint32_t live,
                              const unsigned long long* __restrict__ order, uint32_t F, uint32_t* __restrict__ members,
                              uint32_t* __restrict__ offsets) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > live) return;
    if (p < live) members[p] = (uint32_t)order[(uint32_t)sorted[p]];
    const long long a = p > 0 ? (long long)(sorted[p - 1] >> 32) : -1;
    const long long b = p < live ? (long long)(sorted[p] >> 32) : (long long)F;
    for (long long f = a + 1; f <= b; f++) offsets[f] = p;
}

// ClusterStats rows (src/report.rs:37-56), field order of emb200_cluster_stats.
struct RepCluster {
    uint32_t size;
    float rms, median, mad, p90, p99, max, looseness;
    uint32_t nearest_centroid;
    float nearest_dist, isolation;
    uint32_t family;
};

__global__ void k_rep_clusters(const uint32_t* __restrict__ start, uint32_t k, const float* __restrict__ rms,
                               const float* __restrict__ med, const float* __restrict__ mad,
                               const float* __restrict__ p90, const float* __restrict__ p99,
                               const float* __restrict__ mx, const uint32_t* __restrict__ near_j,
                               const float* __restrict__ near_s, const uint32_t* __restrict__ fam_of,
                               const uint32_t* __restrict__ rank_of, const RepScalars* __restrict__ sc,
                               RepCluster* __restrict__ out) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= k) return;
    RepCluster r;
    r.size = start[j + 1] - start[j];
    r.rms = rms[j];
    r.median = med[j];
    r.mad = mad[j];
    r.p90 = p90[j];
    r.p99 = p99[j];
    r.max = mx[j];
    r.looseness = __fdiv_rn(r.rms, fmaxf(sc->median_rms, FLT_MIN));
    r.nearest_centroid = near_j[j];
    r.nearest_dist = __fsqrt_rn(near_s[j]);
    r.isolation = __fdiv_rn(r.nearest_dist, fmaxf(sc->median_nearest, FLT_MIN));
    r.family = r.size ? rank_of[fam_of[j]] : 0u;
    out[j] = r;
}

}  // namespace emb
