// Device kernels of the training update path (src/lib.rs:276-491): the batch's
// per-cluster sums in row order, the EMA step, revival of dead clusters and the
// closing mean, all in the reference's f32 operation order so that a training
// run on the device follows the CPU trajectory bit for bit.
#pragma once
#include "common.cuh"

namespace emb {

// Initial centroids: rows init[0..k) of x, widened to f32 (src/lib.rs:374-379).
template <typename T>
__global__ void k_gather_centroids(const T* __restrict__ x, const uint32_t* __restrict__ idx, int k, int d,
                                   float* __restrict__ c) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)k * d) return;
    size_t j = i / d, t = i - j * d;
    c[i] = to_f32(x[(size_t)idx[j] * d + t]);
}

__global__ void k_fill_u32(uint32_t* __restrict__ p, size_t n, uint32_t v) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

// counts[l]++ per batch row; slot[i] = this row's arrival order within its label
// (arbitrary; put back in row order by k_segment_sums).
__global__ void k_label_hist(const uint32_t* __restrict__ labels, int m, uint32_t* __restrict__ counts,
                             uint32_t* __restrict__ slot) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) slot[i] = atomicAdd(&counts[labels[i]], 1u);
}

// Exclusive prefix sum of counts[0..k) -> offsets (one CTA of 1024 threads).
__global__ void __launch_bounds__(1024) k_exclusive_scan(const uint32_t* __restrict__ counts, int k,
                                                         uint32_t* __restrict__ offsets) {
    __shared__ uint32_t part[1024];
    const int tid = threadIdx.x;
    const int per = (k + 1023) / 1024;
    const int lo = tid * per, hi = min(k, lo + per);
    uint32_t s = 0;
    for (int j = lo; j < hi; j++) s += counts[j];
    part[tid] = s;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        uint32_t v = tid >= o ? part[tid - o] : 0u;
        __syncthreads();
        part[tid] += v;
        __syncthreads();
    }
    uint32_t base = tid ? part[tid - 1] : 0u;
    for (int j = lo; j < hi; j++) {
        offsets[j] = base;
        base += counts[j];
    }
}

__global__ void k_label_scatter(const uint32_t* __restrict__ labels, const uint32_t* __restrict__ slot, int m,
                                const uint32_t* __restrict__ offsets, uint32_t* __restrict__ list) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) list[offsets[labels[i]] + slot[i]] = (uint32_t)i;
}

// Bitonic sort of E * 32 entries held E per lane (entry lane + 32 h in v[h]),
// ascending; distances below 32 exchange through shuffles, longer ones within
// the lane.
template <int E>
EMB_DEV void warp_bitonic_regs(uint32_t (&v)[E], int lane) {
#pragma unroll
    for (int k2 = 2; k2 <= 32 * E; k2 <<= 1) {
#pragma unroll
        for (int j = k2 >> 1; j > 0; j >>= 1) {
            if (j < 32) {
#pragma unroll
                for (int h = 0; h < E; h++) {
                    const uint32_t e = (uint32_t)(lane + 32 * h);
                    const uint32_t o = __shfl_xor_sync(0xffffffffu, v[h], j);
                    const bool up = (e & (uint32_t)k2) == 0, lower = (e & (uint32_t)j) == 0;
                    v[h] = (lower == up) ? min(v[h], o) : max(v[h], o);
                }
            } else {
#pragma unroll
                for (int h = 0; h < E; h++) {
                    const int h2 = h ^ (j >> 5);
                    if (h2 > h) {
                        const uint32_t e = (uint32_t)(lane + 32 * h);
                        const bool up = (e & (uint32_t)k2) == 0;
                        const uint32_t mn = min(v[h], v[h2]), mx = max(v[h], v[h2]);
                        v[h] = up ? mn : mx;
                        v[h2] = up ? mx : mn;
                    }
                }
            }
        }
    }
}

template <int E>
EMB_DEV const uint32_t* warp_sort_regs(uint32_t* seg, uint32_t c, int lane) {
    uint32_t v[E];
#pragma unroll
    for (int h = 0; h < E; h++) v[h] = (uint32_t)(lane + 32 * h) < c ? seg[lane + 32 * h] : 0xffffffffu;
    warp_bitonic_regs<E>(v, lane);
#pragma unroll
    for (int h = 0; h < E; h++)
        if ((uint32_t)(lane + 32 * h) < c) seg[lane + 32 * h] = v[h];
    __syncwarp();
    return seg;
}

// Ascending sort of one segment of c batch positions by one warp. Up to 512
// entries are sorted in registers; longer segments are copied to `scratch`
// (room for next_pow2(c) <= 2c entries), padded with UINT32_MAX and sorted there
// by a bitonic network. Returns the sorted segment (seg or scratch).
EMB_DEV const uint32_t* warp_sort_segment(uint32_t* seg, uint32_t c, uint32_t* scratch, int lane) {
    // Up to 512 entries the network runs in registers (2 to 16 per lane).
    if (c > 32 && c <= 64) return warp_sort_regs<2>(seg, c, lane);
    if (c > 64 && c <= 128) return warp_sort_regs<4>(seg, c, lane);
    if (c > 128 && c <= 256) return warp_sort_regs<8>(seg, c, lane);
    if (c > 256 && c <= 512) return warp_sort_regs<16>(seg, c, lane);
    if (c <= 32) {
        uint32_t v = (uint32_t)lane < c ? seg[lane] : 0xffffffffu;
        for (int k2 = 2; k2 <= 32; k2 <<= 1) {
            for (int j = k2 >> 1; j > 0; j >>= 1) {
                const uint32_t o = __shfl_xor_sync(0xffffffffu, v, j);
                const bool up = (lane & k2) == 0 || k2 == 32;
                const bool lower = (lane & j) == 0;
                const uint32_t mn = min(v, o), mx = max(v, o);
                v = (lower == up) ? mn : mx;
            }
        }
        if ((uint32_t)lane < c) seg[lane] = v;
        __syncwarp();
        return seg;
    }
    uint32_t n2 = 1;
    while (n2 < c) n2 <<= 1;
    for (uint32_t i = lane; i < n2; i += 32) scratch[i] = i < c ? seg[i] : 0xffffffffu;
    __syncwarp();
    for (uint32_t k2 = 2; k2 <= n2; k2 <<= 1) {
        for (uint32_t j = k2 >> 1; j > 0; j >>= 1) {
            for (uint32_t i = lane; i < n2; i += 32) {
                const uint32_t pi = i ^ j;
                if (pi > i) {
                    const uint32_t a = scratch[i], b = scratch[pi];
                    const bool up = (i & k2) == 0;
                    if ((a > b) == up) {
                        scratch[i] = b;
                        scratch[pi] = a;
                    }
                }
            }
            __syncwarp();
        }
    }
    return scratch;
}

// Per touched cluster l (one warp each): put its batch rows back in row order and
// sum them sequentially per dimension in f32, the order of src/lib.rs:431-441.
// Also the last pass's per-cluster sums (src/lib.rs:446-454) and labels.
// MAXG > 0 (d <= 32 MAXG): lane t keeps the sums of dimensions t, t + 32, ... in
// registers, the warp fetches 32 row offsets at a time (one per lane) and passes
// them by shuffle, so the loads of several rows and dimension groups are in flight
// together while each dimension's adds keep the row order. MAXG = 0: one
// dimension group at a time.
EMB_DEV void cp_async16(void* smem, const void* gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(smem)),
                 "l"(gmem)
                 : "memory");
}
EMB_DEV void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
EMB_DEV void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Shared memory of a 256-thread block of staged segment sums at most: 8 warps x
// 2 chunks x R d <= 1536 floats.
constexpr size_t kSegStageMaxBytes = (size_t)8 * 2 * 1536 * sizeof(float);

// Rows per staging chunk of segment_sums_warp (two chunks per warp, at most
// 12 KB), or 0 for the unstaged form: f32 rows with d % 4 == 0 only.
inline int segment_stage_rows(size_t d, bool f32_rows) {
    if (!f32_rows || d % 4 != 0 || d > 768) return 0;
    int r = 32;
    while (r > 2 && (size_t)r * d > 1536) r >>= 1;
    return r;
}

// Sums of one cluster's c batch rows per dimension, in row order. With `stage`
// (2 R d floats of this warp's shared memory; f32 rows, d % 4 == 0, 16-byte
// aligned), the rows come in chunks of R by cp.async, the next chunk in flight
// while this one is summed: every row of a chunk is requested at once instead of
// a few at a time. Each dimension's adds keep the row order either way.
template <typename T, int MAXG>
EMB_DEV void segment_sums_warp(const T* __restrict__ x, const uint32_t* __restrict__ rows, int d, int l,
                               uint32_t c, uint32_t* seg_list, uint32_t* seg_scratch, float* __restrict__ sums,
                               int is_last, unsigned long long* __restrict__ pass_counts,
                               float* __restrict__ pass_sums, double* __restrict__ pass_sums64, int lane,
                               float* stage = nullptr, int R = 0) {
    const uint32_t* seg = warp_sort_segment(seg_list, c, seg_scratch, lane);
    auto store = [&](int t, float acc, double acc64) {
        sums[(size_t)l * d + t] = acc;
        if (is_last) {
            if (pass_sums64) pass_sums64[(size_t)l * d + t] += acc64;
            else pass_sums[(size_t)l * d + t] = __fadd_rn(pass_sums[(size_t)l * d + t], acc);
        }
    };
    if constexpr (MAXG > 0) {
        float acc[MAXG];
        double acc64[MAXG];
#pragma unroll
        for (int g = 0; g < MAXG; g++) {
            acc[g] = 0.0f;
            acc64[g] = 0.0;
        }
        const bool staged = sizeof(T) == 4 && stage && R > 0 && (d & 3) == 0 && (((uintptr_t)x & 15) == 0);
        if (staged) {
            const uint32_t vpr = (uint32_t)d >> 2;  // 16-byte pieces per row
            const uint32_t nq = (c + (uint32_t)R - 1) / (uint32_t)R;
            auto issue = [&](uint32_t q) {
                const uint32_t j0 = q * (uint32_t)R, n = min((uint32_t)R, c - j0);
                const uint32_t myrow = (uint32_t)lane < n ? rows[seg[j0 + lane]] : 0u;
                float* buf = stage + (q & 1) * (size_t)R * d;
                for (uint32_t e0 = 0; e0 < n * vpr; e0 += 32) {
                    const uint32_t e = e0 + lane, jj = e / vpr, pc = e - jj * vpr;
                    const uint32_t src = __shfl_sync(0xffffffffu, myrow, (int)min(jj, 31u));
                    if (e < n * vpr) cp_async16(buf + jj * d + 4 * pc, (const float*)x + (size_t)src * d + 4 * pc);
                }
                cp_async_commit();
            };
            issue(0);
            for (uint32_t q = 0; q < nq; q++) {
                if (q + 1 < nq) {
                    issue(q + 1);
                    cp_async_wait<1>();
                } else {
                    cp_async_wait<0>();
                }
                __syncwarp();
                const float* buf = stage + (q & 1) * (size_t)R * d;
                const uint32_t n = min((uint32_t)R, c - q * (uint32_t)R);
                for (uint32_t jj = 0; jj < n; jj++) {
#pragma unroll
                    for (int g = 0; g < MAXG; g++) {
                        const int t = g * 32 + lane;
                        if (t < d) {
                            const float v = buf[jj * d + t];
                            acc[g] = __fadd_rn(acc[g], v);
                            if (pass_sums64) acc64[g] += (double)v;
                        }
                    }
                }
                __syncwarp();  // this buffer is refilled two chunks on
            }
        }
        for (uint32_t j0 = 0; j0 < (staged ? 0u : c); j0 += 32) {
            const uint32_t n = min(32u, c - j0);
            const uint32_t myrow = (uint32_t)lane < n ? rows[seg[j0 + lane]] : 0u;
#pragma unroll 4
            for (uint32_t jj = 0; jj < n; jj++) {
                const T* xr = x + (size_t)__shfl_sync(0xffffffffu, myrow, (int)jj) * d;
#pragma unroll
                for (int g = 0; g < MAXG; g++) {
                    const int t = g * 32 + lane;
                    if (t < d) {
                        const float v = to_f32(xr[t]);
                        acc[g] = __fadd_rn(acc[g], v);
                        if (pass_sums64) acc64[g] += (double)v;
                    }
                }
            }
        }
#pragma unroll
        for (int g = 0; g < MAXG; g++) {
            const int t = g * 32 + lane;
            if (t < d) store(t, acc[g], acc64[g]);
        }
    } else {
        for (int t0 = 0; t0 < d; t0 += 32) {
            const int t = t0 + lane;
            float acc = 0.0f;
            double acc64 = 0.0;
            if (t < d) {
                for (uint32_t j = 0; j < c; j++) {
                    const float v = to_f32(x[(size_t)rows[seg[j]] * d + t]);
                    acc = __fadd_rn(acc, v);
                    if (pass_sums64) acc64 += (double)v;
                }
                store(t, acc, acc64);
            }
        }
    }
    if (is_last && lane == 0) pass_counts[l] += c;
}

template <typename T, int MAXG>
__global__ void k_segment_sums(const T* __restrict__ x, const uint32_t* __restrict__ rows, int d, int k,
                               const uint32_t* __restrict__ counts, const uint32_t* __restrict__ offsets,
                               uint32_t* __restrict__ list, uint32_t* __restrict__ scratch, float* __restrict__ sums,
                               const int* __restrict__ last_pass,
                               unsigned long long* __restrict__ pass_counts, float* __restrict__ pass_sums,
                               double* __restrict__ pass_sums64, int R) {
    extern __shared__ float seg_stage[];  // R > 0: (blockDim / 32) x 2 R d floats
    const int l = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (l >= k) return;
    const uint32_t c = counts[l];
    if (c == 0) return;
    // Segment l sorts in scratch[2 offsets[l] ...): next_pow2(c) <= 2c entries,
    // disjoint from every other segment's region.
    float* stage = R ? seg_stage + (size_t)(threadIdx.x >> 5) * 2 * R * d : nullptr;
    segment_sums_warp<T, MAXG>(x, rows, d, l, c, list + offsets[l], scratch + 2 * (size_t)offsets[l], sums,
                               *last_pass, pass_counts, pass_sums, pass_sums64, lane, stage, R);
}

// Per-cluster sums with the dimensions split over warps (f32 rows, d % 4 == 0,
// 16-byte aligned rows, d <= kDgMaxD): block l sums cluster l, warp g dimensions
// [32 g, 32 g + 32). Warp 0 puts the cluster's batch positions in row order
// (as segment_sums_warp) and the block shares the sorted list; each warp then
// streams its 128-byte slice of every row through a ring of kDgStages chunks of
// kDgRows rows (cp.async, kDgStages - 1 chunks in flight) and adds them in row
// order, lane t one dimension. A crowded cluster's rows are read by d / 32 warps
// with up to 14 KB in flight each, where the one-warp form has 12 KB for all d.
constexpr int kDgRows = 16, kDgStages = 8;
constexpr size_t kDgWarpBytes = (size_t)kDgStages * kDgRows * 32 * sizeof(float);
constexpr int kDgMaxD = 384;  // 12 warps x 16 KB of ring

__global__ void __launch_bounds__(384) k_segment_sums_dg(const float* __restrict__ x,
                                                         const uint32_t* __restrict__ rows, int d,
                                                         const uint32_t* __restrict__ counts,
                                                         const uint32_t* __restrict__ offsets,
                                                         uint32_t* __restrict__ list, uint32_t* __restrict__ scratch,
                                                         float* __restrict__ sums, const int* __restrict__ last_pass,
                                                         unsigned long long* __restrict__ pass_counts,
                                                         float* __restrict__ pass_sums,
                                                         double* __restrict__ pass_sums64) {
    extern __shared__ float dg_stage[];  // (blockDim / 32) x kDgStages x kDgRows x 32 floats
    __shared__ int use_scratch;
    const int l = blockIdx.x, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t c = counts[l];
    if (c == 0) return;  // uniform over the block
    uint32_t* seg_list = list + offsets[l];
    uint32_t* seg_scratch = scratch + 2 * (size_t)offsets[l];
    if (warp == 0) {
        const uint32_t* sorted = warp_sort_segment(seg_list, c, seg_scratch, lane);
        if (lane == 0) use_scratch = sorted != seg_list;
    }
    __syncthreads();
    const uint32_t* seg = use_scratch ? seg_scratch : seg_list;
    const int t0 = warp * 32;
    const int nd = min(32, d - t0);  // dimensions of this warp (a multiple of 4)
    const int ppr = nd >> 2;         // 16-byte pieces per row
    float* ring = dg_stage + (size_t)warp * kDgStages * kDgRows * 32;
    const uint32_t nq = (c + kDgRows - 1) / kDgRows;
    auto issue = [&](uint32_t q) {
        if (q < nq) {
            const uint32_t j0 = q * kDgRows, n = min((uint32_t)kDgRows, c - j0);
            const uint32_t myrow = (uint32_t)lane < n ? rows[seg[j0 + lane]] : 0u;
            float* buf = ring + (size_t)(q % kDgStages) * kDgRows * 32;
            for (uint32_t e0 = 0; e0 < n * (uint32_t)ppr; e0 += 32) {
                const uint32_t e = e0 + lane, jj = e / (uint32_t)ppr, pc = e - jj * (uint32_t)ppr;
                const uint32_t src = __shfl_sync(0xffffffffu, myrow, (int)min(jj, 31u));
                if (e < n * (uint32_t)ppr) cp_async16(buf + jj * 32 + 4 * pc, x + (size_t)src * d + t0 + 4 * pc);
            }
        }
        cp_async_commit();  // an empty group past the end keeps the group count uniform
    };
#pragma unroll
    for (int q = 0; q < kDgStages - 1; q++) issue((uint32_t)q);
    float acc = 0.0f;
    double acc64 = 0.0;
    const bool mine = lane < nd;
    for (uint32_t q = 0; q < nq; q++) {
        cp_async_wait<kDgStages - 2>();  // chunk q has landed
        __syncwarp();
        const float* buf = ring + (size_t)(q % kDgStages) * kDgRows * 32;
        const uint32_t n = min((uint32_t)kDgRows, c - q * kDgRows);
        if (mine) {
            for (uint32_t jj = 0; jj < n; jj++) {
                const float v = buf[jj * 32 + lane];
                acc = __fadd_rn(acc, v);
                if (pass_sums64) acc64 += (double)v;
            }
        }
        __syncwarp();  // this buffer is refilled below, kDgStages - 1 chunks on
        issue(q + kDgStages - 1);
    }
    cp_async_wait<0>();
    if (mine) {
        const int t = t0 + lane;
        sums[(size_t)l * d + t] = acc;
        if (*last_pass) {
            if (pass_sums64) pass_sums64[(size_t)l * d + t] += acc64;
            else pass_sums[(size_t)l * d + t] = __fadd_rn(pass_sums[(size_t)l * d + t], acc);
        }
    }
    if (*last_pass && threadIdx.x == 0) pass_counts[l] += c;
}

// The batch's rows gathered into one contiguous block (the proposer's search
// reads contiguous rows).
__global__ void k_gather_rows(const float* __restrict__ x, const uint32_t* __restrict__ rows, int m, int d,
                              float* __restrict__ out) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (size_t)m * d) return;
    const size_t i = e / d, t = e - i * d;
    out[e] = x[(size_t)rows[i] * d + t];
}

// Last pass: labels[i] = l for every row of the batch (src/lib.rs:438-440).
__global__ void k_store_labels(const uint32_t* __restrict__ batch_labels, const uint32_t* __restrict__ rows, int m,
                               uint32_t* __restrict__ labels_all, const int* __restrict__ last_pass) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m && *last_pass) labels_all[rows[i]] = batch_labels[i];
}

// State::apply (src/lib.rs:287-309), one warp per cluster: N *= (1 - a) for all
// clusters; touched ones take mass = N + a n, w = a n / mass, c += w (s/n - c)
// (c = s/n when w == 1). alpha = alphas[*step]: the host-computed cosine schedule.
EMB_DEV void apply_warp(int j, int d, float alpha, float* __restrict__ c, float* __restrict__ usage,
                        const uint32_t* __restrict__ counts, const float* __restrict__ sums, int lane) {
    const bool replace = alpha == 1.0f;
    float u = usage[j];
    if (!replace) u = __fmul_rn(u, __fsub_rn(1.0f, alpha));
    const uint32_t cnt = counts[j];
    if (cnt > 0) {
        const float n = (float)cnt;
        const float retained = replace ? 0.0f : u;
        const float an = __fmul_rn(alpha, n);
        const float mass = __fadd_rn(retained, an);
        const float w = __fdiv_rn(an, mass);
        float* cj = c + (size_t)j * d;
        const float* sj = sums + (size_t)j * d;
        for (int t = lane; t < d; t += 32) {
            const float mean = __fdiv_rn(sj[t], n);
            cj[t] = (w == 1.0f) ? mean : __fadd_rn(cj[t], __fmul_rn(w, __fsub_rn(mean, cj[t])));
        }
        u = mass;
    }
    if (lane == 0) usage[j] = u;
}

__global__ void k_apply(int k, int d, float* __restrict__ c, float* __restrict__ usage,
                        const uint32_t* __restrict__ counts, const float* __restrict__ sums,
                        const float* __restrict__ alphas, const int* __restrict__ step) {
    const int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (j >= k) return;
    apply_warp(j, d, alphas[*step], c, usage, counts, sums, lane);
}

// Balance penalty (src/lib.rs:411-417): when balance > 0 and the previous batch's
// mean squared distance s > 0, bias_j = (balance s / mean(N)) N_j, with mean(N)
// summed sequentially in f64 like the reference; otherwise bias = 0. One CTA.
__global__ void __launch_bounds__(1024) k_balance_bias(const float* __restrict__ usage, int k, float balance,
                                                       const double* __restrict__ mean_sqdist,
                                                       float* __restrict__ bias, int* __restrict__ penalized) {
    __shared__ float scale_s;
    __shared__ int pen_s;
    if (threadIdx.x == 0) {
        const double msd = *mean_sqdist;
        pen_s = (balance > 0.0f && msd > 0.0) ? 1 : 0;
        if (pen_s) {
            double s = -0.0;
            for (int j = 0; j < k; j++) s += (double)usage[j];
            const double mean_mass = s / (double)k;
            scale_s = (float)((double)balance * msd / mean_mass);
        }
        *penalized = pen_s;
    }
    __syncthreads();
    for (int j = threadIdx.x; j < k; j += blockDim.x) bias[j] = pen_s ? __fmul_rn(scale_s, usage[j]) : 0.0f;
}

// Report true distances without the penalty (src/lib.rs:425-430).
__global__ void k_unbias_dist(float* __restrict__ dist, const uint32_t* __restrict__ labels, int m,
                              const float* __restrict__ bias, const int* __restrict__ penalized) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m && *penalized) dist[i] = fmaxf(__fsub_rn(dist[i], bias[labels[i]]), 0.0f);
}

// Batch objective (src/lib.rs:442-445): sum of distances in f64. A fixed-shape
// tree (deterministic, ~1e-16 relative from the reference's sequential sum), or
// the sequential sum itself when the value feeds the balance penalty.
// One CTA of 1024; writes obj[0] += batch, mean_sqdist = batch / m.
__global__ void __launch_bounds__(1024) k_batch_objective(const float* __restrict__ dist, int m, int sequential,
                                                          double* __restrict__ objective, const int* __restrict__ epoch,
                                                          double* __restrict__ mean_sqdist) {
    __shared__ double part[1024];
    double s = 0.0;
    if (sequential) {
        if (threadIdx.x == 0) {
            // src/lib.rs:419-443: per chunk of 65536 rows a sequential f64 sum, chunks added in order.
            double b = 0.0;
            for (int c0 = 0; c0 < m; c0 += 65536) {
                double cs = -0.0;
                const int c1 = min(m, c0 + 65536);
                for (int i = c0; i < c1; i++) cs += (double)dist[i];
                b += cs;
            }
            s = b;
        }
    } else {
        for (int i = threadIdx.x; i < m; i += 1024) s += (double)dist[i];
        part[threadIdx.x] = s;
        __syncthreads();
        for (int o = 512; o > 0; o >>= 1) {
            if (threadIdx.x < o) part[threadIdx.x] += part[threadIdx.x + o];
            __syncthreads();
        }
        s = part[0];
    }
    if (threadIdx.x == 0) {
        objective[*epoch] += s;
        *mean_sqdist = s / (double)m;
    }
}

constexpr uint32_t kReviveSmemSort = 16384;  // donors sorted in shared memory up to this many
constexpr size_t kReviveSmemBytes = kReviveSmemSort * (sizeof(double) + sizeof(uint32_t));

// State::revive (src/lib.rs:314-344), one CTA of 1024 threads:
//   total = sum of N (sequential f32), threshold = total tau / k,
//   unused = {N_j < thr}, donors = {N_j >= thr, N_j > 0} in index order, each
//   keyed ln N_j - g_i where g_i = ln(-ln U_i) is the next value of the revival
//   stream (drawn on the host from the reference's generator), donors sorted by
//   key descending, the first min(|unused|, |donors|) split into the unused slots.
// Scratch: keys and didx with room for next_pow2(k) entries, unused[k]; cursor and
// n_splits updated.
// The body of k_revive for one CTA of 1024 threads (called by every thread of
// the block); sort_smem: dynamic shared memory for smem_sort donors.
EMB_DEV void revive_cta(int k, int d, float* __restrict__ c, float* __restrict__ usage, float tau,
                        const double* __restrict__ gstream, unsigned long long* __restrict__ cursor,
                        double* __restrict__ keys, uint32_t* __restrict__ didx, uint32_t* __restrict__ unused,
                        unsigned long long* __restrict__ n_splits, unsigned long long capacity,
                        double* sort_keys, uint32_t smem_sort) {
    __shared__ float thr_s;
    __shared__ uint32_t wsum_u[32], wsum_d[32];
    __shared__ uint32_t nun_s, ndon_s;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    {
        // total = the sequential f32 sum of usage (src/lib.rs:315). The chain of k
        // dependent adds runs in one thread; usage comes through shared memory
        // (the sort region, free until the sort), staged by all threads in
        // chunks, so each add waits on a shared load rather than a global one.
        float* stage = (float*)sort_keys;
        const int cap = (int)smem_sort * 3;  // floats in the sort region (12 B per entry)
        float total = -0.0f;
        for (int c0 = 0; c0 < k; c0 += cap) {
            const int n = min(cap, k - c0);
            for (int i = tid; i < n; i += blockDim.x) stage[i] = usage[c0 + i];
            __syncthreads();
            if (tid == 0) {
                // Eight values per 2 vector loads, issued ahead of their adds (the
                // adds stay one chain in index order).
                const float4* s4 = reinterpret_cast<const float4*>(stage);
                int i = 0;
#pragma unroll 4
                for (; i + 8 <= n; i += 8) {
                    const float4 a = s4[i >> 2], b = s4[(i >> 2) + 1];
                    total = __fadd_rn(total, a.x);
                    total = __fadd_rn(total, a.y);
                    total = __fadd_rn(total, a.z);
                    total = __fadd_rn(total, a.w);
                    total = __fadd_rn(total, b.x);
                    total = __fadd_rn(total, b.y);
                    total = __fadd_rn(total, b.z);
                    total = __fadd_rn(total, b.w);
                }
                for (; i < n; i++) total = __fadd_rn(total, stage[i]);
            }
            __syncthreads();
        }
        if (tid == 0) thr_s = __fdiv_rn(__fmul_rn(total, tau), (float)k);
    }
    __syncthreads();
    const float thr = thr_s;
    // Ordered compaction of unused and donor indices, in chunks of 1024.
    uint32_t base_u = 0, base_d = 0;
    for (int j0 = 0; j0 < k; j0 += 1024) {
        const int j = j0 + tid;
        const float u = j < k ? usage[j] : 0.0f;
        const bool isu = j < k && u < thr;
        const bool isd = j < k && u >= thr && u > 0.0f;
        const uint32_t bu = __ballot_sync(0xffffffffu, isu), bd = __ballot_sync(0xffffffffu, isd);
        if (lane == 0) {
            wsum_u[warp] = __popc(bu);
            wsum_d[warp] = __popc(bd);
        }
        __syncthreads();
        uint32_t pu = 0, pd = 0, tu = 0, td = 0;
        for (int w = 0; w < 32; w++) {
            if (w < warp) {
                pu += wsum_u[w];
                pd += wsum_d[w];
            }
            tu += wsum_u[w];
            td += wsum_d[w];
        }
        const uint32_t lt = (1u << lane) - 1u;
        if (isu) unused[base_u + pu + __popc(bu & lt)] = (uint32_t)j;
        if (isd) didx[base_d + pd + __popc(bd & lt)] = (uint32_t)j;
        base_u += tu;
        base_d += td;
        __syncthreads();
    }
    if (tid == 0) {
        nun_s = base_u;
        ndon_s = base_d;
    }
    __syncthreads();
    const uint32_t nun = nun_s, ndon = ndon_s;
    if (nun == 0) return;  // src/lib.rs:319-321: no draws when nothing is unused
    const unsigned long long cur = *cursor;
    if (cur + ndon > capacity) {  // the host-drawn stream is too short: flag it, change nothing
        if (tid == 0) *cursor = capacity + 1;
        return;
    }
    // keys/didx have room for next_pow2(k) entries; pad with -inf (sorts last).
    // Up to kReviveSmemSort entries the sort runs in shared memory.
    uint32_t n2 = 1;
    while (n2 < ndon) n2 <<= 1;
    const bool in_smem = n2 <= smem_sort;
    double* sk = in_smem ? sort_keys : keys;
    uint32_t* si = in_smem ? (uint32_t*)(sort_keys + smem_sort) : didx;
    for (uint32_t i = tid; i < n2; i += 1024) {
        if (i < ndon) {
            const uint32_t j = didx[i];
            sk[i] = log((double)usage[j]) - gstream[cur + i];
            si[i] = j;
        } else {
            sk[i] = -__longlong_as_double(0x7ff0000000000000ll);
            si[i] = 0xffffffffu;
        }
    }
    __syncthreads();
    // Bitonic sort of (key, index) by key, descending overall.
    for (uint32_t k2 = 2; k2 <= n2; k2 <<= 1) {
        for (uint32_t jj = k2 >> 1; jj > 0; jj >>= 1) {
            for (uint32_t i = tid; i < n2; i += 1024) {
                const uint32_t pi = i ^ jj;
                if (pi > i) {
                    const double a = sk[i], b = sk[pi];
                    const bool desc = (i & k2) == 0;
                    if (desc ? (a < b) : (a > b)) {
                        sk[i] = b;
                        sk[pi] = a;
                        const uint32_t t = si[i];
                        si[i] = si[pi];
                        si[pi] = t;
                    }
                }
            }
            __syncthreads();
        }
    }
    if (in_smem) {
        for (uint32_t i = tid; i < ndon; i += 1024) didx[i] = si[i];
        __syncthreads();
    }
    const uint32_t nsplit = min(nun, ndon);
    // Each split pair is independent (distinct donors, distinct unused slots).
    for (uint32_t pidx = warp; pidx < nsplit; pidx += 32) {
        const uint32_t src = didx[pidx], dst = unused[pidx];
        const float half = __fdiv_rn(usage[src], 2.0f);
        bool same = true;
        for (int t = lane; t < d; t += 32) {
            const float off = (t % 2 == 0) ? 1e-4f : -1e-4f;
            const float cv = c[(size_t)src * d + t];
            const float a = __fmul_rn(cv, __fsub_rn(1.0f, off));
            const float b = __fmul_rn(cv, __fadd_rn(1.0f, off));
            c[(size_t)src * d + t] = a;
            c[(size_t)dst * d + t] = b;
            same = same && (a == b);
        }
        same = __all_sync(0xffffffffu, same);
        if (lane == 0) {
            // A zero donor would give an identical child: nudge one coordinate up.
            if (same) c[(size_t)dst * d] = nextafterf(c[(size_t)dst * d], __int_as_float(0x7f800000));
            usage[src] = half;
            usage[dst] = half;
        }
    }
    __syncthreads();
    if (tid == 0) {
        *cursor = cur + ndon;
        *n_splits += nsplit;
    }
}

__global__ void __launch_bounds__(1024) k_revive(int k, int d, float* __restrict__ c, float* __restrict__ usage,
                                                 float tau, const double* __restrict__ gstream,
                                                 unsigned long long* __restrict__ cursor, double* __restrict__ keys,
                                                 uint32_t* __restrict__ didx, uint32_t* __restrict__ unused,
                                                 unsigned long long* __restrict__ n_splits,
                                                 unsigned long long capacity, const int* __restrict__ step,
                                                 int every) {
    extern __shared__ double sort_keys[];
    if ((*step + 1) % every != 0 || !(tau > 0.0f)) return;  // every 5th step (src/lib.rs:463-465)
    revive_cta(k, d, c, usage, tau, gstream, cursor, keys, didx, unused, n_splits, capacity, sort_keys,
               kReviveSmemSort);
}

__global__ void k_step_incr(int* step) { *step += 1; }

// Closing mean (src/lib.rs:481-489): c_j = pass_sum_j * (1 / pass_count_j) when
// the last pass assigned rows to j (f32), or the FP64 sums divided in f64.
__global__ void k_closing_mean(int k, int d, float* __restrict__ c, const unsigned long long* __restrict__ pass_counts,
                               const float* __restrict__ pass_sums, const double* __restrict__ pass_sums64) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)k * d) return;
    const size_t j = i / d;
    const unsigned long long n = pass_counts[j];
    if (n == 0) return;
    if (pass_sums64) {
        c[i] = (float)(pass_sums64[i] / (double)n);
    } else {
        const float inv = __fdiv_rn(1.0f, (float)n);
        c[i] = __fmul_rn(pass_sums[i], inv);
    }
}

}  // namespace emb
