// Kernels around the proposer's grouped search: splitting rows by confidence,
// bucketing (row, proposed group) pairs into per-group row tiles, merging each
// row's per-group top-2 into one candidate pair, and the non-learned proposer
// (nearest group centroids) the network is measured against.
#pragma once
#include "common.cuh"

namespace emb {

constexpr int kBucketTile = 128;  // rows per bucket tile (the tensor-core kernel's M)

// Rows whose proposal confidence reaches thr go to the grouped search (hc), the
// others to the full search (lc). Lists hold absolute row indices (row0 + r) and
// chunk-local ones; counts in ctr[0] (hc) and ctr[1] (lc); one atomic per warp and list.
__global__ void k_split_confidence(const float* __restrict__ conf, int m, float thr, uint32_t row0,
                                   uint32_t* __restrict__ hc_abs, uint32_t* __restrict__ hc_loc,
                                   uint32_t* __restrict__ lc_abs, uint32_t* __restrict__ lc_loc,
                                   uint32_t* __restrict__ ctr) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x, lane = threadIdx.x & 31;
    const bool in = r < m;
    const bool hc = in && conf[r] >= thr;
    const uint32_t mh = __ballot_sync(0xffffffffu, hc), ml = __ballot_sync(0xffffffffu, in && !hc);
    uint32_t bh = 0, bl = 0;
    if (lane == 0) {
        if (mh) bh = atomicAdd(ctr, (uint32_t)__popc(mh));
        if (ml) bl = atomicAdd(ctr + 1, (uint32_t)__popc(ml));
    }
    bh = __shfl_sync(0xffffffffu, bh, 0);
    bl = __shfl_sync(0xffffffffu, bl, 0);
    if (!in) return;
    const uint32_t below = (1u << lane) - 1u;
    const uint32_t slot = hc ? bh + __popc(mh & below) : bl + __popc(ml & below);
    (hc ? hc_abs : lc_abs)[slot] = row0 + (uint32_t)r;
    (hc ? hc_loc : lc_loc)[slot] = (uint32_t)r;
}

constexpr int kBucketPairs = 2048;  // (row, slot) pairs per bucketing block (8 per thread)

// counts[g] += number of (hc row, slot < cnt[row]) pairs proposing group g (a
// shared-memory histogram per block, one global atomic per group and block);
// pairs_total += all of them.
__global__ void __launch_bounds__(256) k_bucket_count(const uint16_t* __restrict__ grp, const uint8_t* __restrict__ cnt,
                                                      const uint32_t* __restrict__ hc_loc, int n, int top, int G,
                                                      uint32_t* __restrict__ counts,
                                                      unsigned long long* __restrict__ pairs_total) {
    __shared__ uint32_t hist[512];
    __shared__ uint32_t block_pairs;
    if (threadIdx.x == 0) block_pairs = 0;
    for (int g = threadIdx.x; g < G; g += blockDim.x) hist[g] = 0;
    __syncthreads();
    const int total = n * top, i0 = blockIdx.x * kBucketPairs;
    const int i1 = i0 + kBucketPairs < total ? i0 + kBucketPairs : total;
    for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
        const uint32_t r = hc_loc[i / top];
        const int s = i % top;
        if (s < cnt[r]) atomicAdd(&hist[grp[(size_t)r * top + s]], 1u);
    }
    __syncthreads();
    for (int g = threadIdx.x; g < G; g += blockDim.x)
        if (hist[g]) {
            atomicAdd(&counts[g], hist[g]);
            atomicAdd(&block_pairs, hist[g]);
        }
    __syncthreads();
    if (threadIdx.x == 0 && block_pairs) atomicAdd(pairs_total, (unsigned long long)block_pairs);
}

// One block: group g's bucket starts at the sum of the earlier groups' counts,
// each rounded up to whole tiles; tile_info gives every bucket tile its group's
// (first column, column tiles) ((0, 0) past the last), cursor[g] starts at the
// bucket's first position.
__global__ void k_bucket_layout(const uint32_t* __restrict__ counts, int G, int ntile_max,
                                const int* __restrict__ cbeg, const int* __restrict__ ntiles,
                                uint32_t* __restrict__ cursor, int2* __restrict__ tile_info) {
    __shared__ uint32_t start[1025];
    for (int t = threadIdx.x; t < ntile_max; t += blockDim.x) tile_info[t] = make_int2(0, 0);
    if (threadIdx.x == 0) {
        uint32_t acc = 0;
        for (int g = 0; g < G; g++) {
            start[g] = acc;
            acc += (counts[g] + kBucketTile - 1) / kBucketTile * kBucketTile;
        }
        start[G] = acc;
    }
    __syncthreads();
    for (int g = threadIdx.x; g < G; g += blockDim.x) {
        cursor[g] = start[g];
        const int2 v = make_int2(cbeg[g], ntiles[g]);
        for (uint32_t t = start[g] / kBucketTile; t < start[g + 1] / kBucketTile; t++) tile_info[t] = v;
    }
}

// Every position of the bucket array first names a valid row (padding positions
// are scored and ignored).
__global__ void k_fill_first(uint32_t* __restrict__ out, size_t n, const uint32_t* __restrict__ src) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = src[0];
}

// Place each (hc row, slot < cnt) pair in its group's bucket: brow[pos] =
// rows[hc row] (the caller's numbering), bpos[i * top + s] = pos (UINT32_MAX for slots not searched). Each block
// ranks its pairs in a shared-memory histogram and reserves one range per group.
// The order inside a bucket does not affect any result.
__global__ void __launch_bounds__(256) k_bucket_scatter(const uint16_t* __restrict__ grp,
                                                        const uint8_t* __restrict__ cnt,
                                                        const uint32_t* __restrict__ hc_loc,
                                                        const uint32_t* __restrict__ hc_abs, int n, int top, int G,
                                                        uint32_t* __restrict__ cursor, uint32_t* __restrict__ brow,
                                                        uint32_t* __restrict__ bpos) {
    __shared__ uint32_t hist[512], base[512];
    for (int g = threadIdx.x; g < G; g += blockDim.x) hist[g] = 0;
    __syncthreads();
    const int total = n * top, i0 = blockIdx.x * kBucketPairs;
    constexpr int per = kBucketPairs / 256;
    uint32_t rank[per];
    int gg[per];
#pragma unroll
    for (int j = 0; j < per; j++) {
        const int i = i0 + j * 256 + (int)threadIdx.x;
        gg[j] = -1;
        rank[j] = 0;
        if (i < total) {
            const uint32_t r = hc_loc[i / top];
            const int s = i % top;
            if (s < cnt[r]) {
                gg[j] = grp[(size_t)r * top + s];
                rank[j] = atomicAdd(&hist[gg[j]], 1u);
            }
        }
    }
    __syncthreads();
    for (int g = threadIdx.x; g < G; g += blockDim.x)
        if (hist[g]) base[g] = atomicAdd(&cursor[g], hist[g]);
    __syncthreads();
#pragma unroll
    for (int j = 0; j < per; j++) {
        const int i = i0 + j * 256 + (int)threadIdx.x;
        if (i >= total) continue;
        if (gg[j] < 0) {
            bpos[i] = 0xffffffffu;
            continue;
        }
        const uint32_t pos = base[gg[j]] + rank[j];
        brow[pos] = hc_abs[i / top];
        bpos[i] = pos;
    }
}

// Per group: (max |c|, max |norm|) over the columns its tiles cover in the sorted
// copy (padding rows excluded; columns of neighbouring groups that a tile
// reaches included), upper-rounded as the bounds over all k are. One warp per
// group, a lane per column.
__global__ void k_group_bounds(const float* __restrict__ c, const float* __restrict__ norms,
                               const uint32_t* __restrict__ perm, size_t ks, int d, const int* __restrict__ cbeg,
                               const int* __restrict__ ntiles, int tile_cols, int G, float2* __restrict__ gb) {
    const int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (g >= G) return;
    const size_t c0 = (size_t)cbeg[g];
    size_t c1 = c0 + (size_t)ntiles[g] * tile_cols;
    if (c1 > ks) c1 = ks;
    float cm = 0.0f, nm = 0.0f;
    for (size_t j = c0 + lane; j < c1; j += 32) {
        if (perm[j] == 0xffffffffu) continue;
        float ss = 0.0f;
        for (int t = 0; t < d; t++) {
            const float v = c[j * d + t];
            ss = __fmaf_ru(v, v, ss);
        }
        cm = fmaxf(cm, __fmul_ru(__fsqrt_ru(ss), 1.0000005f));
        nm = fmaxf(nm, fabsf(norms[j]));
    }
    for (int o = 16; o; o >>= 1) {
        cm = fmaxf(cm, __shfl_xor_sync(0xffffffffu, cm, o));
        nm = fmaxf(nm, __shfl_xor_sync(0xffffffffu, nm, o));
    }
    if (lane == 0) gb[g] = make_float2(cm, nm);
}

// Lexicographic (score, index) minimum of two candidates.
EMB_DEV void lex_min_into(float& s, uint32_t& j, float s2, uint32_t j2) {
    if (lex_less(s2, j2, s, j)) {
        s = s2;
        j = j2;
    }
}

// Per hc row (one warp; lane = slot, top <= 32): merge the top-2 of its bucket
// positions (columns of the sorted matrix mapped to centroid indices through
// perm, padding columns dropped) into the part_s/part_i layout the certification
// reads (one split): the lexicographic (score, index) minimum, then the minimum
// among the candidates with another index (a centroid seen twice, when tiles of
// neighbouring groups overlap, counts once). Also the row's bounds: the largest
// (max |c|, max |norm|) of its searched groups.
__global__ void k_merge_slots(int n, int top, const uint32_t* __restrict__ bpos, const float* __restrict__ gs,
                              const uint32_t* __restrict__ gi, const uint32_t* __restrict__ perm, uint32_t ks,
                              float* __restrict__ part_s, uint32_t* __restrict__ part_i,
                              const uint16_t* __restrict__ grp, const uint32_t* __restrict__ hc_loc,
                              const float2* __restrict__ gb, float2* __restrict__ row_bounds) {
    const int i = (int)(((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (i >= n) return;
    const float inf = __int_as_float(0x7f800000);
    float a_s = inf, b_s = inf;  // this lane's two candidates, a before b
    uint32_t a_j = 0xffffffffu, b_j = 0xffffffffu;
    float cm = 0.0f, nm = 0.0f;
    if (lane < top) {
        const uint32_t bp = bpos[(size_t)i * top + lane];
        if (bp != 0xffffffffu) {
            const float2 b = gb[grp[(size_t)hc_loc[i] * top + lane]];
            cm = b.x;
            nm = b.y;
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const uint32_t col = gi[(size_t)bp * 2 + e];
                const uint32_t j = col < ks ? perm[col] : 0xffffffffu;
                if (j == 0xffffffffu) continue;
                const float sc = gs[(size_t)bp * 2 + e];
                if (lex_less(sc, j, a_s, a_j)) {
                    b_s = a_s;
                    b_j = a_j;
                    a_s = sc;
                    a_j = j;
                } else if (lex_less(sc, j, b_s, b_j)) {
                    b_s = sc;
                    b_j = j;
                }
            }
        }
    }
    float s1 = a_s;
    uint32_t j1 = a_j;
    for (int o = 16; o; o >>= 1) {
        lex_min_into(s1, j1, __shfl_xor_sync(0xffffffffu, s1, o), __shfl_xor_sync(0xffffffffu, j1, o));
        cm = fmaxf(cm, __shfl_xor_sync(0xffffffffu, cm, o));
        nm = fmaxf(nm, __shfl_xor_sync(0xffffffffu, nm, o));
    }
    // A lane's two candidates are distinct centroids: if its first is the winner, its second competes.
    float s2 = a_j == j1 ? b_s : a_s;
    uint32_t j2 = a_j == j1 ? b_j : a_j;
    if (j2 == j1) {
        s2 = inf;
        j2 = 0xffffffffu;
    }
    for (int o = 16; o; o >>= 1)
        lex_min_into(s2, j2, __shfl_xor_sync(0xffffffffu, s2, o), __shfl_xor_sync(0xffffffffu, j2, o));
    if (lane == 0) {
        row_bounds[i] = make_float2(cm, nm);
        part_s[(size_t)i * 2] = s1;
        part_s[(size_t)i * 2 + 1] = s2;
        part_i[(size_t)i * 2] = j1;
        part_i[(size_t)i * 2 + 1] = j2;
    }
}

// labels[loc[i]] = src_labels[i] (and dist).
__global__ void k_scatter_results(const uint32_t* __restrict__ src_l, const float* __restrict__ src_d,
                                  const uint32_t* __restrict__ loc, int n, uint32_t* __restrict__ labels,
                                  float* __restrict__ dist) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    labels[loc[i]] = src_l[i];
    dist[loc[i]] = src_d[i];
}

// Non-learned proposer: logits[r][g] = 2 x.gc_g - |gc_g|^2 (larger is nearer),
// from the transposed group centroids gT[t][g]. 32 rows per block.
template <typename T>
__global__ void __launch_bounds__(256) k_group_logits(const T* __restrict__ x, int m, int d,
                                                      const float* __restrict__ gT, const float* __restrict__ gnorm,
                                                      int G, float* __restrict__ logits) {
    extern __shared__ float xs[];  // [32][d]
    const int r0 = blockIdx.x * 32;
    for (int t = threadIdx.x; t < 32 * d; t += blockDim.x) {
        const int r = t / d, c = t % d;
        xs[t] = r0 + r < m ? to_f32(x[(size_t)(r0 + r) * d + c]) : 0.0f;
    }
    __syncthreads();
    for (int g = threadIdx.x; g < G; g += blockDim.x) {
        float acc[32];
#pragma unroll
        for (int r = 0; r < 32; r++) acc[r] = 0.0f;
        for (int t = 0; t < d; t++) {
            const float w = gT[(size_t)t * G + g];
#pragma unroll
            for (int r = 0; r < 32; r++) acc[r] = fmaf(xs[r * d + t], w, acc[r]);
        }
        const float nn = gnorm[g];
#pragma unroll
        for (int r = 0; r < 32; r++)
            if (r0 + r < m) logits[(size_t)(r0 + r) * G + g] = 2.0f * acc[r] - nn;
    }
}

// Training targets: tgt[i] = group_of[labels[rows[i]]].
__global__ void k_gather_targets(const uint32_t* __restrict__ rows, int n, const uint32_t* __restrict__ labels,
                                 const uint32_t* __restrict__ group_of, uint32_t* __restrict__ tgt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) tgt[i] = group_of[labels[rows[i]]];
}

// Group-sorted centroid matrix: out[j] = c[perm[j]] (zeros for padding rows).
__global__ void k_gather_sorted(const float* __restrict__ c, const uint32_t* __restrict__ perm, size_t ks, int d,
                                float* __restrict__ out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ks * d) return;
    const size_t j = i / d;
    const uint32_t src = perm[j];
    out[i] = src == 0xffffffffu ? 0.0f : c[(size_t)src * d + (i - j * d)];
}

// Padding rows of the sorted matrix never win: norm 3e38.
__global__ void k_pad_norms(float* __restrict__ norms, const uint32_t* __restrict__ perm, size_t ks) {
    const size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < ks && perm[j] == 0xffffffffu) norms[j] = 3.0e38f;
}

// Rows split into BF16 hi and lo (x = hi + lo to about 2^-16), [m][kpad] with
// zeros past d: the grouped search gathers them with TMA. One thread per 8 elements.
__global__ void k_rows_split(const float* __restrict__ x, size_t m, int d, int kpad, __nv_bfloat16* __restrict__ hi,
                             __nv_bfloat16* __restrict__ lo) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int nchunk = kpad / 8;
    if (t >= m * nchunk) return;
    const size_t r = t / nchunk;
    const int k0 = (int)(t - r * nchunk) * 8;
    const float* xr = x + r * (size_t)d;
    uint32_t hw[4], lw[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const float a = k0 + 2 * i < d ? xr[k0 + 2 * i] : 0.0f;
        const float b = k0 + 2 * i + 1 < d ? xr[k0 + 2 * i + 1] : 0.0f;
        const __nv_bfloat16 ha = __float2bfloat16_rn(a), hb = __float2bfloat16_rn(b);
        const __nv_bfloat16 la = __float2bfloat16_rn(a - __bfloat162float(ha));
        const __nv_bfloat16 lb = __float2bfloat16_rn(b - __bfloat162float(hb));
        hw[i] = (uint32_t)__bfloat16_as_ushort(ha) | ((uint32_t)__bfloat16_as_ushort(hb) << 16);
        lw[i] = (uint32_t)__bfloat16_as_ushort(la) | ((uint32_t)__bfloat16_as_ushort(lb) << 16);
    }
    *reinterpret_cast<uint4*>(hi + r * kpad + k0) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
    *reinterpret_cast<uint4*>(lo + r * kpad + k0) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
}

// Strided sample of f32 rows (input statistics of the network).
__global__ void k_sample_rows(const float* __restrict__ x, size_t stride, int count, int d, float* __restrict__ out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)count * d) return;
    const size_t r = i / d;
    out[i] = x[r * stride * d + (i - r * d)];
}

}  // namespace emb
