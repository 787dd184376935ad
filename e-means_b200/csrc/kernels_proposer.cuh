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
// each rounded up to whole tiles; tile_group maps every bucket tile to its group
// (-1 past the last), cursor[g] starts at the bucket's first position.
__global__ void k_bucket_layout(const uint32_t* __restrict__ counts, int G, int ntile_max,
                                uint32_t* __restrict__ cursor, int* __restrict__ tile_group) {
    __shared__ uint32_t start[1025];
    for (int t = threadIdx.x; t < ntile_max; t += blockDim.x) tile_group[t] = -1;
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
        for (uint32_t t = start[g] / kBucketTile; t < start[g + 1] / kBucketTile; t++) tile_group[t] = g;
    }
}

// Every position of the bucket array first names a valid row (padding positions
// are scored and ignored).
__global__ void k_fill_first(uint32_t* __restrict__ out, size_t n, const uint32_t* __restrict__ src) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = src[0];
}

// Place each (hc row, slot < cnt) pair in its group's bucket: brow[pos] = absolute
// row, bpos[i * top + s] = pos (UINT32_MAX for slots not searched). Each block
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

// Per hc row: merge the top-2 of its `top` bucket positions (columns of the sorted
// matrix, mapped to centroid indices through perm; padding columns dropped; a
// centroid seen twice, when tiles of neighbouring groups overlap, counted once)
// into the part_s/part_i layout the certification reads (one split).
__global__ void k_merge_slots(int n, int top, const uint32_t* __restrict__ bpos, const float* __restrict__ gs,
                              const uint32_t* __restrict__ gi, const uint32_t* __restrict__ perm, uint32_t ks,
                              float* __restrict__ part_s, uint32_t* __restrict__ part_i) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Top2 t;
    t.init();
    for (int s = 0; s < top; s++) {
        const uint32_t bp = bpos[(size_t)i * top + s];
        if (bp == 0xffffffffu) continue;  // slot not searched
        const size_t pos = bp;
#pragma unroll
        for (int e = 0; e < 2; e++) {
            const uint32_t col = gi[pos * 2 + e];
            const uint32_t j = col < ks ? perm[col] : 0xffffffffu;
            if (j == 0xffffffffu || j == t.i1 || j == t.i2) continue;
            t.push(gs[pos * 2 + e], j);
        }
    }
    part_s[(size_t)i * 2] = t.s1;
    part_s[(size_t)i * 2 + 1] = t.s2;
    part_i[(size_t)i * 2] = t.i1;
    part_i[(size_t)i * 2 + 1] = t.i2;
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

// Strided sample of f32 rows (input statistics of the network).
__global__ void k_sample_rows(const float* __restrict__ x, size_t stride, int count, int d, float* __restrict__ out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)count * d) return;
    const size_t r = i / d;
    out[i] = x[r * stride * d + (i - r * d)];
}

}  // namespace emb
