// FP32 SIMT fused assign: x . c^T contraction in registers with a running
// top-2 per row in the epilogue, so no m x k score matrix ever reaches HBM.
// This is the plain FP32 form of the search (src/cpu.rs:108-167 computes the
// same scores on the CPU); its result is certified and re-scored exactly by
// kernels_exact.cuh.
#pragma once
#include "common.cuh"

namespace emb {

constexpr int kSimtBM = 128, kSimtBN = 128, kSimtBK = 16, kSimtThreads = 256;

// Loads a BM x BK slab of rows (or centroids) into registers: thread t takes
// row t/2, columns (t%2)*8 .. +8 of the slab. Out-of-range entries are zero.
template <typename T>
EMB_DEV void simt_load(float (&r)[8], const T* __restrict__ base, const uint32_t* __restrict__ gather, int row0,
                       int nrows, int d, int k0, bool vec4) {
    int t = threadIdx.x;
    int row = row0 + (t >> 1);
    int col = k0 + (t & 1) * 8;
    if (row >= nrows) {
#pragma unroll
        for (int i = 0; i < 8; i++) r[i] = 0.0f;
        return;
    }
    size_t src = gather ? gather[row] : (size_t)row;
    const T* p = base + src * (size_t)d + col;
    if (sizeof(T) == 4 && vec4 && col + 8 <= d) {
        float4 a = *reinterpret_cast<const float4*>(p);
        float4 b = *reinterpret_cast<const float4*>(p + 4);
        r[0] = a.x; r[1] = a.y; r[2] = a.z; r[3] = a.w;
        r[4] = b.x; r[5] = b.y; r[6] = b.z; r[7] = b.w;
    } else {
#pragma unroll
        for (int i = 0; i < 8; i++) r[i] = (col + i < d) ? to_f32(p[i]) : 0.0f;
    }
}

// Grid: (ceil(m / 128), nsplit). CTA (bx, by) searches rows [128 bx, +128)
// against centroid tiles by, by + nsplit, ... and writes its top-2 per row to
// part_s/part_i[by][row][0..1].
template <typename T>
__global__ void __launch_bounds__(kSimtThreads, 1)
k_assign_simt(const T* __restrict__ x, const uint32_t* __restrict__ gather, int m, int d,
              const float* __restrict__ c, const float* __restrict__ norms, int k,
              float* __restrict__ part_s, uint32_t* __restrict__ part_i, int vec4) {
    __shared__ __align__(16) float As[2][kSimtBK][kSimtBM];
    __shared__ __align__(16) float Bs[2][kSimtBK][kSimtBN];
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    const int row0 = blockIdx.x * kSimtBM;
    const int nsplit = gridDim.y;
    const int ntiles = (k + kSimtBN - 1) / kSimtBN;
    const int nk = (d + kSimtBK - 1) / kSimtBK;

    Top2 top[8];
#pragma unroll
    for (int i = 0; i < 8; i++) top[i].init();

    for (int tile = blockIdx.y; tile < ntiles; tile += nsplit) {
        const int col0 = tile * kSimtBN;
        float acc[8][8];
#pragma unroll
        for (int i = 0; i < 8; i++)
#pragma unroll
            for (int j = 0; j < 8; j++) acc[i][j] = 0.0f;

        float ra[8], rb[8];
        simt_load(ra, x, gather, row0, m, d, 0, vec4);
        simt_load(rb, c, (const uint32_t*)nullptr, col0, k, d, 0, vec4);
        __syncthreads();  // previous tile's readers are done with buffer 0
        {
            int r = tid >> 1, kk0 = (tid & 1) * 8;
#pragma unroll
            for (int i = 0; i < 8; i++) {
                As[0][kk0 + i][r] = ra[i];
                Bs[0][kk0 + i][r] = rb[i];
            }
        }
        __syncthreads();
        for (int kt = 0; kt < nk; kt++) {
            const int buf = kt & 1;
            if (kt + 1 < nk) {
                simt_load(ra, x, gather, row0, m, d, (kt + 1) * kSimtBK, vec4);
                simt_load(rb, c, (const uint32_t*)nullptr, col0, k, d, (kt + 1) * kSimtBK, vec4);
            }
#pragma unroll
            for (int kk = 0; kk < kSimtBK; kk++) {
                float a[8], b[8];
                float4 a0 = *reinterpret_cast<const float4*>(&As[buf][kk][ty * 4]);
                float4 a1 = *reinterpret_cast<const float4*>(&As[buf][kk][64 + ty * 4]);
                float4 b0 = *reinterpret_cast<const float4*>(&Bs[buf][kk][tx * 4]);
                float4 b1 = *reinterpret_cast<const float4*>(&Bs[buf][kk][64 + tx * 4]);
                a[0] = a0.x; a[1] = a0.y; a[2] = a0.z; a[3] = a0.w;
                a[4] = a1.x; a[5] = a1.y; a[6] = a1.z; a[7] = a1.w;
                b[0] = b0.x; b[1] = b0.y; b[2] = b0.z; b[3] = b0.w;
                b[4] = b1.x; b[5] = b1.y; b[6] = b1.z; b[7] = b1.w;
#pragma unroll
                for (int i = 0; i < 8; i++)
#pragma unroll
                    for (int j = 0; j < 8; j++) acc[i][j] = __fmaf_rn(a[i], b[j], acc[i][j]);
            }
            if (kt + 1 < nk) {
                int r = tid >> 1, kk0 = (tid & 1) * 8;
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    As[buf ^ 1][kk0 + i][r] = ra[i];
                    Bs[buf ^ 1][kk0 + i][r] = rb[i];
                }
            }
            __syncthreads();
        }
        // Epilogue: score = norms_j - 2 acc (one rounding), running top-2 per row.
#pragma unroll
        for (int j = 0; j < 8; j++) {
            int col = col0 + (j < 4 ? tx * 4 + j : 64 + tx * 4 + (j - 4));
            if (col < k) {
                float nj = norms[col];
#pragma unroll
                for (int i = 0; i < 8; i++) top[i].push(__fmaf_rn(-2.0f, acc[i][j], nj), (uint32_t)col);
            }
        }
    }
    // Merge the 16 column-threads of each row group (lanes differing in tx).
#pragma unroll
    for (int i = 0; i < 8; i++) {
        top[i].merge_shfl_xor(1);
        top[i].merge_shfl_xor(2);
        top[i].merge_shfl_xor(4);
        top[i].merge_shfl_xor(8);
    }
    if (tx == 0) {
#pragma unroll
        for (int i = 0; i < 8; i++) {
            int row = row0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + (i - 4));
            if (row < m) {
                size_t o = ((size_t)blockIdx.y * m + row) * 2;
                part_s[o] = top[i].s1;
                part_i[o] = top[i].i1;
                part_s[o + 1] = top[i].s2;
                part_i[o + 1] = top[i].i2;
            }
        }
    }
}

}  // namespace emb
