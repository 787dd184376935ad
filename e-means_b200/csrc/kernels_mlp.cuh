// Kernels of the learned proposer: a BF16 MLP d -> H -> H -> G that predicts a
// row's centroid group, trained on the GPU with its own forward and backward
// kernels (FP32 accumulation, FP32 master weights, Adam).
//
// The GEMM is one tiled tensor-core kernel, C[M x N] = A[M x K] . B[K x N] in
// BF16 with FP32 accumulation (mma.sync m16n8k16, ldmatrix from 128 x 32 smem
// tiles), that reads either operand in either orientation, so the forward pass
// (X W^T), the input gradient (dY W) and the weight gradient (dY^T X) all run on
// it without transposing anything in memory. Epilogues: FP32 out, or BF16 out
// with bias and ReLU fused.
#pragma once
#include <cuda_bf16.h>

#include "common.cuh"

namespace emb {

constexpr int kGemmBM = 128, kGemmBN = 128, kGemmBK = 32, kGemmThreads = 256;
constexpr int kGemmPad = 8;  // bf16 elements of row padding against ldmatrix bank conflicts

// Operand orientation: A is M x K stored row-major (kMK, A[m * lda + k]) or
// K x M (kKM, A[k * lda + m]); B is K x N stored as N x K (kNK, B[n * ldb + k])
// or K x N (kKN, B[k * ldb + n]).
enum { kMK = 0, kKM = 1, kNK = 0, kKN = 1 };
// Epilogue: FP32 store; BF16 store of (acc + bias[n]); BF16 store of relu(acc + bias[n]);
// FP32 store of (acc + bias[n]); BF16 store of acc.
enum { kEpiF32 = 0, kEpiBiasBf16 = 1, kEpiBiasReluBf16 = 2, kEpiBiasF32 = 3, kEpiBf16 = 4 };

EMB_DEV void ldsm_x4(uint32_t (&r)[4], const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"((uint32_t)__cvta_generic_to_shared(p)));
}
EMB_DEV void ldsm_x4_t(uint32_t (&r)[4], const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"((uint32_t)__cvta_generic_to_shared(p)));
}
EMB_DEV void mma_bf16_16816(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Copies a 2-D bf16 tile (rows x cols, cols a multiple of 8) from global memory
// (row stride ld elements, valid region vr x vc) into shared memory (row stride
// cols + kGemmPad), zero-filling outside the valid region. 16-byte vectors when
// the 8 elements are in range and aligned, element by element otherwise.
template <int ROWS, int COLS>
EMB_DEV void gemm_tile_load(__nv_bfloat16* s, const __nv_bfloat16* __restrict__ g, size_t ld, int r0, int c0, int vr,
                            int vc) {
    constexpr int VEC = COLS / 8;
    for (int t = threadIdx.x; t < ROWS * VEC; t += kGemmThreads) {
        const int r = t / VEC, cv = (t % VEC) * 8;
        const int gr = r0 + r, gc = c0 + cv;
        __nv_bfloat16* dst = s + r * (COLS + kGemmPad) + cv;
        if (gr < vr && gc + 8 <= vc && (ld & 7) == 0 && ((uintptr_t)g & 15) == 0) {
            *reinterpret_cast<uint4*>(dst) = *reinterpret_cast<const uint4*>(g + (size_t)gr * ld + gc);
        } else {
#pragma unroll
            for (int i = 0; i < 8; i++)
                dst[i] = (gr < vr && gc + i < vc) ? g[(size_t)gr * ld + gc + i] : __float2bfloat16(0.0f);
        }
    }
}

// C = A . B (+ epilogue). Grid: (ceil(N / 128), ceil(M / 128)). 8 warps as 2 (M) x 4 (N),
// each computing a 64 x 32 block as 4 x 4 m16n8 tiles.
template <int AL, int BL, int EPI>
__global__ void __launch_bounds__(kGemmThreads)
k_gemm_bf16(int M, int N, int K, const __nv_bfloat16* __restrict__ A, size_t lda, const __nv_bfloat16* __restrict__ B,
            size_t ldb, void* __restrict__ C, size_t ldc, const float* __restrict__ bias) {
    // A tile: [BM][BK] (kMK) or [BK][BM] (kKM); B tile: [BN][BK] (kNK) or [BK][BN] (kKN).
    __shared__ __align__(16) __nv_bfloat16 As[kGemmBM * (kGemmBK + kGemmPad) > kGemmBK * (kGemmBM + kGemmPad)
                                                  ? kGemmBM * (kGemmBK + kGemmPad)
                                                  : kGemmBK * (kGemmBM + kGemmPad)];
    __shared__ __align__(16) __nv_bfloat16 Bs[kGemmBN * (kGemmBK + kGemmPad) > kGemmBK * (kGemmBN + kGemmPad)
                                                  ? kGemmBN * (kGemmBK + kGemmPad)
                                                  : kGemmBK * (kGemmBN + kGemmPad)];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wm = warp >> 2, wn = warp & 3;  // 2 x 4 warps
    const int m0 = blockIdx.y * kGemmBM, n0 = blockIdx.x * kGemmBN;
    float acc[4][4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int e = 0; e < 4; e++) acc[i][j][e] = 0.0f;

    for (int k0 = 0; k0 < K; k0 += kGemmBK) {
        __syncthreads();
        if (AL == kMK) gemm_tile_load<kGemmBM, kGemmBK>(As, A, lda, m0, k0, M, K);
        else gemm_tile_load<kGemmBK, kGemmBM>(As, A, lda, k0, m0, K, M);
        if (BL == kNK) gemm_tile_load<kGemmBN, kGemmBK>(Bs, B, ldb, n0, k0, N, K);
        else gemm_tile_load<kGemmBK, kGemmBN>(Bs, B, ldb, k0, n0, K, N);
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kGemmBK; kk += 16) {
            uint32_t af[4][4], bfr[4][2];
            const int r8 = lane & 7, mi = lane >> 3;  // ldmatrix: this lane addresses row r8 of matrix mi
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const int mb = wm * 64 + i * 16;
                if (AL == kMK) {
                    // matrices: (m 0-7, k 0-7), (m 8-15, k 0-7), (m 0-7, k 8-15), (m 8-15, k 8-15)
                    const int row = mb + r8 + ((mi & 1) << 3), col = kk + ((mi >> 1) << 3);
                    ldsm_x4(af[i], As + row * (kGemmBK + kGemmPad) + col);
                } else {
                    // stored [k][m]: transposed loads of the same four 8 x 8 blocks
                    const int krow = kk + r8 + ((mi >> 1) << 3), mcol = mb + ((mi & 1) << 3);
                    ldsm_x4_t(af[i], As + krow * (kGemmBM + kGemmPad) + mcol);
                }
            }
#pragma unroll
            for (int jp = 0; jp < 2; jp++) {
                const int nb = wn * 32 + jp * 16;
                uint32_t r[4];
                if (BL == kNK) {
                    // matrices: (n 0-7, k 0-7), (n 0-7, k 8-15), (n 8-15, k 0-7), (n 8-15, k 8-15)
                    const int row = nb + r8 + ((mi >> 1) << 3), col = kk + ((mi & 1) << 3);
                    ldsm_x4(r, Bs + row * (kGemmBK + kGemmPad) + col);
                } else {
                    const int krow = kk + r8 + ((mi & 1) << 3), ncol = nb + ((mi >> 1) << 3);
                    ldsm_x4_t(r, Bs + krow * (kGemmBN + kGemmPad) + ncol);
                }
                bfr[2 * jp][0] = r[0];
                bfr[2 * jp][1] = r[1];
                bfr[2 * jp + 1][0] = r[2];
                bfr[2 * jp + 1][1] = r[3];
            }
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) mma_bf16_16816(acc[i][j], af[i], bfr[j][0], bfr[j][1]);
        }
    }
    // Epilogue: lane holds rows (lane/4, +8), columns 2 (lane%4) + {0, 1} of each m16n8 tile.
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int row = m0 + wm * 64 + i * 16 + (lane >> 2) + h * 8;
                const int col = n0 + wn * 32 + j * 8 + (lane & 3) * 2;
                if (row >= M) continue;
#pragma unroll
                for (int e = 0; e < 2; e++) {
                    if (col + e >= N) continue;
                    float v = acc[i][j][2 * h + e];
                    if (EPI == kEpiF32) {
                        ((float*)C)[(size_t)row * ldc + col + e] = v;
                    } else if (EPI == kEpiBiasF32) {
                        ((float*)C)[(size_t)row * ldc + col + e] = v + bias[col + e];
                    } else if (EPI == kEpiBf16) {
                        ((__nv_bfloat16*)C)[(size_t)row * ldc + col + e] = __float2bfloat16_rn(v);
                    } else {
                        v += bias[col + e];
                        if (EPI == kEpiBiasReluBf16) v = fmaxf(v, 0.0f);
                        ((__nv_bfloat16*)C)[(size_t)row * ldc + col + e] = __float2bfloat16_rn(v);
                    }
                }
            }
}

// Standardised BF16 network input: (x - mean) * inv_std per dimension.
template <typename T>
__global__ void k_mlp_input(const T* __restrict__ x, const uint32_t* __restrict__ rows, int m, int d,
                            const float* __restrict__ mean, const float* __restrict__ inv_std,
                            __nv_bfloat16* __restrict__ out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)m * d) return;
    const size_t r = i / d, t = i - r * d;
    const size_t src = rows ? rows[r] : r;
    out[i] = __float2bfloat16_rn((to_f32(x[src * d + t]) - mean[t]) * inv_std[t]);
}

// Softmax cross-entropy over G logits per row (one warp per row): writes the
// gradient (softmax - onehot) / scale as BF16 and accumulates the loss.
__global__ void k_softmax_xent(const float* __restrict__ logits, const uint32_t* __restrict__ target, int m, int G,
                               float scale, __nv_bfloat16* __restrict__ grad, float* __restrict__ loss) {
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (row >= m) return;
    const float* l = logits + (size_t)row * G;
    float mx = -INFINITY;
    for (int g = lane; g < G; g += 32) mx = fmaxf(mx, l[g]);
    for (int o = 16; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    float se = 0.0f;
    for (int g = lane; g < G; g += 32) se += __expf(l[g] - mx);
    for (int o = 16; o; o >>= 1) se += __shfl_xor_sync(0xffffffffu, se, o);
    const uint32_t t = target[row];
    const float inv = 1.0f / se;
    for (int g = lane; g < G; g += 32) {
        const float p = __expf(l[g] - mx) * inv;
        grad[(size_t)row * G + g] = __float2bfloat16_rn((p - (g == (int)t ? 1.0f : 0.0f)) / scale);
    }
    if (lane == 0 && loss) atomicAdd(loss, (logf(se) + mx - l[t]) / scale);
}

// Gradient through ReLU: g *= (h > 0), both BF16.
__global__ void k_relu_grad(__nv_bfloat16* __restrict__ g, const __nv_bfloat16* __restrict__ h, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && !(__bfloat162float(h[i]) > 0.0f)) g[i] = __float2bfloat16(0.0f);
}

// Bias gradient: column sums of a BF16 m x n matrix into FP32 (one thread per column).
__global__ void k_colsum(const __nv_bfloat16* __restrict__ g, int m, int n, float* __restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    float s = 0.0f;
    for (int r = 0; r < m; r++) s += __bfloat162float(g[(size_t)r * n + c]);
    out[c] = s;
}

// BF16 copy of FP32 values.
__global__ void k_f32_to_bf16(const float* __restrict__ w, __nv_bfloat16* __restrict__ wb, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) wb[i] = __float2bfloat16_rn(w[i]);
}

// Adam on FP32 master weights, refreshing their BF16 copy.
__global__ void k_adam(float* __restrict__ w, __nv_bfloat16* __restrict__ wb, const float* __restrict__ g,
                       float* __restrict__ m1, float* __restrict__ m2, size_t n, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float a = b1 * m1[i] + (1.0f - b1) * gi;
    const float b = b2 * m2[i] + (1.0f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = b;
    const float v = w[i] - lr * (a / c1) / (sqrtf(b / c2) + eps);
    w[i] = v;
    if (wb) wb[i] = __float2bfloat16_rn(v);
}

// Top-m groups per row from G logits (one warp per row), the softmax mass those
// m groups carry (the proposer's confidence), and how many of them to search:
// the fewest whose mass reaches mass_target (all m when mass_target <= 0 or
// when the m together fall short).
__global__ void k_topm_groups(const float* __restrict__ logits, int m, int G, int top, uint16_t* __restrict__ groups,
                              float* __restrict__ conf, float mass_target, uint8_t* __restrict__ cnt) {
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (row >= m) return;
    const float* l = logits + (size_t)row * G;
    // Each lane keeps its G/32 logits; repeated warp argmax picks the top m.
    float v[16];
    const int per = (G + 31) / 32;
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = (i < per && lane + 32 * i < G) ? l[lane + 32 * i] : -INFINITY;
    float mx = -INFINITY;
#pragma unroll
    for (int i = 0; i < 16; i++) mx = fmaxf(mx, v[i]);
    for (int o = 16; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    float se = 0.0f;
#pragma unroll
    for (int i = 0; i < 16; i++) se += (v[i] > -INFINITY) ? __expf(v[i] - mx) : 0.0f;
    for (int o = 16; o; o >>= 1) se += __shfl_xor_sync(0xffffffffu, se, o);
    float mass = 0.0f;
    int n_search = top;
    for (int s = 0; s < top; s++) {
        float bv = -INFINITY;
        int bi = 0x7fffffff;
#pragma unroll
        for (int i = 0; i < 16; i++)
            if (v[i] > bv) {
                bv = v[i];
                bi = lane + 32 * i;
            }
        for (int o = 16; o; o >>= 1) {
            const float ov = __shfl_xor_sync(0xffffffffu, bv, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ov > bv || (ov == bv && oi < bi)) {
                bv = ov;
                bi = oi;
            }
        }
        if (bi >= G) bi = 0;  // no finite logit left (a diverged network): any valid group
        if (lane == 0) groups[(size_t)row * top + s] = (uint16_t)bi;
        mass += __expf(bv - mx);
        if (mass_target > 0.0f && n_search == top && mass >= mass_target * se) n_search = s + 1;
        if ((bi & 31) == lane) {
#pragma unroll
            for (int i = 0; i < 16; i++)
                if (lane + 32 * i == bi) v[i] = -INFINITY;
        }
    }
    if (lane == 0) {
        conf[row] = mass / se;
        cnt[row] = (uint8_t)n_search;
    }
}

}  // namespace emb
