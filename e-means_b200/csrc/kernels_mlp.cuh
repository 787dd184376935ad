// Kernels of the learned proposer: a BF16 MLP d -> H -> H -> G that predicts a
// row's centroid group, trained on the GPU with its own forward and backward
// kernels (FP32 accumulation, FP32 master weights, Adam). Its GEMMs run on the
// tcgen05 kernel of kernels_gemm_tc.cuh; this file holds the element-wise and
// reduction kernels around them (input standardisation, softmax cross-entropy,
// ReLU gradients, column sums, Adam, the top-m group selection).
#pragma once
#include <cuda_bf16.h>

#include "common.cuh"

namespace emb {

// Epilogue of the network's GEMM (k_gemm_tc): FP32 store; BF16 store of (acc + bias[n]);
// BF16 store of relu(acc + bias[n]); FP32 store of (acc + bias[n]); BF16 store of acc.
enum { kEpiF32 = 0, kEpiBiasBf16 = 1, kEpiBiasReluBf16 = 2, kEpiBiasF32 = 3, kEpiBf16 = 4 };

// Standardised BF16 network input: (x - mean) * inv_std per dimension, rows of
// stride ld >= d.
template <typename T>
__global__ void k_mlp_input(const T* __restrict__ x, const uint32_t* __restrict__ rows, int m, int d,
                            const float* __restrict__ mean, const float* __restrict__ inv_std,
                            __nv_bfloat16* __restrict__ out, size_t ld) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)m * d) return;
    const size_t r = i / d, t = i - r * d;
    const size_t src = rows ? rows[r] : r;
    out[r * ld + t] = __float2bfloat16_rn((to_f32(x[src * d + t]) - mean[t]) * inv_std[t]);
}

// BF16 rows of C elements copied to row stride ld (the tail left as it is: the
// GEMM's tensor map reads zeros past C).
__global__ void k_pad_rows_bf16(const __nv_bfloat16* __restrict__ src, int R, int C, __nv_bfloat16* __restrict__ dst,
                                size_t ld) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)R * C) return;
    const size_t r = i / C, c = i - r * C;
    dst[r * ld + c] = src[i];
}

// Softmax cross-entropy over G logits per row (one warp per row): writes the
// gradient (softmax - onehot) / scale as BF16 and accumulates the loss.
__global__ void k_softmax_xent(const float* __restrict__ logits, const uint32_t* __restrict__ target, int m, int G,
                               float scale, __nv_bfloat16* __restrict__ grad, size_t ldg, float* __restrict__ loss) {
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
        grad[(size_t)row * ldg + g] = __float2bfloat16_rn((p - (g == (int)t ? 1.0f : 0.0f)) / scale);
    }
    if (lane == 0 && loss) atomicAdd(loss, (logf(se) + mx - l[t]) / scale);
}

// Gradient through ReLU: g *= (h > 0), both BF16.
__global__ void k_relu_grad(__nv_bfloat16* __restrict__ g, const __nv_bfloat16* __restrict__ h, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && !(__bfloat162float(h[i]) > 0.0f)) g[i] = __float2bfloat16(0.0f);
}

// Bias gradient: column sums of a BF16 m x n matrix (row stride ld) into FP32, in
// two fixed-order passes (the same bits on every run). k_colsum_part: block
// (x, y) sums rows [128 y, 128 y + 128) of columns [32 x, 32 x + 32), warp p its
// 16 rows 16 p .. 16 p + 15 in order (all 16 loads in flight), the eight warps'
// sums then in warp order, into part[y][col]. k_colsum_final adds the parts of
// a column in y order.
constexpr int kColsumRows = 128;
__global__ void __launch_bounds__(256) k_colsum_part(const __nv_bfloat16* __restrict__ g, int m, int n, size_t ld,
                                                     float* __restrict__ part) {
    __shared__ float ws[8][32];
    const int lane = threadIdx.x & 31, p = threadIdx.x >> 5;
    const int c = blockIdx.x * 32 + lane;
    const int r0 = blockIdx.y * kColsumRows + p * 16;
    float v[16];
#pragma unroll
    for (int q = 0; q < 16; q++)
        v[q] = (c < n && r0 + q < m) ? __bfloat162float(g[(size_t)(r0 + q) * ld + c]) : 0.0f;
    float s = 0.0f;
#pragma unroll
    for (int q = 0; q < 16; q++) s += v[q];
    ws[p][lane] = s;
    __syncthreads();
    if (p == 0 && c < n) {
        float t = ws[0][lane];
#pragma unroll
        for (int q = 1; q < 8; q++) t += ws[q][lane];
        part[(size_t)blockIdx.y * n + c] = t;
    }
}
__global__ void k_colsum_final(const float* __restrict__ part, int nparts, int n, float* __restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    float t = 0.0f;
    for (int y = 0; y < nparts; y++) t += part[(size_t)y * n + c];
    out[c] = t;
}

// BF16 copy of FP32 values.
__global__ void k_f32_to_bf16(const float* __restrict__ w, __nv_bfloat16* __restrict__ wb, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) wb[i] = __float2bfloat16_rn(w[i]);
}

// Adam on FP32 master weights, refreshing their BF16 copy. The step's learning
// rate and bias corrections come from sched[3 s .. 3 s + 2], s = *step (the
// training loop's device step counter, so that one captured step replays).
__global__ void k_adam(float* __restrict__ w, __nv_bfloat16* __restrict__ wb, const float* __restrict__ g,
                       float* __restrict__ m1, float* __restrict__ m2, size_t n, const float* __restrict__ sched,
                       const uint32_t* __restrict__ step, float b1, float b2, float eps) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* sc = sched + 3 * (size_t)*step;
    const float lr = sc[0], c1 = sc[1], c2 = sc[2];
    const float gi = g[i];
    const float a = b1 * m1[i] + (1.0f - b1) * gi;
    const float b = b2 * m2[i] + (1.0f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = b;
    const float v = w[i] - lr * (a / c1) / (sqrtf(b / c2) + eps);
    w[i] = v;
    if (wb) wb[i] = __float2bfloat16_rn(v);
}

// One training step's rows and group targets: rows brows[(step % per_upload) B ..)
// of the uploaded block into cur_rows, their label's group into tgt.
__global__ void k_step_rows(const uint32_t* __restrict__ brows, const uint32_t* __restrict__ step, uint32_t per_upload,
                            int B, const uint32_t* __restrict__ labels, const uint32_t* __restrict__ group_of,
                            uint32_t* __restrict__ cur_rows, uint32_t* __restrict__ tgt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B) return;
    const uint32_t r = brows[(size_t)(*step % per_upload) * B + i];
    cur_rows[i] = r;
    tgt[i] = group_of[labels[r]];
}

// End of a training step: its loss into losses[step], the accumulator cleared,
// the step counter advanced (one thread).
__global__ void k_step_end(uint32_t* __restrict__ step, float* __restrict__ loss_acc, float* __restrict__ losses) {
    losses[*step] = *loss_acc;
    *loss_acc = 0.0f;
    *step += 1;
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
