// tcgen05 GEMM of the proposer's network training: C[M x N] = A[M x K] . B[N x K]^T
// with BF16 operands stored K-major (row-major, K contiguous; row strides a
// multiple of 8 elements, 16-byte aligned bases) and FP32 accumulation in TMEM.
//
// One CTA per 128 x 128 output tile and K range (grid (ceil(N/128), ceil(M/128),
// splits)):
//   warp 0      TMA producer: per stage one K atom (64 BF16, 128-byte swizzle) of
//               the 128-row A tile and of the 128-row B tile; a 4-stage ring
//   warp 1      TMEM allocation (128 columns); tcgen05.mma kind::f16 M=128 N=128
//               K=16 from one thread, committing stages and the accumulator
//   warps 2-5   epilogue: each reads its TMEM lane quarter (32 rows) 32 columns at
//               a time and applies the fused epilogue (bias, ReLU, BF16 or FP32
//               store); with several K splits it writes FP32 partials that
//               k_gemm_tc_reduce adds in split order (deterministic)
// Rows past M and columns past N read as zeros (TMA fill) and are not stored.
// Every wait is bounded; a timeout raises *err, and the host reports the call
// as failed.
#pragma once
#include "kernels_mlp.cuh"
#include "kernels_tc.cuh"

namespace emb {

constexpr int kGtBM = 128, kGtBN = 128, kGtStages = 4, kGtThreads = 192;

// Two FP32 values as round-to-nearest BF16 in one word (the lower column in the low half).
EMB_DEV uint32_t pack_bf16x2(float lo, float hi) {
    return (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(lo)) |
           ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(hi)) << 16);
}
constexpr uint32_t kGtAtomBytes = 128 * 128;                  // 128 rows x one 128-byte K atom
constexpr uint32_t kGtStageBytes = 2 * kGtAtomBytes;          // A and B atoms
constexpr size_t kGtSmemBytes = kGtStages * kGtStageBytes + 256 + 1024;

template <int EPI>
__global__ void __launch_bounds__(kGtThreads, 1)
k_gemm_tc(int M, int N, int K, int kc, const __grid_constant__ CUtensorMap map_a,
          const __grid_constant__ CUtensorMap map_b, void* __restrict__ C, size_t ldc, const float* __restrict__ bias,
          float* __restrict__ part, int* __restrict__ err) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = smem_align1024(smem_raw);
    uint64_t* full = (uint64_t*)(smem + kGtStages * kGtStageBytes);  // [kGtStages]
    uint64_t* empty = full + kGtStages;                              // [kGtStages]
    uint64_t* acc_full = empty + kGtStages;
    uint64_t* mma_done = acc_full + 1;
    uint32_t* tmem_slot = (uint32_t*)(mma_done + 1);
    volatile int* abort_flag = (volatile int*)(tmem_slot + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n0 = blockIdx.x * kGtBN, m0 = blockIdx.y * kGtBM;
    const int kb = (int)blockIdx.z * kc, ke = min(K, kb + kc);
    const int natoms = ke > kb ? (ke - kb + 63) / 64 : 0;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kGtStages; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(acc_full, 1);
        mbar_init(mma_done, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) tmem_alloc(tmem_slot, 128);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            int issued = 0;
            for (int a = 0; a < natoms; a++) {
                const int s = a % kGtStages;
                if (a >= kGtStages && !mbar_wait(&empty[s], ((uint32_t)(a / kGtStages) & 1u) ^ 1u, abort_flag)) break;
                uint8_t* st = smem + s * kGtStageBytes;
                mbar_expect_tx(&full[s], kGtStageBytes);
                tma_load_2d(st, &map_a, &full[s], kb + a * 64, m0);
                tma_load_2d(st + kGtAtomBytes, &map_b, &full[s], kb + a * 64, n0);
                issued = a + 1;
            }
            if (*abort_flag)
                for (int a = issued > kGtStages ? issued - kGtStages : 0; a < issued; a++)
                    mbar_drain(&full[a % kGtStages], (uint32_t)(a / kGtStages) & 1u);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = idesc_bf16(kGtBM, kGtBN);
            bool ok = true;
            for (int a = 0; a < natoms; a++) {
                const int s = a % kGtStages;
                if (!mbar_wait(&full[s], (uint32_t)(a / kGtStages) & 1u, abort_flag)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint64_t ad = sw128_desc(smem_u32(smem + s * kGtStageBytes));
                const uint64_t bd = sw128_desc(smem_u32(smem + s * kGtStageBytes + kGtAtomBytes));
#pragma unroll
                for (int kk = 0; kk < 4; kk++) mma_bf16(tmem_base, ad + 2 * kk, bd + 2 * kk, idesc, (a > 0 || kk > 0) ? 1u : 0u);
                mma_commit(&empty[s]);
            }
            if (ok) mma_commit(acc_full);
            mma_drain(mma_done);
        }
    } else {
        // ---- epilogue: warps 2..5, TMEM lane quarter warp & 3
        const int q = warp & 3;
        const int row = m0 + q * 32 + lane;
        // warp-uniform: every lane then takes part in the .sync.aligned TMEM loads
        const bool have = __all_sync(0xffffffffu, natoms > 0 && mbar_wait(acc_full, 0, abort_flag, 2000));
        tc_fence_after();
#pragma unroll 1
        for (int ch = 0; ch < kGtBN / 32; ch++) {
            uint32_t v[32];
            if (have) {
                EMB_TMEM_LD32(tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(ch * 32), v);
                tmem_wait_ld();
                tc_regs_ready(v);
            } else {
#pragma unroll
                for (int j = 0; j < 32; j++) v[j] = 0u;  // an empty K range contributes zeros
            }
            if (row >= M || *abort_flag) continue;
            const int c0 = n0 + ch * 32;
            // The lane's 32 consecutive columns of its row: 16-byte stores when the
            // whole chunk is inside the matrix and the row is 16-byte aligned.
            float o[32];
#pragma unroll
            for (int j = 0; j < 32; j++) {
                float x = __uint_as_float(v[j]);
                if (!part && (EPI == kEpiBiasF32 || EPI == kEpiBiasBf16 || EPI == kEpiBiasReluBf16))
                    x += c0 + j < N ? bias[c0 + j] : 0.0f;
                if (!part && EPI == kEpiBiasReluBf16) x = fmaxf(x, 0.0f);
                o[j] = x;
            }
            const bool f32out = part || EPI == kEpiF32 || EPI == kEpiBiasF32;
            void* dst = part ? (void*)(part + ((size_t)blockIdx.z * M + row) * N + c0)
                             : (f32out ? (void*)((float*)C + (size_t)row * ldc + c0)
                                       : (void*)((__nv_bfloat16*)C + (size_t)row * ldc + c0));
            if (c0 + 32 <= N && ((uintptr_t)dst & 15) == 0) {
                if (f32out) {
#pragma unroll
                    for (int j = 0; j < 32; j += 4)
                        reinterpret_cast<float4*>(dst)[j / 4] = make_float4(o[j], o[j + 1], o[j + 2], o[j + 3]);
                } else {
#pragma unroll
                    for (int j = 0; j < 32; j += 8) {
                        uint4 w;
                        w.x = pack_bf16x2(o[j], o[j + 1]);
                        w.y = pack_bf16x2(o[j + 2], o[j + 3]);
                        w.z = pack_bf16x2(o[j + 4], o[j + 5]);
                        w.w = pack_bf16x2(o[j + 6], o[j + 7]);
                        reinterpret_cast<uint4*>(dst)[j / 8] = w;
                    }
                }
            } else {
#pragma unroll
                for (int j = 0; j < 32; j++) {
                    if (c0 + j >= N) break;
                    if (f32out) ((float*)dst)[j] = o[j];
                    else ((__nv_bfloat16*)dst)[j] = __float2bfloat16_rn(o[j]);
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (*abort_flag && threadIdx.x == 0) atomicExch(err, 1);
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem_base, 128);
    }
}

// C[M x N] (FP32, row stride ldc) = sum over the S partials [s][M][N] in split order.
__global__ void k_gemm_tc_reduce(const float* __restrict__ part, int S, int M, int N, float* __restrict__ C,
                                 size_t ldc) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (size_t)M * N) return;
    const size_t r = e / N, c = e - r * N;
    float s = part[e];
    for (int z = 1; z < S; z++) s += part[(size_t)z * M * N + e];
    C[r * ldc + c] = s;
}

// dst[C][R] = src[R][C] (BF16, row strides ld_src, ld_dst), through 32 x 32 shared tiles.
__global__ void k_transpose_bf16(const __nv_bfloat16* __restrict__ src, size_t ld_src, int R, int Cn,
                                 __nv_bfloat16* __restrict__ dst, size_t ld_dst) {
    __shared__ __nv_bfloat16 t[32][33];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int r = r0 + i, c = c0 + threadIdx.x;
        t[i][threadIdx.x] = (r < R && c < Cn) ? src[(size_t)r * ld_src + c] : __float2bfloat16(0.0f);
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int c = c0 + i, r = r0 + threadIdx.x;
        if (c < Cn && r < R) dst[(size_t)c * ld_dst + r] = t[threadIdx.x][i];
    }
}

}  // namespace emb
