// tcgen05 BF16 throughput microbenchmark: back-to-back kind::f16 MMAs of the
// search kernel's shapes on operands resident in shared memory (no TMA, no
// epilogue), the ceiling of the MMA issue path that k_assign_tc builds on.
//   PAIR = false: one CTA per SM, tcgen05.mma.cta_group::1 M=128 N=256 K=16
//   PAIR = true:  clusters of two CTAs, tcgen05.mma.cta_group::2 M=256 N=256
//                 K=16 issued by the even CTA: each CTA holds its 128 rows of A
//                 and half (128 rows) of B; each CTA's TMEM its 128 rows of D
// Two accumulators alternate (512 TMEM columns). The operands are zeros.
#pragma once
#include "kernels_tc.cuh"

namespace emb {

constexpr uint32_t kPeakABytes = 128 * 128;  // 128 rows x one 128-byte K atom
constexpr uint32_t kPeakBBytes = 256 * 128;  // up to 256 rows x one K atom
// More shared memory than two CTAs fit in, so that each SM holds one CTA (one
// 512-column TMEM allocation).
constexpr size_t kPeakSmem = 120 * 1024;

EMB_DEV uint32_t cluster_ctarank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
EMB_DEV void cluster_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\nbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

template <bool PAIR>
__global__ void __launch_bounds__(128, 1) k_mma_peak(int iters, int* __restrict__ err) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = smem_align1024(smem_raw);
    uint8_t* a = smem;
    uint8_t* b = smem + kPeakABytes;
    uint64_t* done = (uint64_t*)(smem + kPeakABytes + kPeakBBytes);
    uint32_t* slot = (uint32_t*)(done + 1);
    volatile int* abort_flag = (volatile int*)(slot + 1);
    const int warp = threadIdx.x >> 5;
    const uint32_t rank = PAIR ? cluster_ctarank() : 0u;
    for (uint32_t i = threadIdx.x; i < (kPeakABytes + kPeakBBytes) / 16; i += blockDim.x)
        reinterpret_cast<uint4*>(smem)[i] = make_uint4(0, 0, 0, 0);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (threadIdx.x == 0) {
        mbar_init(done, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        if (PAIR) {
            asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                         "r"(512));
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
        } else {
            tmem_alloc(slot, 512);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (PAIR) cluster_sync();  // both CTAs' operands, barriers and TMEM are ready
    tc_fence_after();
    const uint32_t tmem = *slot;
    if (threadIdx.x == 32 && rank == 0) {
        const uint32_t idesc = idesc_bf16(PAIR ? 256 : 128, 256);
        const uint64_t ad = sw128_desc(smem_u32(a)), bd = sw128_desc(smem_u32(b));
        for (int it = 0; it < iters; it++) {
            const uint32_t d = tmem + (uint32_t)((it & 1) * 256);
#pragma unroll
            for (int kk = 0; kk < 4; kk++) {
                const uint32_t acc = (it >= 2 || kk > 0) ? 1u : 0u;
                if (PAIR)
                    asm volatile(
                        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                        " tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
                        "l"(ad + 2 * kk), "l"(bd + 2 * kk), "r"(idesc), "r"(acc));
                else
                    mma_bf16(d, ad + 2 * kk, bd + 2 * kk, idesc, acc);
            }
        }
        if (PAIR)
            asm volatile(
                "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
                    smem_u32(done)),
                "h"((uint16_t)3)
                : "memory");
        else
            mma_commit(done);
    }
    if (threadIdx.x == 32) {
        // every MMA has completed (this CTA's TMEM written) before TMEM is freed
        if (!mbar_wait(done, 0, abort_flag, 1000, kWaitLimitNs)) atomicExch(err, 1);
    }
    tc_fence_before();
    __syncthreads();
    if (PAIR) cluster_sync();
    tc_fence_after();
    if (warp == 0) {
        if (PAIR)
            asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
        else
            tmem_dealloc(tmem, 512);
    }
}

}  // namespace emb
