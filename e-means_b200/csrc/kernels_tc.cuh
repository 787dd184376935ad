// tcgen05 fused assign: BF16 operands on the 5th-generation tensor cores with
// FP32 accumulators in TMEM, a per-row running top-2 in the epilogue, so no
// m x k score matrix reaches HBM.
//
// One CTA owns 128 rows (one TMEM lane per row) and walks its share of the
// centroid tiles (128 centroids each):
//   warp 0      TMA producer: centroid tiles (BF16 hi and lo parts, 128B swizzle)
//               into a 2-stage shared-memory ring
//   warp 1      allocates TMEM, issues tcgen05.mma (one thread), commits to mbarriers
//   warps 2..5  epilogue: tcgen05.ld of a 128 x 128 FP32 accumulator, score =
//               norm - 2 acc, running top-2 per row; two accumulators in TMEM so
//               the epilogue of tile t overlaps the MMAs of tile t+1
// The row tile is converted once per CTA (f32 -> BF16 hi + lo) by all threads
// and stays resident in shared memory for the whole centroid walk.
//
// Three-term products (hi*hi + hi*lo + lo*hi, FP32 accumulation) give scores
// within ~3 2^-18 |x||c| of exact, which certifies nearly every row's top-2; the
// exact re-score happens in kernels_exact.cuh.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>

#include "common.cuh"

namespace emb {

constexpr int kTcBM = 128;       // rows per CTA (TMEM lanes)
constexpr int kTcBN = 128;       // centroids per tile (accumulator columns)
constexpr int kTcStages = 2;     // centroid-tile ring depth
constexpr int kTcThreads = 192;  // 6 warps
constexpr int kTcTmemCols = 256; // two 128-column accumulators

struct TcParams {
    int m, d, k, kpad;   // kpad: d rounded up to 64 (one 128-byte swizzle atom per 64 BF16)
    int nterms;          // 1: hi*hi; 2: hi*hi + hi*lo (integer rows); 3: + lo*hi
    const uint32_t* gather;
    const float* norms;
    float* part_s;
    uint32_t* part_i;
    int* err;            // set to 1 if a wait gave up (results then re-searched exactly)
    int xvec;            // rows are 16-byte aligned f32 with d % 4 == 0: vector loads
};

// ---- PTX wrappers -----------------------------------------------------------
EMB_DEV uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

EMB_DEV void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
EMB_DEV void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
EMB_DEV void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
EMB_DEV bool mbar_try(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
EMB_DEV uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
constexpr uint64_t kWaitLimitNs = 4000000000ull;  // a healthy wait takes microseconds

// Bounded wait: returns false (and raises the abort flag) if the phase does not
// complete within kWaitLimitNs, or if another role already aborted.
EMB_DEV bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag) {
    if (mbar_try(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t i = 1;; i++) {
        if (mbar_try(bar, parity)) return true;
        if ((i & 63) == 0) {
            if (*abort_flag) return false;
            if (global_ns() - t0 > kWaitLimitNs) {
                *abort_flag = 1;
                return false;
            }
        }
    }
}

EMB_DEV void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
        ::"r"(smem_u32(dst)), "l"((uint64_t)map), "r"(smem_u32(bar)), "r"(c0), "r"(c1)
        : "memory");
}

EMB_DEV void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
EMB_DEV void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}
EMB_DEV void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
EMB_DEV void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups 1024 B apart.
EMB_DEV uint64_t sw128_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);        // start address
    d |= (uint64_t)1 << 16;                         // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(1024 >> 4) << 32;               // stride byte offset: 8 rows x 128 B
    d |= (uint64_t)1 << 46;                         // descriptor version (sm_100)
    d |= (uint64_t)2 << 61;                         // SWIZZLE_128B
    return d;
}

// Instruction descriptor, kind::f16: BF16 x BF16 -> F32, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

EMB_DEV void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
        ::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}
EMB_DEV void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

#define EMB_TMEM_LD32(taddr, r)                                                                                  \
    asm volatile(                                                                                                \
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"        \
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"                              \
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),      \
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), \
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]),           \
          "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),           \
          "=r"(r[30]), "=r"(r[31])                                                                               \
        : "r"(taddr))

EMB_DEV void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Byte offset of 16-byte chunk `kc` (8 BF16 along K) of row r in a K-major,
// 128B-swizzled tile of `rows` rows: atoms of 64 BF16 (128 B per row), 16-byte
// chunks XOR-permuted by the row index mod 8 (the layout TMA SWIZZLE_128B writes).
EMB_DEV uint32_t sw128_offset(int r, int kc, int rows) {
    int atom = kc >> 3, c = kc & 7;
    return (uint32_t)(atom * rows * 128 + r * 128 + ((c ^ (r & 7)) << 4));
}

struct TcSmem {
    // Offsets (bytes) inside the dynamic shared memory block (1024-aligned base).
    uint32_t a_hi, a_lo, b0, stage_bytes, term_bytes, bars, total;
};

__host__ __device__ inline TcSmem tc_smem_layout(int kpad, int nterms) {
    TcSmem s;
    uint32_t a_bytes = (uint32_t)kTcBM * kpad * 2;
    uint32_t b_term = (uint32_t)kTcBN * kpad * 2;
    int bterms = nterms == 1 ? 1 : 2;
    s.a_hi = 0;
    s.a_lo = a_bytes;
    uint32_t a_total = nterms == 3 ? 2 * a_bytes : a_bytes;
    s.b0 = a_total;
    s.term_bytes = b_term;
    s.stage_bytes = b_term * bterms;
    s.bars = s.b0 + kTcStages * s.stage_bytes;
    s.total = s.bars + 256;
    return s;
}

template <typename T>
EMB_DEV void tc_load_rows(uint8_t* smem, const TcSmem& L, const T* __restrict__ x, const TcParams& p, int row0) {
    // 128 rows x (kpad / 8) chunks of 8 elements; each thread converts chunks.
    const int nchunk = p.kpad / 8;
    const int total = kTcBM * nchunk;
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
        int r = t / nchunk, kc = t % nchunk;
        int g = row0 + r;
        float v[8];
        if (g < p.m) {
            size_t src = p.gather ? p.gather[g] : (size_t)g;
            const T* xr = x + src * (size_t)p.d;
            int k0 = kc * 8;
            if (sizeof(T) == 4 && p.xvec && k0 + 8 <= p.d) {
                float4 a = *reinterpret_cast<const float4*>(xr + k0);
                float4 b = *reinterpret_cast<const float4*>(xr + k0 + 4);
                v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
            } else {
#pragma unroll
                for (int i = 0; i < 8; i++) v[i] = (k0 + i < p.d) ? to_f32(xr[k0 + i]) : 0.0f;
            }
        } else {
#pragma unroll
            for (int i = 0; i < 8; i++) v[i] = 0.0f;
        }
        uint32_t hw[4], lw[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            __nv_bfloat16 h0 = __float2bfloat16_rn(v[2 * i]), h1 = __float2bfloat16_rn(v[2 * i + 1]);
            __nv_bfloat16 l0 = __float2bfloat16_rn(v[2 * i] - __bfloat162float(h0));
            __nv_bfloat16 l1 = __float2bfloat16_rn(v[2 * i + 1] - __bfloat162float(h1));
            hw[i] = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
            lw[i] = (uint32_t)__bfloat16_as_ushort(l0) | ((uint32_t)__bfloat16_as_ushort(l1) << 16);
        }
        uint32_t off = sw128_offset(r, kc, kTcBM);
        *reinterpret_cast<uint4*>(smem + L.a_hi + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
        if (p.nterms == 3) *reinterpret_cast<uint4*>(smem + L.a_lo + off) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
    }
}

// Grid: (ceil(m / 128), nsplit); CTA (bx, by) walks centroid tiles by, by + nsplit, ...
template <typename T>
__global__ void __launch_bounds__(kTcThreads, 1)
k_assign_tc(const T* __restrict__ x, const __grid_constant__ CUtensorMap map_hi,
            const __grid_constant__ CUtensorMap map_lo, const TcParams p) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const TcSmem L = tc_smem_layout(p.kpad, p.nterms);
    uint64_t* full = (uint64_t*)(smem + L.bars);         // [kTcStages]
    uint64_t* empty = full + kTcStages;                  // [kTcStages]
    uint64_t* acc_full = empty + kTcStages;              // [2]
    uint64_t* acc_empty = acc_full + 2;                  // [2]
    uint32_t* tmem_slot = (uint32_t*)(acc_empty + 2);
    volatile int* abort_flag = (volatile int*)(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int row0 = blockIdx.x * kTcBM;
    const int nsplit = gridDim.y;
    const int ntiles_all = (p.k + kTcBN - 1) / kTcBN;
    const int my_tiles = blockIdx.y < ntiles_all ? (ntiles_all - blockIdx.y + nsplit - 1) / nsplit : 0;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kTcStages; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], 4);  // one arrival per epilogue warp
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) tmem_alloc(tmem_slot, kTcTmemCols);
    tc_load_rows(smem, L, x, p, row0);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            // ---- TMA producer
            int issued = 0;
            for (int t = 0; t < my_tiles; t++) {
                int s = t % kTcStages;
                uint32_t ph = (uint32_t)(t / kTcStages) & 1u;
                if (!mbar_wait(&empty[s], ph ^ 1u, abort_flag)) break;
                int tile = blockIdx.y + t * nsplit;
                uint8_t* stage = smem + L.b0 + s * L.stage_bytes;
                mbar_expect_tx(&full[s], L.stage_bytes);
                for (int a = 0; a < p.kpad / 64; a++) {
                    tma_load_2d(stage + a * (kTcBN * 128), &map_hi, &full[s], a * 64, tile * kTcBN);
                    if (p.nterms > 1)
                        tma_load_2d(stage + L.term_bytes + a * (kTcBN * 128), &map_lo, &full[s], a * 64, tile * kTcBN);
                }
                issued = t + 1;
            }
            // After an abort, let the copies still in flight (the last stages
            // issued) land before the CTA exits; bounded like every wait.
            if (*abort_flag) {
                for (int t = issued > kTcStages ? issued - kTcStages : 0; t < issued; t++) {
                    int s = t % kTcStages;
                    uint32_t ph = (uint32_t)(t / kTcStages) & 1u;
                    const uint64_t t0 = global_ns();
                    while (!mbar_try(&full[s], ph) && global_ns() - t0 < kWaitLimitNs) {
                    }
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // ---- MMA issuer
            const uint32_t idesc = idesc_bf16(kTcBM, kTcBN);
            const uint32_t a_hi = smem_u32(smem + L.a_hi), a_lo = smem_u32(smem + L.a_lo);
            const int ksteps = p.kpad / 16;
            for (int t = 0; t < my_tiles; t++) {
                int s = t % kTcStages;
                uint32_t ph = (uint32_t)(t / kTcStages) & 1u;
                int b = t & 1;
                uint32_t bph = (uint32_t)(t >> 1) & 1u;
                if (!mbar_wait(&acc_empty[b], bph ^ 1u, abort_flag)) break;
                if (!mbar_wait(&full[s], ph, abort_flag)) break;
                tc_fence_after();
                const uint32_t d_tmem = tmem_base + (uint32_t)(b * kTcBN);
                const uint32_t b_hi = smem_u32(smem + L.b0 + s * L.stage_bytes);
                const uint32_t b_lo = b_hi + L.term_bytes;
                uint32_t acc = 0;
                for (int term = 0; term < p.nterms; term++) {
                    uint32_t abase = term == 2 ? a_lo : a_hi;
                    uint32_t bbase = term == 1 ? b_lo : b_hi;
                    for (int kk = 0; kk < ksteps; kk++) {
                        uint32_t koff = (uint32_t)((kk >> 2) * (kTcBM * 128) + (kk & 3) * 32);
                        uint32_t kofb = (uint32_t)((kk >> 2) * (kTcBN * 128) + (kk & 3) * 32);
                        mma_bf16(d_tmem, sw128_desc(abase + koff), sw128_desc(bbase + kofb), idesc, acc);
                        acc = 1;
                    }
                }
                mma_commit(&empty[s]);
                mma_commit(&acc_full[b]);
            }
        }
    } else {
        // ---- epilogue: warps 2..5, thread = row (TMEM lane)
        const int q = warp & 3;  // TMEM lane quarter this warp may access
        const int r = q * 32 + lane;
        Top2 top;
        top.init();
        for (int t = 0; t < my_tiles; t++) {
            int b = t & 1;
            uint32_t bph = (uint32_t)(t >> 1) & 1u;
            if (!mbar_wait(&acc_full[b], bph, abort_flag)) break;
            tc_fence_after();
            const int col0 = (blockIdx.y + t * nsplit) * kTcBN;
            const uint32_t taddr = tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * kTcBN);
#pragma unroll 1
            for (int ch = 0; ch < kTcBN / 32; ch++) {
                uint32_t v[32];
                EMB_TMEM_LD32(taddr + ch * 32, v);
                tmem_wait_ld();
                const int cbase = col0 + ch * 32;
                if (cbase + 32 <= p.k) {
#pragma unroll
                    for (int j = 0; j < 32; j++) {
                        float s = __fmaf_rn(-2.0f, __uint_as_float(v[j]), __ldg(&p.norms[cbase + j]));
                        if (s < top.s2) top.push(s, (uint32_t)(cbase + j));
                    }
                } else {
#pragma unroll
                    for (int j = 0; j < 32; j++) {
                        if (cbase + j < p.k) {
                            float s = __fmaf_rn(-2.0f, __uint_as_float(v[j]), __ldg(&p.norms[cbase + j]));
                            if (s < top.s2) top.push(s, (uint32_t)(cbase + j));
                        }
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acc_empty[b]);
        }
        const int row = row0 + r;
        if (row < p.m) {
            size_t o = ((size_t)blockIdx.y * p.m + row) * 2;
            p.part_s[o] = top.s1;
            p.part_i[o] = top.i1;
            p.part_s[o + 1] = top.s2;
            p.part_i[o + 1] = top.i2;
        }
    }
    tc_fence_before();
    __syncthreads();
    if (*abort_flag && threadIdx.x == 0) atomicExch(p.err, 1);
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem_base, kTcTmemCols);
    }
}

}  // namespace emb
