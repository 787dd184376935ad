// tcgen05 kind::i8 search for i8 rows with i8 centroids: the semantics of
// CpuI8Assigner(CentroidBits::I8) (src/cpu_i8.rs:72-191) on the tensor cores.
// s8 x s8 products accumulate exactly in s32 TMEM, so the argmin is exact and
// needs no certification.
//
// Same CTA organisation as k_assign_tc (kernels_tc.cuh): 128 rows per CTA, the
// row tile resident in shared memory (raw i8, 128B-swizzled), centroid tiles of
// 256 streamed by TMA one 128-byte K atom per stage, MMA M=128 N=256 K=32 from
// one thread into two 256-column s32 accumulators, 16 epilogue warps.
//
// Epilogue: the score s_j = off_j - 2 acc_j (off_j = sum c8^2 + bias) is folded
// into one integer key per column, key = -64 acc_j + P_j with
// P_j = 32 off_j + (j mod 32) + 2^30, i.e. key = 32 s_j + (j mod 32) + 2^30:
// one IMAD per score, ordered by (score, column), non-negative and below
// 0x7f800000 for |off| <= 2^23 and d <= 512, so 3-input float min on the bit
// patterns orders them like the integers. The host only selects this kernel
// when those bounds hold.
#pragma once
#include "kernels_tc.cuh"

namespace emb {

constexpr int kI8KeyBias = 1 << 30;

struct TcI8Params {
    int m, d, k, kpad;         // kpad: d rounded up to 128 (one 128-byte swizzle atom)
    const uint32_t* gather;
    const int* pkeys;          // P_j, padded to whole tiles with 0x7f000000
    long long* part_s;         // [split][row] exact score
    uint32_t* part_i;          // [split][row] label
    int* err;
    int stall_tile;            // abort-path test, as TcParams::stall_tile
    uint64_t stall_ns;
};

__host__ __device__ inline TcSmem tc_i8_smem_layout(int kpad) {
    TcSmem s;
    const uint32_t a_bytes = (uint32_t)kTcBM * kpad;
    s.a_hi = 0;
    s.a_lo = 0;
    s.b0 = a_bytes;
    s.term_bytes = (uint32_t)kTcBN * 128;
    s.stage_bytes = s.term_bytes;
    const uint32_t fixed = kTcNormSlots * kTcBN * 4 + 3 * kTcBM * 16 + 256 + 1024;
    int st = 0;
    while (st < kTcMaxStages && a_bytes + (st + 1) * s.stage_bytes + fixed <= (uint32_t)kTcSmemLimit) st++;
    s.stages = st;
    s.norms = s.b0 + st * s.stage_bytes;
    s.merge = s.norms + kTcNormSlots * kTcBN * 4;
    s.bars = s.merge + 3 * kTcBM * 16;
    s.total = s.bars + 256;
    return s;
}

// Instruction descriptor, kind::i8: S8 x S8 -> S32, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_s8(int M, int N) {
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

EMB_DEV void mma_s8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n"
        ::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// Grid: (ceil(m / 128), nsplit); CTA (bx, by) walks centroid tiles by, by + nsplit, ...
__global__ void __launch_bounds__(kTcThreads, 1)
k_assign_tc_i8(const int8_t* __restrict__ x, const __grid_constant__ CUtensorMap map_c8, const TcI8Params p) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = smem_align1024(smem_raw);
    const TcSmem L = tc_i8_smem_layout(p.kpad);
    const int S = L.stages;
    uint64_t* full = (uint64_t*)(smem + L.bars);
    uint64_t* empty = full + kTcMaxStages;
    uint64_t* acc_full = empty + kTcMaxStages;
    uint64_t* acc_empty = acc_full + 2;
    uint64_t* keys_full = acc_empty + 2;
    uint64_t* mma_done = keys_full + kTcNormSlots;  // every issued MMA completed (teardown)
    uint64_t* stall_bar = mma_done + 1;             // never completed (abort-path test)
    uint32_t* tmem_slot = (uint32_t*)(stall_bar + 1);
    volatile int* abort_flag = (volatile int*)(tmem_slot + 1);
    int* keys_s = (int*)(smem + L.norms);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int row0 = blockIdx.x * kTcBM;
    const int nsplit = gridDim.y;
    const int ntiles_all = (p.k + kTcBN - 1) / kTcBN;
    const int my_tiles = (int)blockIdx.y < ntiles_all ? (ntiles_all - (int)blockIdx.y + nsplit - 1) / nsplit : 0;
    const int natoms = p.kpad / 128;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kTcMaxStages; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], kTcEpiWarps);
        }
        for (int i = 0; i < kTcNormSlots; i++) mbar_init(&keys_full[i], 1);
        mbar_init(mma_done, 1);
        mbar_init(stall_bar, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) tmem_alloc(tmem_slot, kTcTmemCols);
    // Row tile: raw i8 copied into the 128B-swizzled K-major layout (16-byte chunks).
    {
        const int nchunk = p.kpad / 16;
        for (int t = threadIdx.x; t < kTcBM * nchunk; t += blockDim.x) {
            const int r = t / nchunk, kc = t % nchunk;
            const int g = row0 + r;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (g < p.m) {
                const size_t src = p.gather ? p.gather[g] : (size_t)g;
                const int8_t* xr = x + src * (size_t)p.d + kc * 16;
                if (kc * 16 + 16 <= p.d && ((uintptr_t)xr & 15) == 0) {
                    v = *reinterpret_cast<const uint4*>(xr);
                } else {
                    uint32_t w[4] = {0, 0, 0, 0};
                    for (int b = 0; b < 16; b++)
                        if (kc * 16 + b < p.d) w[b >> 2] |= (uint32_t)(uint8_t)xr[b] << (8 * (b & 3));
                    v = make_uint4(w[0], w[1], w[2], w[3]);
                }
            }
            *reinterpret_cast<uint4*>(smem + sw128_offset(r, kc, kTcBM)) = v;
        }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            const int nunits = my_tiles * natoms;
            int issued = 0;
            for (int u = 0; u < nunits; u++) {
                const int t = u / natoms, a = u - t * natoms;
                const int s = u % S;
                const uint32_t ph = (uint32_t)(u / S) & 1u;
                if (!mbar_wait(&empty[s], ph ^ 1u, abort_flag)) break;
                const int tile = blockIdx.y + t * nsplit;
                mbar_expect_tx(&full[s], L.stage_bytes);
                tma_load_2d(smem + L.b0 + s * L.stage_bytes, &map_c8, &full[s], a * 128, tile * kTcBN);
                if (a == 0) {
                    const int ns = t % kTcNormSlots;
                    mbar_expect_tx(&keys_full[ns], kTcBN * 4);
                    bulk_load(keys_s + ns * kTcBN, p.pkeys + (size_t)tile * kTcBN, kTcBN * 4, &keys_full[ns]);
                }
                issued = u + 1;
            }
            if (*abort_flag) {
                for (int u = issued > S ? issued - S : 0; u < issued; u++) mbar_drain(&full[u % S], (uint32_t)(u / S) & 1u);
                const int tl = issued > 0 ? (issued - 1) / natoms : -1;
                for (int t = tl >= kTcNormSlots ? tl - kTcNormSlots + 1 : 0; t <= tl; t++)
                    mbar_drain(&keys_full[t % kTcNormSlots], (uint32_t)(t / kTcNormSlots) & 1u);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = idesc_s8(kTcBM, kTcBN);
            const uint64_t a0 = sw128_desc(smem_u32(smem));
            const uint32_t a_atom = (kTcBM * 128) >> 4;
            bool ok = true;
            int u = 0;
            for (int t = 0; t < my_tiles && ok; t++) {
                const int b = t & 1;
                const uint32_t bph = (uint32_t)(t >> 1) & 1u;
                if (!mbar_wait(&acc_empty[b], bph ^ 1u, abort_flag)) break;
                tc_fence_after();
                const uint32_t d_tmem = tmem_base + (uint32_t)(b * kTcBN);
                for (int a = 0; a < natoms; a++, u++) {
                    const int s = u % S;
                    const uint32_t ph = (uint32_t)(u / S) & 1u;
                    if (!mbar_wait(&full[s], ph, abort_flag)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint64_t bd = sw128_desc(smem_u32(smem + L.b0 + s * L.stage_bytes));
                    const uint64_t ad = a0 + (uint64_t)(a * a_atom);
#pragma unroll
                    for (int kk = 0; kk < 4; kk++)  // 32 bytes of K per step = 2 descriptor units
                        mma_s8(d_tmem, ad + 2 * kk, bd + 2 * kk, idesc, (a > 0 || kk > 0) ? 1u : 0u);
                    mma_commit(&empty[s]);
                }
                if (ok) mma_commit(&acc_full[b]);
            }
            mma_drain(mma_done);  // no MMA may outlive the TMEM allocation (see k_assign_tc)
        }
    } else {
        const int q = warp & 3;
        const int cq = (warp - 2) >> 2;
        const int r = q * 32 + lane;
        const int row = row0 + r;
        int best = 0x7fffffff;  // best key so far
        int bbase = 0;          // column of the best key's chunk
        for (int t = 0; t < my_tiles; t++) {
            const int b = t & 1;
            const uint32_t bph = (uint32_t)(t >> 1) & 1u;
            if (!mbar_wait(&acc_full[b], bph, abort_flag, 20000)) break;
            if (!mbar_wait(&keys_full[t % kTcNormSlots], (uint32_t)(t / kTcNormSlots) & 1u, abort_flag)) break;
            if (p.stall_ns && t == p.stall_tile && warp == 2 && !mbar_wait(stall_bar, 0, abort_flag, 0, p.stall_ns)) break;
            tc_fence_after();
            const int cq0 = (blockIdx.y + t * nsplit) * kTcBN + cq * 64;
            const int* pk = keys_s + (t % kTcNormSlots) * kTcBN + cq * 64;
            const uint32_t taddr = tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * kTcBN + cq * 64);
#pragma unroll
            for (int ch = 0; ch < 2; ch++) {
                uint32_t v[32];
                EMB_TMEM_LD32(taddr + ch * 32, v);
                tmem_wait_ld();
                tc_regs_ready(v);
                if (ch == 1) {
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&acc_empty[b]);
                }
                float kf[32];
#pragma unroll
                for (int j = 0; j < 32; j += 4) {
                    const int4 p4 = *reinterpret_cast<const int4*>(pk + ch * 32 + j);
                    kf[j] = __int_as_float((int)v[j] * -64 + p4.x);
                    kf[j + 1] = __int_as_float((int)v[j + 1] * -64 + p4.y);
                    kf[j + 2] = __int_as_float((int)v[j + 2] * -64 + p4.z);
                    kf[j + 3] = __int_as_float((int)v[j + 3] * -64 + p4.w);
                }
                const int kc = __float_as_int(tc_min32(kf));
                // Strictly smaller score only: an equal score in a later chunk has a higher column.
                if ((kc >> 5) < (best >> 5)) {
                    best = kc;
                    bbase = cq0 + ch * 32;
                }
            }
        }
        // Merge the four column quarters: lowest (score, column).
        uint32_t* mg = (uint32_t*)(smem + L.merge);
        if (cq > 0) {
            uint32_t* e = mg + ((cq - 1) * kTcBM + r) * 4;
            e[0] = (uint32_t)best;
            e[1] = (uint32_t)bbase;
        }
        asm volatile("bar.sync 1, %0;" ::"n"(kTcEpiWarps * 32) : "memory");
        if (cq == 0 && row < p.m) {
            long long bs = (long long)((best - kI8KeyBias) >> 5);
            uint32_t bl = (uint32_t)(bbase + (best & 31));
            for (int o = 0; o < 3; o++) {
                const uint32_t* e = mg + (o * kTcBM + r) * 4;
                const int ob = (int)e[0];
                const long long os = (long long)((ob - kI8KeyBias) >> 5);
                const uint32_t ol = e[1] + (uint32_t)(ob & 31);
                if (ob != 0x7fffffff && (os < bs || (os == bs && ol < bl) || best == 0x7fffffff)) {
                    bs = os;
                    bl = ol;
                    best = ob;
                }
            }
            const size_t oo = (size_t)blockIdx.y * p.m + row;
            p.part_s[oo] = best == 0x7fffffff ? 0x7fffffffffffffffll : bs;
            p.part_i[oo] = best == 0x7fffffff ? 0u : bl;
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

// P_j = 32 off_j + (j mod 32) + 2^30 for real centroids, 0x7f000000 for padding.
__global__ void k_i8_keys(const long long* __restrict__ off, int k, int kp, int* __restrict__ pkeys) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= kp) return;
    pkeys[j] = j < k ? (int)(32 * off[j]) + (j & 31) + kI8KeyBias : 0x7f000000;
}

}  // namespace emb
