// Persistent grouped search: the tcgen05 contraction of k_assign_tc for the
// proposer's buckets, where every row tile (128 bucket positions of one
// centroid group) scores only its group's column tiles, usually one or two.
// A CTA per SM walks the bucket tiles blockIdx.x, + gridDim.x, ... and keeps
// its barriers, TMEM and centroid-stage pipeline across them:
//   warp 0       TMA producer: the stages of every column tile of every bucket
//                tile in order, plus the norms of each column tile
//   warp 1       TMEM allocation and the MMAs; before a bucket tile's first MMA
//                it waits until the epilogue warps have gathered its rows
//   warps 2..17  gather the first bucket tile's rows, then for each bucket tile:
//                once its last accumulator is full (every MMA reading its rows
//                has completed) they gather the next tile's rows, so the MMAs of
//                the next tile overlap the epilogue of this one; top-2 per row
//                as in k_assign_tc, merged across the four column quarters.
// Every bucket tile has at least one column tile (the host gives empty groups one).
#pragma once
#include "kernels_tc.cuh"

namespace emb {

// Ask L2 for the rows of a bucket tile ahead of their gather (prefetches are
// hints: nothing waits on them, and an address is never past its row's end).
template <typename T>
EMB_DEV void prefetch_rows_l2(const T* __restrict__ x, const TcParams& p, int row0, int tid, int nthr) {
    const int row_bytes = p.d * (int)sizeof(T);
    const int lines = row_bytes / 128 + 2;  // rows need not start on a 128-byte line
    for (int t = tid; t < kTcBM * lines; t += nthr) {
        const int r = t / lines, l = t - r * lines;
        const int g = row0 + r;
        if (g >= p.m) continue;
        const size_t src = p.gather ? (size_t)p.gather[g] : (size_t)g;
        const char* base = (const char*)(x + src * (size_t)p.d);
        const int off = l * 128 < row_bytes ? l * 128 : row_bytes - 1;
        asm volatile("prefetch.global.L2 [%0];" ::"l"(base + off));
    }
}

template <typename T>
__global__ void __launch_bounds__(kTcThreads, 1)
k_assign_grouped(const T* __restrict__ x, const __grid_constant__ CUtensorMap map_hi,
                 const __grid_constant__ CUtensorMap map_lo, const TcParams p) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const TcSmem L = tc_smem_layout(p.kpad, p.nterms);
    const int S = L.stages;
    uint64_t* full = (uint64_t*)(smem + L.bars);  // [kTcMaxStages]
    uint64_t* empty = full + kTcMaxStages;        // [kTcMaxStages]
    uint64_t* acc_full = empty + kTcMaxStages;    // [2]
    uint64_t* acc_empty = acc_full + 2;           // [2]
    uint64_t* norms_full = acc_empty + 2;         // [kTcNormSlots]
    uint64_t* a_full = norms_full + kTcNormSlots; // rows of the current bucket tile gathered
    uint32_t* tmem_slot = (uint32_t*)(a_full + 1);
    volatile int* abort_flag = (volatile int*)(tmem_slot + 1);
    float* norms_s = (float*)(smem + L.norms);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nwt = p.m / kTcBM;  // bucket tiles in the launch (m is a whole number of tiles)
    // Bucket tile of this CTA's i-th work item and its group (false past the last one).
    auto work = [&](int i, int& w, int& g) -> bool {
        w = (int)blockIdx.x + i * (int)gridDim.x;
        if (w >= nwt) return false;
        g = p.tile_group[w];
        return g >= 0;
    };
    int w0, g0;
    if (!work(0, w0, g0)) return;  // no work: the whole CTA leaves before any setup
    const int natoms = p.kpad / 64;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kTcMaxStages; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], kTcEpiWarps);
        }
        for (int i = 0; i < kTcNormSlots; i++) mbar_init(&norms_full[i], 1);
        mbar_init(a_full, kTcEpiWarps);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) tmem_alloc(tmem_slot, kTcTmemCols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            // ---- TMA producer
            int u = 0, tg = 0, norms_issued = 0, w, g;
            bool ok = true;
            for (int i = 0; ok && work(i, w, g); i++) {
                const int nt = p.grp_ntiles[g], c0 = p.grp_cbeg[g];
                for (int t = 0; ok && t < nt; t++, tg++) {
                    const int col = c0 + t * kTcBN;
                    for (int a = 0; a < natoms; a++, u++) {
                        const int s = u % S;
                        const uint32_t ph = (uint32_t)(u / S) & 1u;
                        if (!mbar_wait(&empty[s], ph ^ 1u, abort_flag)) {
                            ok = false;
                            break;
                        }
                        uint8_t* stage = smem + L.b0 + s * L.stage_bytes;
                        mbar_expect_tx(&full[s], L.stage_bytes);
                        tma_load_2d(stage, &map_hi, &full[s], a * 64, col);
                        if (p.nterms > 1) tma_load_2d(stage + L.term_bytes, &map_lo, &full[s], a * 64, col);
                        if (a == 0) {
                            const int ns = tg % kTcNormSlots;
                            mbar_expect_tx(&norms_full[ns], kTcBN * 4);
                            bulk_load(norms_s + ns * kTcBN, p.norms + (size_t)col, kTcBN * 4, &norms_full[ns]);
                            norms_issued = tg + 1;
                        }
                    }
                }
            }
            // After an abort, let the copies still in flight land before the CTA exits.
            if (*abort_flag) {
                const uint64_t t0 = global_ns();
                for (int v = u > S ? u - S : 0; v < u; v++) {
                    const uint32_t ph = (uint32_t)(v / S) & 1u;
                    while (!mbar_try(&full[v % S], ph) && global_ns() - t0 < kWaitLimitNs) {
                    }
                }
                for (int t = norms_issued > kTcNormSlots ? norms_issued - kTcNormSlots : 0; t < norms_issued; t++) {
                    const uint32_t nph = (uint32_t)(t / kTcNormSlots) & 1u;
                    while (!mbar_try(&norms_full[t % kTcNormSlots], nph) && global_ns() - t0 < kWaitLimitNs) {
                    }
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // ---- MMA issuer
            const uint32_t idesc = idesc_bf16(kTcBM, kTcBN);
            const uint64_t a_hi0 = sw128_desc(smem_u32(smem + L.a_hi));
            const uint64_t a_lo0 = sw128_desc(smem_u32(smem + L.a_lo));
            const uint32_t a_atom = (kTcBM * 128) >> 4;
            int u = 0, tg = 0, w, g;
            uint32_t aph = 0;
            bool ok = true;
            for (int i = 0; ok && work(i, w, g); i++) {
                if (!mbar_wait(a_full, aph, abort_flag)) break;
                aph ^= 1u;
                tc_fence_after();
                const int nt = p.grp_ntiles[g];
                for (int t = 0; ok && t < nt; t++, tg++) {
                    const int b = tg & 1;
                    const uint32_t bph = (uint32_t)(tg >> 1) & 1u;
                    if (!mbar_wait(&acc_empty[b], bph ^ 1u, abort_flag)) {
                        ok = false;
                        break;
                    }
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
                        const uint64_t bh = sw128_desc(smem_u32(smem + L.b0 + s * L.stage_bytes));
                        const uint64_t bl = bh + (L.term_bytes >> 4);
                        const uint64_t ah = a_hi0 + (uint64_t)(a * a_atom), al = a_lo0 + (uint64_t)(a * a_atom);
                        uint32_t acc = a > 0 ? 1u : 0u;
#pragma unroll
                        for (int kk = 0; kk < 4; kk++) {
                            mma_bf16(d_tmem, ah + 2 * kk, bh + 2 * kk, idesc, acc);
                            acc = 1;
                        }
                        if (p.nterms > 1) {
#pragma unroll
                            for (int kk = 0; kk < 4; kk++) mma_bf16(d_tmem, ah + 2 * kk, bl + 2 * kk, idesc, 1u);
                        }
                        if (p.nterms > 2) {
#pragma unroll
                            for (int kk = 0; kk < 4; kk++) mma_bf16(d_tmem, al + 2 * kk, bh + 2 * kk, idesc, 1u);
                        }
                        mma_commit(&empty[s]);
                    }
                    if (ok) mma_commit(&acc_full[b]);
                }
            }
        }
    } else {
        // ---- epilogue warps 2..17 (and row gathering)
        const int q = warp & 3;
        const int cq = (warp - 2) >> 2;
        const int r = q * 32 + lane;
        const int et = threadIdx.x - 64;
        uint32_t* mg = (uint32_t*)(smem + L.merge);
        tc_load_rows(smem, L, x, p, w0 * kTcBM, p.m, et, kTcEpiWarps * 32);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive(a_full);
        int tg = 0, w, g;
        bool ok = true;
        // After an abort every epilogue warp still walks all work items and reaches
        // every named barrier, skipping the waits and the work.
        for (int i = 0; work(i, w, g); i++) {
            const int nt = p.grp_ntiles[g], c0 = p.grp_cbeg[g];
            int wn, gn;
            const bool has_next = work(i + 1, wn, gn);
            if (has_next && ok) prefetch_rows_l2(x, p, wn * kTcBM, et, kTcEpiWarps * 32);
            const int row = w * kTcBM + r;
            Top2 top;
            top.init();
            for (int t = 0; t < nt; t++, tg++) {
                const int b = tg & 1;
                const uint32_t bph = (uint32_t)(tg >> 1) & 1u;
                ok = ok && mbar_wait(&acc_full[b], bph, abort_flag, 20000);
                ok = ok && mbar_wait(&norms_full[tg % kTcNormSlots], (uint32_t)(tg / kTcNormSlots) & 1u, abort_flag);
                if (!ok) continue;
                tc_fence_after();
                if (t == nt - 1 && has_next) {
                    // Every MMA that reads this tile's rows has completed: gather the
                    // next tile's rows now, so that its MMAs overlap this epilogue.
                    tc_load_rows(smem, L, x, p, wn * kTcBM, p.m, et, kTcEpiWarps * 32);
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    __syncwarp();
                    if (lane == 0) mbar_arrive(a_full);
                }
                const int cq0 = c0 + t * kTcBN + cq * 64;
                const float* nrm = norms_s + (tg % kTcNormSlots) * kTcBN + cq * 64;
                const uint32_t taddr = tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * kTcBN + cq * 64);
#pragma unroll
                for (int ch = 0; ch < 2; ch++) {
                    uint32_t v[32];
                    float s[32];
                    EMB_TMEM_LD32(taddr + ch * 32, v);
                    tmem_wait_ld();
                    tc_regs_ready(v);
                    if (ch == 1) {
                        tc_fence_before();
                        __syncwarp();
                        if (lane == 0) mbar_arrive(&acc_empty[b]);
                    }
                    tc_scores32(v, nrm + ch * 32, s);
                    float k1, k2;
                    tc_top2_32(s, k1, k2);
                    top2_merge_keys(top, k1, k2, cq0 + ch * 32);
                }
            }
            // Merge the four column quarters of each row through shared memory.
            if (cq > 0) {
                uint32_t* e = mg + ((cq - 1) * kTcBM + r) * 4;
                e[0] = __float_as_uint(top.s1);
                e[1] = top.i1;
                e[2] = __float_as_uint(top.s2);
                e[3] = top.i2;
            }
            asm volatile("bar.sync 1, %0;" ::"n"(kTcEpiWarps * 32) : "memory");
            if (ok && cq == 0 && row < p.m) {
#pragma unroll
                for (int o = 0; o < 3; o++) {
                    const uint32_t* e = mg + (o * kTcBM + r) * 4;
                    Top2 ot;
                    ot.s1 = __uint_as_float(e[0]);
                    ot.i1 = e[1];
                    ot.s2 = __uint_as_float(e[2]);
                    ot.i2 = e[3];
                    top.merge(ot);
                }
                const size_t oo = (size_t)row * 2;
                p.part_s[oo] = top.s1;
                p.part_i[oo] = top.i1;
                p.part_s[oo + 1] = top.s2;
                p.part_i[oo + 1] = top.i2;
            }
            // The next work item's quarter records overwrite these.
            asm volatile("bar.sync 1, %0;" ::"n"(kTcEpiWarps * 32) : "memory");
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
