// Persistent grouped search: the tcgen05 contraction of k_assign_tc for the
// proposer's buckets, where every row tile (128 bucket positions of one
// centroid group) scores only its group's columns of the group-sorted
// centroid copy. A CTA per SM walks the bucket tiles blockIdx.x, + gridDim.x, ...
// and keeps its barriers, TMEM and pipelines across them.
//
// Column tiles are 128 centroids (groups hold a few hundred centroids, so a
// narrower tile wastes less past a group's end); a stage is one 64-wide K slice
// of a column tile, hi and lo (32 KB), which leaves room for two row buffers:
//   warp 0       TMA producer: the stages of every column tile of every bucket
//                tile in order, plus the norms of each column tile
//   warp 1       TMEM allocation (four 128-column accumulators) and the MMAs,
//                M=128 N=128 K=16; a bucket tile's MMAs wait for its row
//                buffer, and a commit after its last MMA frees that buffer
//   warps 2..17  epilogue, one 32-column chunk per warp and column tile: top-2
//                per row as in k_assign_tc, merged across the four chunks
//   warp 18      row gatherer: the rows arrive already split into BF16 hi and
//                lo (one pass over the chunk before the launch), so a bucket
//                tile's 128 rows are four-row TMA gathers (tile::gather4) into
//                the row buffer of that tile, one tile ahead of the MMAs; it
//                also asks L2 for the rows of the tile after.
// Every bucket tile has at least one column tile (the host gives empty groups one).
#pragma once
#include "kernels_tc.cuh"

namespace emb {

constexpr int kGrpBN = 128;          // centroids per column tile (MMA N)
constexpr int kGrpAcc = 4;           // TMEM accumulators of kGrpBN columns
constexpr int kGrpMaxStages = 4;
constexpr int kGrpNormSlots = 8;
constexpr int kGrpThreads = kTcThreads + 32;  // plus the row-gathering warp
constexpr int kGrpRowWarp = kGrpThreads / 32 - 1;

struct GrpSmem {
    // Offsets (bytes) inside the 1024-aligned dynamic shared memory; row buffer k at k * a_buf.
    uint32_t a_buf, a_lo, b0, stage_bytes, term_bytes, norms, merge, bars, total;
    int stages;
};

__host__ __device__ inline GrpSmem grp_smem_layout(int kpad, int nterms) {
    GrpSmem s;
    const uint32_t a_term = (uint32_t)kTcBM * kpad * 2;
    const uint32_t a_buf = nterms == 3 ? 2 * a_term : a_term;
    const uint32_t b_term = (uint32_t)kGrpBN * 128;
    s.a_buf = a_buf;
    s.a_lo = a_term;  // within a row buffer
    s.b0 = 2 * a_buf;
    s.term_bytes = b_term;
    s.stage_bytes = b_term * (nterms == 1 ? 1 : 2);
    const uint32_t fixed = kGrpNormSlots * kGrpBN * 4 + 3 * kTcBM * 16 + 256 + 1024;
    int st = 0;
    while (st < kGrpMaxStages && s.b0 + (st + 1) * s.stage_bytes + fixed <= (uint32_t)kTcSmemLimit) st++;
    s.stages = st;
    s.norms = s.b0 + st * s.stage_bytes;
    s.merge = s.norms + kGrpNormSlots * kGrpBN * 4;
    s.bars = s.merge + 3 * kTcBM * 16;
    s.total = s.bars + 256;
    return s;
}

// Four rows (r0..r3) of 64 BF16 from a 2-D map with one-row boxes, into 512
// consecutive bytes of shared memory (swizzled as the map says).
EMB_DEV void tma_gather4(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int r0, int r1, int r2, int r3) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5, %6, %7}], [%2];"
        ::"r"(smem_u32(dst)), "l"((uint64_t)map), "r"(smem_u32(bar)), "r"(c0), "r"(r0), "r"(r1), "r"(r2), "r"(r3)
        : "memory");
}

// map_hi / map_lo: the sorted centroid copy (64 x 128 boxes); map_rows_hi /
// map_rows_lo: the chunk's rows as BF16 hi / lo, [rows][kpad] (64 x 1 boxes);
// p.gather: chunk row of every bucket position.
__global__ void __launch_bounds__(kGrpThreads, 1)
k_assign_grouped(const __grid_constant__ CUtensorMap map_hi, const __grid_constant__ CUtensorMap map_lo,
                 const __grid_constant__ CUtensorMap map_rows_hi, const __grid_constant__ CUtensorMap map_rows_lo,
                 const TcParams p) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = smem_align1024(smem_raw);
    const GrpSmem L = grp_smem_layout(p.kpad, p.nterms);
    const int S = L.stages;
    uint64_t* full = (uint64_t*)(smem + L.bars);   // [kGrpMaxStages]
    uint64_t* empty = full + kGrpMaxStages;        // [kGrpMaxStages]
    uint64_t* acc_full = empty + kGrpMaxStages;    // [kGrpAcc]
    uint64_t* acc_empty = acc_full + kGrpAcc;      // [kGrpAcc]
    uint64_t* norms_full = acc_empty + kGrpAcc;    // [kGrpNormSlots]
    uint64_t* a_full = norms_full + kGrpNormSlots; // [2] row buffer gathered
    uint64_t* a_empty = a_full + 2;                // [2] every MMA reading the row buffer completed
    uint64_t* mma_done = a_empty + 2;              // every issued MMA completed (teardown)
    uint32_t* tmem_slot = (uint32_t*)(mma_done + 1);
    volatile int* abort_flag = (volatile int*)(tmem_slot + 1);
    float* norms_s = (float*)(smem + L.norms);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nwt = p.m / kTcBM;  // bucket tiles in the launch (m is a whole number of tiles)
    // Work item i of this CTA is bucket tile blockIdx.x + i * gridDim.x; its (first
    // column, column tiles), no tiles past the last bucket tile. Every role loads
    // the next item's record while it works on the current one.
    auto info = [&](int i) -> int2 {
        const int w = (int)blockIdx.x + i * (int)gridDim.x;
        return w < nwt ? p.tile_info[w] : make_int2(0, 0);
    };
    const int2 info0 = info(0);
    if (info0.y <= 0) return;  // no work: the whole CTA leaves before any setup
    const int w0 = (int)blockIdx.x;
    const int natoms = p.kpad / 64;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kGrpMaxStages; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < kGrpAcc; b++) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], kTcEpiWarps);
        }
        for (int i = 0; i < kGrpNormSlots; i++) mbar_init(&norms_full[i], 1);
        for (int b = 0; b < 2; b++) {
            mbar_init(&a_full[b], 1);
            mbar_init(&a_empty[b], 1);
        }
        mbar_init(mma_done, 1);
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
            // ---- TMA producer of the centroid stages
            int u = 0, tg = 0, norms_issued = 0;
            bool ok = true;
            int2 cur = info0;
            for (int i = 0; ok && cur.y > 0; i++) {
                const int2 nxt = info(i + 1);
                const int nt = cur.y, c0 = cur.x;
                for (int t = 0; ok && t < nt; t++, tg++) {
                    const int col = c0 + t * kGrpBN;
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
                            const int ns = tg % kGrpNormSlots;
                            mbar_expect_tx(&norms_full[ns], kGrpBN * 4);
                            bulk_load(norms_s + ns * kGrpBN, p.norms + (size_t)col, kGrpBN * 4, &norms_full[ns]);
                            norms_issued = tg + 1;
                        }
                    }
                }
                cur = nxt;
            }
            // After an abort, let the copies still in flight land before the CTA exits.
            if (*abort_flag) {
                const uint64_t t0 = global_ns();
                for (int v = u > S ? u - S : 0; v < u; v++) {
                    const uint32_t ph = (uint32_t)(v / S) & 1u;
                    while (!mbar_try(&full[v % S], ph) && global_ns() - t0 < kWaitLimitNs) {
                    }
                }
                for (int t = norms_issued > kGrpNormSlots ? norms_issued - kGrpNormSlots : 0; t < norms_issued; t++) {
                    const uint32_t nph = (uint32_t)(t / kGrpNormSlots) & 1u;
                    while (!mbar_try(&norms_full[t % kGrpNormSlots], nph) && global_ns() - t0 < kWaitLimitNs) {
                    }
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // ---- MMA issuer
            const uint32_t idesc = idesc_bf16(kTcBM, kGrpBN);
            const uint32_t a_atom = (kTcBM * 128) >> 4;  // descriptor units per A atom
            int u = 0, tg = 0;
            bool ok = true;
            int2 cur = info0;
            for (int i = 0; ok && cur.y > 0; i++) {
                const int2 nxt = info(i + 1);
                const int ab = i & 1;
                if (!mbar_wait(&a_full[ab], (uint32_t)(i >> 1) & 1u, abort_flag)) break;
                tc_fence_after();
                const uint64_t a_hi0 = sw128_desc(smem_u32(smem + ab * L.a_buf));
                const uint64_t a_lo0 = sw128_desc(smem_u32(smem + ab * L.a_buf + L.a_lo));
                const int nt = cur.y;
                for (int t = 0; ok && t < nt; t++, tg++) {
                    const int b = tg % kGrpAcc;
                    const uint32_t bph = (uint32_t)(tg / kGrpAcc) & 1u;
                    if (!mbar_wait(&acc_empty[b], bph ^ 1u, abort_flag)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t d_tmem = tmem_base + (uint32_t)(b * kGrpBN);
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
                if (ok) mma_commit(&a_empty[ab]);  // the row buffer is free once these MMAs complete
                cur = nxt;
            }
            mma_drain(mma_done);  // no MMA may outlive the TMEM allocation (see k_assign_tc)
        }
    } else if (warp == kGrpRowWarp) {
        // ---- row gatherer: lane l gathers rows 4l .. 4l + 3 of every bucket tile
        const int a_terms = p.nterms == 3 ? 2 : 1;
        const uint32_t bytes = (uint32_t)kTcBM * 128u * (uint32_t)natoms * (uint32_t)a_terms;
        int issued = 0;
        bool ok = true;
        uint32_t idx[4];
        for (int j = 0; j < 4; j++) idx[j] = p.gather[(size_t)w0 * kTcBM + lane * 4 + j];
        int2 cur = info0;
        for (int i = 0; ok && cur.y > 0; i++) {
            const int2 nxt = info(i + 1);
            const int ab = i & 1;
            if (i >= 2) {
                // tile i - 2 used this buffer: its MMAs must have completed
                if (lane == 0) ok = mbar_wait(&a_empty[ab], (uint32_t)((i - 2) >> 1) & 1u, abort_flag);
                ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
                if (!ok) break;
            }
            if (lane == 0) mbar_expect_tx(&a_full[ab], bytes);
            __syncwarp();
            uint8_t* buf = smem + ab * L.a_buf;
            for (int a = 0; a < natoms; a++) {
                const uint32_t off = (uint32_t)(a * kTcBM * 128 + lane * 4 * 128);
                tma_gather4(buf + off, &map_rows_hi, &a_full[ab], a * 64, (int)idx[0], (int)idx[1], (int)idx[2],
                            (int)idx[3]);
                if (a_terms == 2)
                    tma_gather4(buf + L.a_lo + off, &map_rows_lo, &a_full[ab], a * 64, (int)idx[0], (int)idx[1],
                                (int)idx[2], (int)idx[3]);
            }
            issued = i + 1;
            cur = nxt;
            if (nxt.y > 0) {
                const int wn = (int)blockIdx.x + (i + 1) * (int)gridDim.x;
                // the next tile's rows: indices now, their lines into L2 while this tile computes
                for (int j = 0; j < 4; j++) idx[j] = p.gather[(size_t)wn * kTcBM + lane * 4 + j];
                const int row_bytes = p.kpad * 2;
                for (int j = 0; j < 4; j++)
                    for (int o = 0; o < row_bytes; o += 128) {
                        asm volatile("prefetch.global.L2 [%0];" ::"l"((const char*)(p.rows_hi + (size_t)idx[j] * p.kpad) + o));
                        if (a_terms == 2)
                            asm volatile("prefetch.global.L2 [%0];" ::"l"((const char*)(p.rows_lo + (size_t)idx[j] * p.kpad) + o));
                    }
            }
        }
        // After an abort, let the gathers still in flight land before the CTA exits.
        if (*abort_flag && lane == 0) {
            const uint64_t t0 = global_ns();
            for (int i = issued > 2 ? issued - 2 : 0; i < issued; i++)
                while (!mbar_try(&a_full[i & 1], (uint32_t)(i >> 1) & 1u) && global_ns() - t0 < kWaitLimitNs) {
                }
        }
    } else {
        // ---- epilogue warps 2..17
        const int q = warp & 3;
        const int cq = (warp - 2) >> 2;
        const int r = q * 32 + lane;
        uint32_t* mg = (uint32_t*)(smem + L.merge);
        int tg = 0;
        bool ok = true;
        int2 cur = info0;
        // After an abort every epilogue warp still walks all work items and reaches
        // every named barrier, skipping the waits and the work.
        for (int i = 0; cur.y > 0; i++) {
            const int2 nxt = info(i + 1);
            const int nt = cur.y, c0 = cur.x;
            const int row = ((int)blockIdx.x + i * (int)gridDim.x) * kTcBM + r;
            Top2 top;
            top.init();
            for (int t = 0; t < nt; t++, tg++) {
                const int b = tg % kGrpAcc;
                ok = ok && mbar_wait(&acc_full[b], (uint32_t)(tg / kGrpAcc) & 1u, abort_flag, 20000);
                ok = ok && mbar_wait(&norms_full[tg % kGrpNormSlots], (uint32_t)(tg / kGrpNormSlots) & 1u, abort_flag);
                if (!ok) continue;
                tc_fence_after();
                const float* nrm = norms_s + (tg % kGrpNormSlots) * kGrpBN + cq * 32;
                const uint32_t taddr = tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * kGrpBN + cq * 32);
                uint32_t v[32];
                float s[32];
                EMB_TMEM_LD32(taddr, v);
                tmem_wait_ld();
                tc_regs_ready(v);
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&acc_empty[b]);
                tc_scores32(v, nrm, s);
                float k1, k2;
                tc_top2_32(s, k1, k2);
                top2_merge_keys(top, k1, k2, c0 + t * kGrpBN + cq * 32);
            }
            // Merge the four column chunks of each row through shared memory.
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
            // The next work item's chunk records overwrite these.
            asm volatile("bar.sync 1, %0;" ::"n"(kTcEpiWarps * 32) : "memory");
            cur = nxt;
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
