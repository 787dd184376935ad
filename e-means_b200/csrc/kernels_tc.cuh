// tcgen05 fused assign: BF16 operands on the 5th-generation tensor cores with
// FP32 accumulators in TMEM, a per-row running top-2 in the epilogue, so no
// m x k score matrix reaches HBM.
//
// One CTA owns 128 rows (one TMEM lane per row) and walks its share of the
// centroid tiles (256 centroids each, one 128 x 256 FP32 accumulator in TMEM):
//   warp 0       TMA producer: each stage holds one 64-wide K slice (a 128-byte
//                swizzle atom) of a tile's BF16 hi and lo parts; stages ring
//                through as much shared memory as is left (2..4 stages)
//   warp 1       allocates TMEM, issues tcgen05.mma M=128 N=256 K=16 (one thread),
//                commits to mbarriers
//   warps 2..17  epilogue: four warps per TMEM lane quarter, each owning 64
//                columns of the tile: tcgen05.ld, score = norm - 2 acc (packed
//                f32x2 FMA, norms staged in shared memory by a bulk copy),
//                branch-free top-2 of each 32 columns merged into a running top-2
//                per row. Two accumulators (512 TMEM columns) let the epilogue of
//                tile t overlap the MMAs of tile t+1.
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

constexpr int kTcBM = 128;        // rows per CTA (TMEM lanes)
constexpr int kTcBN = 256;        // centroids per tile (accumulator columns, MMA N)
constexpr int kTcMaxStages = 4;   // stage ring depth limit (one K atom of a tile per stage)
constexpr int kTcEpiWarps = 16;   // four warps per TMEM lane quarter
constexpr int kTcThreads = 64 + kTcEpiWarps * 32;  // producer, MMA, epilogue warps
constexpr int kTcTmemCols = 512;  // two 256-column accumulators
// Norms ring. The producer runs at most S <= 4 stages ahead of the MMA, the MMA
// at most two tiles ahead of the epilogue's accumulator release, and a warp
// finishes reading tile t's norms before it releases tile t+1: slot t % 8 is
// therefore refilled (for tile t+8) only after every warp is done with tile t.
constexpr int kTcNormSlots = 8;
constexpr int kTcSmemLimit = 227 * 1024;

struct TcParams {
    int m, d, k, kpad;   // kpad: d rounded up to 64 (one 128-byte swizzle atom per 64 BF16)
    int nterms;          // 1: hi*hi; 2: hi*hi + hi*lo (integer rows); 3: + lo*hi
    const uint32_t* gather;
    const float* norms;  // padded to whole tiles with a huge finite value
    float* part_s;
    uint32_t* part_i;
    int* err;            // set to 1 if a wait gave up (results then re-searched exactly)
    int xvec;            // rows are 16-byte aligned f32 with d % 4 == 0: vector loads
    const uint32_t* gather2;  // optional first-level row map (kernel row -> batch row)
    const float* theta;       // COLLECT: per kernel row, collect scores <= theta
    uint32_t* cand;           // COLLECT: [m][cand_cap] centroid indices
    uint32_t* cand_count;     // COLLECT: [m] candidates found (may exceed cand_cap)
    int cand_cap;
    const uint32_t* m_dev;    // COLLECT: if set, the row count is min(m, *m_dev), read on the device
    // Grouped search (k_assign_grouped, centroid groups of a group-sorted matrix):
    // bucket tile t scores columns [tile_info[t].x, + 128 tile_info[t].y) of its
    // group (y = 0: past the last tile). Column starts are multiples of 32, so
    // packed keys and the norms copy stay aligned.
    const int2* tile_info;
    const __nv_bfloat16* rows_hi;  // grouped search: the chunk's rows split into BF16 hi / lo, [rows][kpad]
    const __nv_bfloat16* rows_lo;
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
// Same, letting the warp sleep up to `hint_ns` inside the instruction (it
// returns as soon as the phase completes): waiting warps stop taking issue slots.
EMB_DEV bool mbar_try_sleep(uint64_t* bar, uint32_t parity, uint32_t hint_ns) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(hint_ns)
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
EMB_DEV bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag, uint32_t hint_ns = 0) {
    if (mbar_try(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t i = 1;; i++) {
        if (hint_ns ? mbar_try_sleep(bar, parity, hint_ns) : mbar_try(bar, parity)) return true;
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

struct TcSmem {
    // Offsets (bytes) inside the dynamic shared memory block (1024-aligned base).
    uint32_t a_hi, a_lo, b0, stage_bytes, term_bytes, norms, merge, bars, pub, total;
    int stages;
};

__host__ __device__ inline TcSmem tc_smem_layout(int kpad, int nterms) {
    TcSmem s;
    const uint32_t a_bytes = (uint32_t)kTcBM * kpad * 2;
    const uint32_t b_term = (uint32_t)kTcBN * 128;  // one K atom (64 BF16) of 256 centroids
    const int bterms = nterms == 1 ? 1 : 2;
    s.a_hi = 0;
    s.a_lo = a_bytes;
    const uint32_t a_total = nterms == 3 ? 2 * a_bytes : a_bytes;
    s.b0 = a_total;
    s.term_bytes = b_term;
    s.stage_bytes = b_term * bterms;
    // norms, merge, barriers, published top-2 keys, alignment
    const uint32_t fixed = kTcNormSlots * kTcBN * 4 + 3 * kTcBM * 16 + 256 + 4 * kTcBM * 8 + 1024;
    int st = 0;
    while (st < kTcMaxStages && a_total + (st + 1) * s.stage_bytes + fixed <= (uint32_t)kTcSmemLimit) st++;
    s.stages = st;
    s.norms = s.b0 + st * s.stage_bytes;                 // [8][256] f32
    s.merge = s.norms + kTcNormSlots * kTcBN * 4;        // [3][128] x (s1, i1, s2, i2)
    s.bars = s.merge + 3 * kTcBM * 16;
    s.pub = s.bars + 256;                                // [4 column quarters][128 rows] float2 (s1, s2)
    s.total = s.pub + 4 * kTcBM * 8;
    return s;
}

// Byte offset of 16-byte chunk `kc` (8 BF16 along K) of row r in a K-major,
// 128B-swizzled tile of `rows` rows: atoms of 64 BF16 (128 B per row), 16-byte
// chunks XOR-permuted by the row index mod 8 (the layout TMA SWIZZLE_128B writes).
EMB_DEV uint32_t sw128_offset(int r, int kc, int rows) {
    int atom = kc >> 3, c = kc & 7;
    return (uint32_t)(atom * rows * 128 + r * 128 + ((c ^ (r & 7)) << 4));
}

template <typename T>
EMB_DEV void tc_load_rows(uint8_t* smem, const TcSmem& L, const T* __restrict__ x, const TcParams& p, int row0,
                          int m, int tid, int nthr) {
    // 128 rows x (kpad / 8) chunks of 8 elements. Each thread issues the loads of
    // up to four chunks before converting any of them, so that four gathered
    // rows' latencies overlap instead of following one another.
    constexpr int kBatch = 4;
    const int nchunk = p.kpad / 8;
    const int total = kTcBM * nchunk;
    for (int base = tid; base < total; base += kBatch * nthr) {
        float v[kBatch][8];
#pragma unroll
        for (int u = 0; u < kBatch; u++) {
            const int t = base + u * nthr;
#pragma unroll
            for (int i = 0; i < 8; i++) v[u][i] = 0.0f;
            if (t >= total) continue;
            const int r = t / nchunk, kc = t % nchunk;
            const int g = row0 + r;
            if (g >= m) continue;
            size_t src = p.gather2 ? (size_t)p.gather2[g] : (size_t)g;
            if (p.gather) src = p.gather[src];
            const T* xr = x + src * (size_t)p.d;
            const int k0 = kc * 8;
            if (sizeof(T) == 4 && p.xvec && k0 + 8 <= p.d) {
                const float4 a = *reinterpret_cast<const float4*>(xr + k0);
                const float4 b = *reinterpret_cast<const float4*>(xr + k0 + 4);
                v[u][0] = a.x; v[u][1] = a.y; v[u][2] = a.z; v[u][3] = a.w;
                v[u][4] = b.x; v[u][5] = b.y; v[u][6] = b.z; v[u][7] = b.w;
            } else {
#pragma unroll
                for (int i = 0; i < 8; i++) v[u][i] = (k0 + i < p.d) ? to_f32(xr[k0 + i]) : 0.0f;
            }
        }
#pragma unroll
        for (int u = 0; u < kBatch; u++) {
            const int t = base + u * nthr;
            if (t >= total) continue;
            const int r = t / nchunk, kc = t % nchunk;
            uint32_t hw[4], lw[4];
#pragma unroll
            for (int i = 0; i < 4; i++) {
                __nv_bfloat16 h0 = __float2bfloat16_rn(v[u][2 * i]), h1 = __float2bfloat16_rn(v[u][2 * i + 1]);
                __nv_bfloat16 l0 = __float2bfloat16_rn(v[u][2 * i] - __bfloat162float(h0));
                __nv_bfloat16 l1 = __float2bfloat16_rn(v[u][2 * i + 1] - __bfloat162float(h1));
                hw[i] = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
                lw[i] = (uint32_t)__bfloat16_as_ushort(l0) | ((uint32_t)__bfloat16_as_ushort(l1) << 16);
            }
            const uint32_t off = sw128_offset(r, kc, kTcBM);
            *reinterpret_cast<uint4*>(smem + L.a_hi + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
            if (p.nterms == 3) *reinterpret_cast<uint4*>(smem + L.a_lo + off) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
        }
    }
}

EMB_DEV void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"((uint64_t)src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

EMB_DEV float min3f(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// s = norm - 2 acc for two columns at once (fma.rn.f32x2: two IEEE fmas).
EMB_DEV void fma2_scores(float a0, float a1, float n0, float n1, float& s0, float& s1) {
    asm("{\n .reg .b64 ra, rb, rc, rd;\n mov.b64 ra, {%2, %3};\n mov.b64 rb, {%4, %5};\n mov.b64 rc, {%6, %7};\n"
        " fma.rn.f32x2 rd, ra, rb, rc;\n mov.b64 {%0, %1}, rd;\n}\n"
        : "=f"(s0), "=f"(s1)
        : "f"(a0), "f"(a1), "f"(-2.0f), "f"(-2.0f), "f"(n0), "f"(n1));
}

// Scores of 32 accumulator columns: s = norm - 2 acc (one rounding).
EMB_DEV void tc_scores32(const uint32_t (&v)[32], const float* __restrict__ nrm, float (&s)[32]) {
#pragma unroll
    for (int j = 0; j < 32; j += 4) {
        float4 n4 = *reinterpret_cast<const float4*>(nrm + j);
        fma2_scores(__uint_as_float(v[j]), __uint_as_float(v[j + 1]), n4.x, n4.y, s[j], s[j + 1]);
        fma2_scores(__uint_as_float(v[j + 2]), __uint_as_float(v[j + 3]), n4.z, n4.w, s[j + 2], s[j + 3]);
    }
}

// Smallest of 32 scores (NaN-ignoring).
EMB_DEV float tc_min32(const float (&s)[32]) {
    float m[11];
#pragma unroll
    for (int i = 0; i < 10; i++) m[i] = min3f(s[3 * i], s[3 * i + 1], s[3 * i + 2]);
    m[10] = fminf(s[30], s[31]);
    float a = min3f(m[0], m[1], m[2]), b = min3f(m[3], m[4], m[5]), c = min3f(m[6], m[7], m[8]);
    return min3f(min3f(a, b, c), m[9], m[10]);
}

// Two smallest of 32 scores, branch-free. Each score's 5 low mantissa bits are
// replaced by its column j (a relative change below 2^-18, which the error bound
// covers), so min/max carry the column along; NaN keys are ignored by min/max.
// Returns keys k1 <= k2.
EMB_DEV void tc_top2_32(const float (&s)[32], float& k1, float& k2) {
    float lo[16], hi[16];
#pragma unroll
    for (int p = 0; p < 16; p++) {
        float a = __uint_as_float((__float_as_uint(s[2 * p]) & ~31u) | (uint32_t)(2 * p));
        float b = __uint_as_float((__float_as_uint(s[2 * p + 1]) & ~31u) | (uint32_t)(2 * p + 1));
        lo[p] = fminf(a, b);
        hi[p] = fmaxf(a, b);
    }
#pragma unroll
    for (int w = 8; w >= 1; w >>= 1) {
#pragma unroll
        for (int p = 0; p < w; p++) {
            float a1 = lo[p], a2 = hi[p], b1 = lo[p + w], b2 = hi[p + w];
            lo[p] = fminf(a1, b1);
            hi[p] = min3f(fmaxf(a1, b1), a2, b2);
        }
    }
    k1 = lo[0];
    k2 = hi[0];
}

// An upper bound of a row's final second-smallest key from the running top-2
// pairs (s1 <= s2) that the four column-quarter warps of the row publish: the
// second smallest of their union, or at least the smaller of the second
// smallest s1 and the smallest s2. Values only decrease, so stale reads of
// another warp's pair are still bounds.
EMB_DEV float tc_row_bound(const float2* pub, int r) {
    float2 v[4];
#pragma unroll
    for (int c = 0; c < 4; c++)
        asm volatile("ld.volatile.shared.v2.f32 {%0, %1}, [%2];"
                     : "=f"(v[c].x), "=f"(v[c].y)
                     : "r"(smem_u32(pub + c * kTcBM + r)));
    const float lo01 = fminf(v[0].x, v[1].x), hi01 = fmaxf(v[0].x, v[1].x);
    const float lo23 = fminf(v[2].x, v[3].x), hi23 = fmaxf(v[2].x, v[3].x);
    const float second_s1 = min3f(fmaxf(lo01, lo23), hi01, hi23);
    return fminf(second_s1, fminf(fminf(v[0].y, v[1].y), fminf(v[2].y, v[3].y)));
}

// Two smallest keys of the 16 scores s[h*16 .. h*16+15] (columns h*16 + j in the
// key bits), as tc_top2_32 for half a chunk.
EMB_DEV void tc_top2_16(const float (&s)[32], int h, float& k1, float& k2) {
    float lo[8], hi[8];
#pragma unroll
    for (int p = 0; p < 8; p++) {
        const int j0 = h * 16 + 2 * p;
        float a = __uint_as_float((__float_as_uint(s[j0]) & ~31u) | (uint32_t)j0);
        float b = __uint_as_float((__float_as_uint(s[j0 + 1]) & ~31u) | (uint32_t)(j0 + 1));
        lo[p] = fminf(a, b);
        hi[p] = fmaxf(a, b);
    }
#pragma unroll
    for (int w = 4; w >= 1; w >>= 1) {
#pragma unroll
        for (int p = 0; p < w; p++) {
            float a1 = lo[p], a2 = hi[p], b1 = lo[p + w], b2 = hi[p + w];
            lo[p] = fminf(a1, b1);
            hi[p] = min3f(fmaxf(a1, b1), a2, b2);
        }
    }
    k1 = lo[0];
    k2 = hi[0];
}

// Smallest of the 16 scores s[h*16 .. h*16+15] (NaN-ignoring).
EMB_DEV float tc_min16(const float (&s)[32], int h) {
    const int o = h * 16;
    const float a = min3f(s[o], s[o + 1], s[o + 2]), b = min3f(s[o + 3], s[o + 4], s[o + 5]);
    const float c = min3f(s[o + 6], s[o + 7], s[o + 8]), d = min3f(s[o + 9], s[o + 10], s[o + 11]);
    const float e = min3f(s[o + 12], s[o + 13], s[o + 14]);
    return fminf(min3f(a, b, c), min3f(d, e, s[o + 15]));
}

// Whether scores whose smallest is m can hold one of a row's final two smallest
// keys: only a key below an upper bound T of the row's final second key can. A
// key differs from its score by less than 2^-18 relative (the 5 column bits), so
// scores whose smallest, lowered by 2^-17 relative, is still >= T cannot; NaN
// scores never rule a chunk out.
EMB_DEV bool tc_min_may_enter(float m, float T) { return !(fmaf(-fabsf(m), 0x1p-17f, m) >= T); }

// Merge a chunk's top-2 (keys k1 <= k2 at columns cb + key&31) into a running top-2.
EMB_DEV void top2_merge_keys(Top2& t, float k1, float k2, int cb) {
    const uint32_t j1 = (uint32_t)cb + (__float_as_uint(k1) & 31u), j2 = (uint32_t)cb + (__float_as_uint(k2) & 31u);
    const bool cw = k1 < t.s1;  // chunk wins first place
    const float w2 = cw ? k2 : t.s2, l1 = cw ? t.s1 : k1;
    const uint32_t w2i = cw ? j2 : t.i2, l1i = cw ? t.i1 : j1;
    t.s1 = cw ? k1 : t.s1;
    t.i1 = cw ? j1 : t.i1;
    const bool bw = w2 < l1;
    t.s2 = bw ? w2 : l1;
    t.i2 = bw ? w2i : l1i;
}

// Keep the compiler from reading registers of a tcgen05.ld before its wait.
EMB_DEV void tc_regs_ready(uint32_t (&v)[32]) {
#pragma unroll
    for (int j = 0; j < 32; j++) asm volatile("" : "+r"(v[j]));
}

// Grid: (ceil(m / 128), nsplit); CTA (bx, by) walks centroid tiles by, by + nsplit, ...
// COLLECT = false: per-row top-2 of approximate scores to part_s/part_i.
// COLLECT = true : every centroid with approximate score <= theta[row] is appended
//                  to cand[row][*] (cand_count[row] counts all, capped storage).
template <typename T, bool COLLECT>
__global__ void __launch_bounds__(kTcThreads, 1)
k_assign_tc(const T* __restrict__ x, const __grid_constant__ CUtensorMap map_hi,
            const __grid_constant__ CUtensorMap map_lo, const TcParams p) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const TcSmem L = tc_smem_layout(p.kpad, p.nterms);
    const int S = L.stages;
    uint64_t* full = (uint64_t*)(smem + L.bars);          // [kTcMaxStages]
    uint64_t* empty = full + kTcMaxStages;                // [kTcMaxStages]
    uint64_t* acc_full = empty + kTcMaxStages;            // [2]
    uint64_t* acc_empty = acc_full + 2;                   // [2]
    uint64_t* norms_full = acc_empty + 2;                 // [kTcNormSlots]
    uint32_t* tmem_slot = (uint32_t*)(norms_full + kTcNormSlots);
    volatile int* abort_flag = (volatile int*)(tmem_slot + 1);
    float* norms_s = (float*)(smem + L.norms);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int row0 = blockIdx.x * kTcBM;
    int m = p.m;
    if (COLLECT && p.m_dev) {
        // Row count known only on the device (graph-captured refine): CTAs past it leave at once.
        const int md = (int)*p.m_dev;
        m = md < m ? md : m;
        if (row0 >= m) return;
    }
    const int nsplit = gridDim.y;
    const int ntiles_all = (p.k + kTcBN - 1) / kTcBN;
    const int my_tiles = (int)blockIdx.y < ntiles_all ? (ntiles_all - (int)blockIdx.y + nsplit - 1) / nsplit : 0;
    // Column of this CTA's tile t: col_first + t * col_step.
    const int col_first = (int)blockIdx.y * kTcBN, col_step = nsplit * kTcBN;
    const int natoms = p.kpad / 64;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kTcMaxStages; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], kTcEpiWarps);  // one arrival per epilogue warp
        }
        for (int i = 0; i < kTcNormSlots; i++) mbar_init(&norms_full[i], 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) tmem_alloc(tmem_slot, kTcTmemCols);
    // ---- TMA producer unit u = (tile t, K atom a) into stage u % S; norms once per tile
    const int nunits = my_tiles * natoms;
    auto issue = [&](int u) {
        const int t = u / natoms, a = u - t * natoms;
        const int s = u % S;
        const int col = col_first + t * col_step;
        uint8_t* stage = smem + L.b0 + s * L.stage_bytes;
        mbar_expect_tx(&full[s], L.stage_bytes);
        tma_load_2d(stage, &map_hi, &full[s], a * 64, col);
        if (p.nterms > 1) tma_load_2d(stage + L.term_bytes, &map_lo, &full[s], a * 64, col);
        if (a == 0) {
            const int ns = t % kTcNormSlots;
            mbar_expect_tx(&norms_full[ns], kTcBN * 4);
            bulk_load(norms_s + ns * kTcBN, p.norms + (size_t)col, kTcBN * 4, &norms_full[ns]);
        }
    };
    __syncthreads();  // barriers initialised: the first stages load while the rows are gathered
    int issued = 0;
    if (warp == 0 && lane == 0) {
        // The first S stages are free: no wait on `empty` before them.
        issued = nunits < S ? nunits : S;
        for (int u = 0; u < issued; u++) issue(u);
    }
    tc_load_rows(smem, L, x, p, row0, m, threadIdx.x, blockDim.x);
    {  // published top-2 pairs of the single-term epilogue start at +inf
        float2* pub = (float2*)(smem + L.pub);
        for (int i = threadIdx.x; i < 4 * kTcBM; i += blockDim.x) pub[i] = make_float2(INFINITY, INFINITY);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            for (int u = issued; u < nunits; u++) {
                const int s = u % S;
                const uint32_t ph = (uint32_t)(u / S) & 1u;
                if (!mbar_wait(&empty[s], ph ^ 1u, abort_flag)) break;
                issue(u);
                issued = u + 1;
            }
            // After an abort, let the copies still in flight land before the CTA
            // exits; bounded like every wait.
            if (*abort_flag) {
                const uint64_t t0 = global_ns();
                for (int u = issued > S ? issued - S : 0; u < issued; u++) {
                    const uint32_t ph = (uint32_t)(u / S) & 1u;
                    while (!mbar_try(&full[u % S], ph) && global_ns() - t0 < kWaitLimitNs) {
                    }
                }
                const int tl = issued > 0 ? (issued - 1) / natoms : -1;
                for (int t = tl >= kTcNormSlots ? tl - kTcNormSlots + 1 : 0; t <= tl; t++) {
                    const uint32_t nph = (uint32_t)(t / kTcNormSlots) & 1u;
                    while (!mbar_try(&norms_full[t % kTcNormSlots], nph) && global_ns() - t0 < kWaitLimitNs) {
                    }
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // ---- MMA issuer: per unit, nterms x 4 MMAs of M=128 N=256 K=16
            const uint32_t idesc = idesc_bf16(kTcBM, kTcBN);
            const uint64_t a_hi0 = sw128_desc(smem_u32(smem + L.a_hi));
            const uint64_t a_lo0 = sw128_desc(smem_u32(smem + L.a_lo));
            const uint32_t a_atom = (kTcBM * 128) >> 4;  // descriptor units (16 B) per A atom
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
                    const uint64_t bh = sw128_desc(smem_u32(smem + L.b0 + s * L.stage_bytes));
                    const uint64_t bl = bh + (L.term_bytes >> 4);
                    const uint64_t ah = a_hi0 + (uint64_t)(a * a_atom), al = a_lo0 + (uint64_t)(a * a_atom);
                    uint32_t acc = a > 0 ? 1u : 0u;
#pragma unroll
                    for (int kk = 0; kk < 4; kk++) {  // 16 BF16 = 32 B = 2 descriptor units per K step
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
    } else {
        // ---- epilogue: warps 2..17. Thread = row (TMEM lane); warp w takes the
        // 64-column quarter (w - 2) / 4 of every tile, as two 32-column chunks.
        const int q = warp & 3;  // TMEM lane quarter this warp may access
        const int cq = (warp - 2) >> 2;
        const int r = q * 32 + lane;
        const int row = row0 + r;
        Top2 top;
        top.init();
        float theta = 0.0f;
        if (COLLECT) theta = row < m ? p.theta[row] : __int_as_float(0x7fc00000);
        for (int t = 0; t < my_tiles; t++) {
            const int b = t & 1;
            const uint32_t bph = (uint32_t)(t >> 1) & 1u;
            if (!mbar_wait(&acc_full[b], bph, abort_flag, 20000)) break;
            if (!mbar_wait(&norms_full[t % kTcNormSlots], (uint32_t)(t / kTcNormSlots) & 1u, abort_flag)) break;
            tc_fence_after();
            const int cq0 = col_first + t * col_step + cq * 64;
            const float* nrm = norms_s + (t % kTcNormSlots) * kTcBN + cq * 64;
            const uint32_t taddr = tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * kTcBN + cq * 64);
            // The published bound is read once per tile (the epilogue is issue-bound);
            // within the tile the warp's own second key tightens it.
            const float tile_bound = (!COLLECT && p.nterms == 1) ? tc_row_bound((const float2*)(smem + L.pub), r) : 0.0f;
#pragma unroll
            for (int ch = 0; ch < 2; ch++) {
                uint32_t v[32];
                float s[32];
                EMB_TMEM_LD32(taddr + ch * 32, v);
                tmem_wait_ld();
                tc_regs_ready(v);
                if (ch == 1) {
                    // Both chunks of this warp are in registers: release the accumulator.
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&acc_empty[b]);
                }
                tc_scores32(v, nrm + ch * 32, s);
                const int cb = cq0 + ch * 32;
                if (!COLLECT) {
                    // Single-term search (epilogue-bound): the keyed tournament only for
                    // chunks that can hold one of the row's final two keys, judged
                    // against the top-2 pairs that the row's four column-quarter warps
                    // publish in shared memory (the branch stays uniform across the
                    // warp). The three-term search is tensor-bound and takes every chunk.
                    float2* pub = (float2*)(smem + L.pub);
                    if (p.nterms > 1) {
                        float k1, k2;
                        tc_top2_32(s, k1, k2);
                        top2_merge_keys(top, k1, k2, cb);
                    } else {
                        // Judged per 16-column half: a half needs its tournament less
                        // often than the whole chunk, and costs less than half of it.
                        // The warp's own running s2 is an upper bound of the row's final
                        // s2 too (its columns are a subset of the row's).
                        const float bound = fminf(tile_bound, top.s2);
                        bool changed = false;
#pragma unroll
                        for (int hh = 0; hh < 2; hh++) {
                            if (__any_sync(__activemask(), tc_min_may_enter(tc_min16(s, hh), bound))) {
                                float k1, k2;
                                tc_top2_16(s, hh, k1, k2);
                                top2_merge_keys(top, k1, k2, cb);
                                changed = true;
                            }
                        }
                        if (changed)
                            asm volatile("st.volatile.shared.v2.f32 [%0], {%1, %2};" ::"r"(smem_u32(pub + cq * kTcBM + r)),
                                         "f"(top.s1), "f"(top.s2)
                                         : "memory");
                    }
                } else if (tc_min32(s) <= theta) {
#pragma unroll
                    for (int j = 0; j < 32; j++) {
                        if (s[j] <= theta && cb + j < p.k) {
                            uint32_t slot = atomicAdd(&p.cand_count[row], 1u);
                            if (slot < (uint32_t)p.cand_cap) p.cand[(size_t)row * p.cand_cap + slot] = (uint32_t)(cb + j);
                        }
                    }
                }
            }
        }
        if (!COLLECT) {
            // Merge the four column quarters of each row through shared memory.
            uint32_t* mg = (uint32_t*)(smem + L.merge);
            if (cq > 0) {
                uint32_t* e = mg + ((cq - 1) * kTcBM + r) * 4;
                e[0] = __float_as_uint(top.s1);
                e[1] = top.i1;
                e[2] = __float_as_uint(top.s2);
                e[3] = top.i2;
            }
            asm volatile("bar.sync 1, %0;" ::"n"(kTcEpiWarps * 32) : "memory");
            if (cq == 0 && row < m) {
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
                size_t oo = ((size_t)blockIdx.y * p.m + row) * 2;
                p.part_s[oo] = top.s1;
                p.part_i[oo] = top.i1;
                p.part_s[oo + 1] = top.s2;
                p.part_i[oo + 1] = top.i2;
            }
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
