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
// within ~3 2^-16 |x||c| of exact, which certifies nearly every row's top-2; the
// exact re-score happens in kernels_exact.cuh.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>

#include "common.cuh"
#include "kernels_exact.cuh"

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
// Suspend-time hint of the control warps' barrier waits (producer, MMA issuer,
// row loaders): a waiting thread sleeps until the phase completes (or the hint
// runs out) instead of spinning on issue slots the epilogue warps need.
constexpr uint32_t kTcCtlSleepNs = 2000;
// The persistent search kernel k_assign_tc adds two row-loading warps (2, 3)
// before its 16 epilogue warps (4..19).
constexpr int kTcLoadWarps = 2;
constexpr int kTcEpi0 = 2 + kTcLoadWarps;
constexpr int kTcPThreads = 32 * (kTcEpi0 + kTcEpiWarps);
constexpr int kTcRowScaleSlots = 4;  // FP8 per-row scales, a ring over work items
// Norms inside the contraction (single-term BF16 search of f32 rows): each tile
// starts with one K = 16 MMA of a constant row operand [1, 1, 1, 0, ...] against
// the tile's half-norms split into three BF16 parts, so the accumulator holds
// norm / 2 - x . c (the rows enter negated), half the score, and the epilogue
// scores without loading norms or multiplying. A ring of two 8 KB slices.
constexpr int kTcNmSlots = 2;
constexpr uint32_t kTcNmSlotBytes = (uint32_t)kTcBN * 32;  // 256 centroids x 16 BF16
constexpr uint32_t kTcNmConstBytes = (uint32_t)kTcBM * 32;  // 128 rows x 16 BF16

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
    // Test of the bounded-wait abort path: when stall_ns > 0, the first epilogue
    // warp waits at tile stall_tile on a barrier nothing completes, with limit
    // stall_ns, so the wait runs out and the kernel takes its abort path (results
    // re-searched). Zero (the default of a zeroed struct): off.
    int stall_tile;
    uint64_t stall_ns;
    // FP8 (e4m3) operands: rows scaled per row by a power of two and centroids per
    // centroid; wf8[j] = -2 / (centroid j's scale), 0 past k (score = norm + acc r w).
    const float* wf8;
    int nsplit;  // column splits of the search (work item = row tile x split)
    // Norms inside the contraction: [tiles * 256][16] BF16, row j = the three BF16
    // parts of norms[j] / 2, then zeros (k_prep_nrm16).
    const __nv_bfloat16* nrm16;
    // Certification at the end of each work item (norms inside the contraction,
    // one column split, f32 rows with d % 16 == 0 and 16-byte aligned rows and
    // centroids, AVX-512 rounding): the decisions of k_certify16v, taken by the
    // epilogue warps from the row tile's merged top-2, in place of that kernel.
    int fuse;
    const float* cx;  // f32 centroids [k][d]
    const Bounds* bounds;
    float ka, kb, kr, ka2, kb2;
    uint32_t* labels;
    float* dist;
    uint32_t* redo_rows;
    float* redo_theta;
    uint32_t* redo_count;
    uint32_t* cert_count;
};

// ---- PTX wrappers -----------------------------------------------------------
EMB_DEV uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// The dynamic shared memory base raised to a 1024-byte boundary (the 128-byte
// swizzle atoms' alignment). Pointer arithmetic on the shared array, not an
// integer round trip, so the compiler keeps the accesses in the shared window
// (ld.shared / st.shared) instead of generic loads.
EMB_DEV uint8_t* smem_align1024(uint8_t* raw) { return raw + ((1024u - (smem_u32(raw) & 1023u)) & 1023u); }

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
// complete within limit_ns, or if another role already aborted.
EMB_DEV bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag, uint32_t hint_ns = 0,
                       uint64_t limit_ns = kWaitLimitNs) {
    if (mbar_try(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t i = 1;; i++) {
        if (hint_ns ? mbar_try_sleep(bar, parity, hint_ns) : mbar_try(bar, parity)) return true;
        if ((i & 63) == 0) {
            if (*abort_flag) return false;
            if (global_ns() - t0 > limit_ns) {
                *abort_flag = 1;
                return false;
            }
        }
    }
}

// Wait, bounded by kWaitLimitNs and whatever the abort flag says, for a phase
// that is certain to complete (copies or MMAs already issued): used on the way
// out of a kernel, so that no asynchronous operation still reads or writes
// shared memory or TMEM when the CTA frees them.
EMB_DEV void mbar_drain(uint64_t* bar, uint32_t parity) {
    const uint64_t t0 = global_ns();
    while (!mbar_try(bar, parity) && global_ns() - t0 < kWaitLimitNs) {
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

// Same for a K-major operand of 16 BF16 per row (32-byte rows), 32-byte swizzle:
// 8-row groups 256 B apart. The swizzle only exchanges the two 16-byte halves of
// a row, which the norm operands are built to be indifferent to (see kTcNmSlots).
EMB_DEV uint64_t sw32_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);        // start address
    d |= (uint64_t)1 << 16;                         // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(256 >> 4) << 32;                // stride byte offset: 8 rows x 32 B
    d |= (uint64_t)1 << 46;                         // descriptor version (sm_100)
    d |= (uint64_t)6 << 61;                         // SWIZZLE_32B
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

// Called once by the MMA-issuing thread before it leaves, normally or after an
// abort: a commit tracks every tcgen05.mma the thread issued before it, so once
// `bar` (initialised with one arrival, used only here) completes its phase no
// MMA is still reading shared memory or writing TMEM, and TMEM may be freed.
EMB_DEV void mma_drain(uint64_t* bar) {
    mma_commit(bar);
    mbar_drain(bar, 0);
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

// Shared memory of the persistent search kernel k_assign_tc (offsets in bytes from
// a 1024-aligned base). kpad is d rounded up to one 128-byte swizzle atom per row:
// 64 BF16 or 128 e4m3 elements.
struct TcLayout {
    uint32_t a_buf;        // bytes of one row-tile buffer (hi, then lo for three terms)
    uint32_t a_lo;         // offset of the lo part inside a buffer
    uint32_t b0, stage_bytes, term_bytes;
    uint32_t norms, nrm_slot_bytes;  // ring of per-tile norms (FP8: norms, then column factors;
                                     // norms in the contraction: kTcNmSlots BF16 slices)
    uint32_t nconst;       // norms in the contraction: the constant row operand
    uint32_t fin;          // norms in the contraction: an item's merged top-2 for the certification
    uint32_t rscale;       // FP8: ring of per-row scales [kTcRowScaleSlots][128]
    uint32_t merge, bars, pub, total;
    int stages, nbuf;
};

// nm: norms inside the contraction (kTcNmSlots), which also needs 512 bytes of
// barriers instead of 256.
__host__ __device__ inline TcLayout tc_layout(int kpad, int nterms, bool fp8, bool nm = false) {
    TcLayout s;
    const uint32_t a_term = (uint32_t)kTcBM * (uint32_t)kpad * (fp8 ? 1u : 2u);
    s.a_buf = a_term * ((!fp8 && nterms == 3) ? 2u : 1u);
    s.a_lo = a_term;
    s.term_bytes = (uint32_t)kTcBN * 128;  // one K atom of 256 centroids
    s.stage_bytes = s.term_bytes * ((fp8 || nterms == 1) ? 1u : 2u);
    s.nrm_slot_bytes = nm ? kTcNmSlotBytes : (uint32_t)kTcBN * 4 * (fp8 ? 2u : 1u);
    const uint32_t nrm_bytes =
        nm ? kTcNmSlots * kTcNmSlotBytes + kTcNmConstBytes + kTcBM * 16 : kTcNormSlots * s.nrm_slot_bytes;
    const uint32_t bar_bytes = nm ? 512u : 256u;
    const uint32_t fixed = nrm_bytes + kTcRowScaleSlots * kTcBM * 4 + 3 * kTcBM * 16 + bar_bytes + 4 * kTcBM * 4 + 1024;
    // Two row-tile buffers (the next tile's rows load while the current one is
    // searched) when they leave room for three stages, else one.
    s.nbuf = 2 * s.a_buf + 3 * s.stage_bytes + fixed <= (uint32_t)kTcSmemLimit ? 2 : 1;
    int st = 0;
    while (st < kTcMaxStages && s.nbuf * s.a_buf + (st + 1) * s.stage_bytes + fixed <= (uint32_t)kTcSmemLimit) st++;
    s.stages = st;
    s.b0 = s.nbuf * s.a_buf;
    s.norms = s.b0 + st * s.stage_bytes;
    s.nconst = s.norms + (nm ? kTcNmSlots * kTcNmSlotBytes : 0u);
    s.fin = s.nconst + (nm ? kTcNmConstBytes : 0u);
    s.rscale = s.norms + nrm_bytes;
    s.merge = s.rscale + kTcRowScaleSlots * kTcBM * 4;
    s.bars = s.merge + 3 * kTcBM * 16;
    s.pub = s.bars + bar_bytes;            // [4 column quarters][128 rows] published best key
    s.total = s.pub + 4 * kTcBM * 4;
    return s;
}

// Byte offset of 16-byte chunk `kc` (8 BF16 along K) of row r in a K-major,
// 128B-swizzled tile of `rows` rows: atoms of 64 BF16 (128 B per row), 16-byte
// chunks XOR-permuted by the row index mod 8 (the layout TMA SWIZZLE_128B writes).
EMB_DEV uint32_t sw128_offset(int r, int kc, int rows) {
    int atom = kc >> 3, c = kc & 7;
    return (uint32_t)(atom * rows * 128 + r * 128 + ((c ^ (r & 7)) << 4));
}

// Source row of kernel row g: through the optional first-level map, then the gather.
EMB_DEV size_t tc_src_row(const TcParams& p, int g) {
    size_t src = p.gather2 ? (size_t)p.gather2[g] : (size_t)g;
    if (p.gather) src = p.gather[src];
    return src;
}

// Row tile -> BF16 hi (and lo for three terms) in the K-major 128B-swizzled layout,
// by threads tid = 0 .. nthr-1: 128 rows x (kpad / 8) chunks of 8 elements. Each
// thread issues the loads of up to four chunks before converting any of them, so
// that the gathered rows' latencies overlap. neg: the rows negated (exact; BF16
// rounding to nearest is symmetric), for the norms-in-the-contraction search.
template <typename T>
EMB_DEV void tc_load_rows(uint8_t* a_hi, uint8_t* a_lo, const T* __restrict__ x, const TcParams& p, int row0, int m,
                          int tid, int nthr, bool neg = false) {
    const float sg = neg ? -1.0f : 1.0f;
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
            const T* xr = x + tc_src_row(p, g) * (size_t)p.d;
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
                const float v0 = sg * v[u][2 * i], v1 = sg * v[u][2 * i + 1];
                __nv_bfloat16 h0 = __float2bfloat16_rn(v0), h1 = __float2bfloat16_rn(v1);
                __nv_bfloat16 l0 = __float2bfloat16_rn(v0 - __bfloat162float(h0));
                __nv_bfloat16 l1 = __float2bfloat16_rn(v1 - __bfloat162float(h1));
                hw[i] = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
                lw[i] = (uint32_t)__bfloat16_as_ushort(l0) | ((uint32_t)__bfloat16_as_ushort(l1) << 16);
            }
            const uint32_t off = sw128_offset(r, kc, kTcBM);
            *reinterpret_cast<uint4*>(a_hi + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
            if (p.nterms == 3) *reinterpret_cast<uint4*>(a_lo + off) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
        }
    }
}

// Largest magnitudes for which the FP8 operands keep their error bound: the
// scale below stays a normal power of two and e4m3 rounding stays relative
// (plus a floor the bound covers) for elements near the largest.
constexpr float kFp8MinMag = 0x1p-60f, kFp8MaxMag = 0x1p60f;

// Power-of-two scale that maps a largest magnitude mx into (224, 448], the top
// binade of e4m3 (448 is its largest finite value). Outside [kFp8MinMag,
// kFp8MaxMag] (zero, tiny, huge, inf or NaN) the scale is 1 and *ok false.
EMB_DEV float fp8_scale(float mx, bool* ok) {
    *ok = mx >= kFp8MinMag && mx <= kFp8MaxMag;
    if (!*ok) return 1.0f;
    return __uint_as_float(__float_as_uint(448.0f / mx) & 0xFF800000u);  // round down to a power of two
}

// Two scaled values -> two e4m3 bytes (round to nearest, saturating to +-448).
EMB_DEV uint32_t fp8x2(float a, float b) {
    uint16_t r;
    asm("cvt.rn.satfinite.e4m3x2.f32 %0, %2, %1;" : "=h"(r) : "f"(a), "f"(b));
    return r;
}

// Row tile -> e4m3, one power-of-two scale per row (fp8_scale of its largest
// magnitude), K-major 128B-swizzled: 16-byte chunks of 16 elements, kpad / 16 (8
// or 16) consecutive threads per row, the row maximum reduced across them by
// shuffles. rscale[r] = 1 / scale (exact). Threads tid = 0 .. 63.
template <typename T>
EMB_DEV void tc_load_rows_fp8(uint8_t* a, float* rscale, const T* __restrict__ x, const TcParams& p, int row0, int m,
                              int tid) {
    const int cpr = p.kpad / 16;          // 8 or 16 threads per row
    const int rpp = 64 / cpr;             // rows per pass
    for (int rb = 0; rb < kTcBM; rb += 2 * rpp) {
        float v[2][16];
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const int r = rb + u * rpp + tid / cpr, kc = tid % cpr;
            const int g = row0 + r;
#pragma unroll
            for (int i = 0; i < 16; i++) v[u][i] = 0.0f;
            if (g < m) {
                const T* xr = x + tc_src_row(p, g) * (size_t)p.d;
                const int k0 = kc * 16;
                if (sizeof(T) == 4 && p.xvec && k0 + 16 <= p.d) {
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const float4 f = *reinterpret_cast<const float4*>(xr + k0 + 4 * q);
                        v[u][4 * q] = f.x; v[u][4 * q + 1] = f.y; v[u][4 * q + 2] = f.z; v[u][4 * q + 3] = f.w;
                    }
                } else {
                    for (int i = 0; i < 16; i++) v[u][i] = (k0 + i < p.d) ? to_f32(xr[k0 + i]) : 0.0f;
                }
            }
        }
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const int r = rb + u * rpp + tid / cpr, kc = tid % cpr;
            float mx = 0.0f;
#pragma unroll
            for (int i = 0; i < 16; i++) mx = fmaxf(mx, fabsf(v[u][i]));
            for (int o = cpr >> 1; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            bool in_range;
            const float sc = fp8_scale(mx, &in_range);
            uint32_t w[4];
#pragma unroll
            for (int q = 0; q < 4; q++)
                w[q] = fp8x2(v[u][4 * q] * sc, v[u][4 * q + 1] * sc) | (fp8x2(v[u][4 * q + 2] * sc, v[u][4 * q + 3] * sc) << 16);
            *reinterpret_cast<uint4*>(a + sw128_offset(r, kc, kTcBM)) = make_uint4(w[0], w[1], w[2], w[3]);
            // A zero row is exact (every product 0). Any other row outside the range
            // gets a NaN scale: all its scores are NaN, no candidate survives, and
            // the certification sends it to the exact search.
            if (kc == 0) rscale[r] = in_range ? 1.0f / sc : (mx == 0.0f ? 1.0f : __int_as_float(0x7fc00000));
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

// FP8 centroid operands: per centroid a power-of-two scale (fp8_scale of its
// largest magnitude), the e4m3 codes of c * scale in rows of kp8 bytes (zeros
// past d), and w[j] = -2 / scale (exact), 0 for the padding up to kp. A centroid
// whose largest magnitude is outside [kFp8MinMag, kFp8MaxMag] (and not zero) gets
// w = 0 and scoring norm nf8[j] = -3e38: its approximate score is below every
// other, so it can only be a row's first candidate, which the certification
// re-scores exactly (two such columns leave no margin: refine). nf8 holds the
// reference norms otherwise. One warp per centroid.
__global__ void k_prep_fp8(const float* __restrict__ c, int k, int d, int kp8, int kp, uint8_t* __restrict__ c8,
                           float* __restrict__ w, float* __restrict__ nf8) {
    const int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (j >= kp) return;
    if (j >= k) {
        if (lane == 0) w[j] = 0.0f;
        return;
    }
    const float* cj = c + (size_t)j * d;
    float mx = 0.0f;
    for (int i = lane; i < d; i += 32) mx = fmaxf(mx, fabsf(cj[i]));
    for (int o = 16; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    bool in_range;
    const float sc = fp8_scale(mx, &in_range);
    for (int i = 2 * lane; i < kp8; i += 64) {
        const float a = i < d ? cj[i] * sc : 0.0f, b = i + 1 < d ? cj[i + 1] * sc : 0.0f;
        *reinterpret_cast<uint16_t*>(c8 + (size_t)j * kp8 + i) = (uint16_t)fp8x2(a, b);
    }
    if (lane == 0) {
        w[j] = in_range ? -2.0f / sc : 0.0f;
        if (!in_range && mx != 0.0f) nf8[j] = -3.0e38f;
    }
}

// The bias on the FP8 scoring norms (set_bias adds it to the reference norms;
// a -3e38 entry stays far below every real score).
__global__ void k_add_bias_f8(float* __restrict__ nf8, const float* __restrict__ bias, int k) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < k) nf8[j] = __fadd_rn(nf8[j], bias[j]);
}

#define EMB_TMEM_LD16(taddr, r)                                                                                  \
    asm volatile(                                                                                                \
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];" \
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),      \
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])  \
        : "r"(taddr))

EMB_DEV void tc_regs_ready16(uint32_t (&v)[16]) {
#pragma unroll
    for (int j = 0; j < 16; j++) asm volatile("" : "+r"(v[j]));
}

// FP8 (e4m3 x e4m3 -> f32) instruction descriptor, both operands K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_e4m3(int M, int N) {
    return (1u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

EMB_DEV void mma_e4m3(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n}\n"
        ::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// Norms inside the contraction: row j of `out` (16 BF16) holds the three BF16
// parts of h = norms[j] / 2 (p1 = bf16(h), p2 = bf16(h - p1), p3 = bf16(h - p1 - p2);
// both differences are exact in f32 and p3 is exact in BF16, so p1 + p2 + p3 = h
// for every h in the normal range), then zeros. A non-finite h keeps p1 = h and
// zeros after it, so the MMA sums the same +-inf or NaN the epilogue's
// norm - 2 acc would give. Rows up to kp (whole tiles): the padding's 3e38 too.
__global__ void k_prep_nrm16(const float* __restrict__ norms, int kp, __nv_bfloat16* __restrict__ out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= kp) return;
    const float h = 0.5f * norms[j];
    const __nv_bfloat16 p1 = __float2bfloat16_rn(h);
    __nv_bfloat16 p2 = __float2bfloat16_rn(0.0f), p3 = p2;
    if (isfinite(h)) {
        const float r1 = h - __bfloat162float(p1);
        p2 = __float2bfloat16_rn(r1);
        p3 = __float2bfloat16_rn(r1 - __bfloat162float(p2));
    }
    uint4* o = reinterpret_cast<uint4*>(out + (size_t)j * 16);
    o[0] = make_uint4((uint32_t)__bfloat16_as_ushort(p1) | ((uint32_t)__bfloat16_as_ushort(p2) << 16),
                      (uint32_t)__bfloat16_as_ushort(p3), 0u, 0u);
    o[1] = make_uint4(0u, 0u, 0u, 0u);
}

// Scores of 16 accumulator columns (in place): s = norm - 2 acc (BF16), or
// s = norm + (acc r) w (FP8: acc r undoes the row's power-of-two scale exactly,
// w = -2 / the centroid's scale), one rounding each.
// Paired f32 operations (fma.rn.f32x2 / mul.rn.f32x2: two IEEE roundings), with
// the register pairs left to the compiler.
template <bool FP8>
EMB_DEV void tc_scores16(uint32_t (&v)[16], const float* __restrict__ nrm, const float* __restrict__ wcol, float rs,
                         float (&s)[16]) {
    const float2 m2 = make_float2(-2.0f, -2.0f), r2 = make_float2(rs, rs);
#pragma unroll
    for (int j = 0; j < 16; j += 4) {
        const float4 n4 = *reinterpret_cast<const float4*>(nrm + j);
        const float2 a01 = make_float2(__uint_as_float(v[j]), __uint_as_float(v[j + 1]));
        const float2 a23 = make_float2(__uint_as_float(v[j + 2]), __uint_as_float(v[j + 3]));
        float2 s01, s23;
        if (FP8) {
            const float4 w4 = *reinterpret_cast<const float4*>(wcol + j);
            s01 = __ffma2_rn(__fmul2_rn(a01, r2), make_float2(w4.x, w4.y), make_float2(n4.x, n4.y));
            s23 = __ffma2_rn(__fmul2_rn(a23, r2), make_float2(w4.z, w4.w), make_float2(n4.z, n4.w));
        } else {
            s01 = __ffma2_rn(a01, m2, make_float2(n4.x, n4.y));
            s23 = __ffma2_rn(a23, m2, make_float2(n4.z, n4.w));
        }
        s[j] = s01.x;
        s[j + 1] = s01.y;
        s[j + 2] = s23.x;
        s[j + 3] = s23.y;
    }
}

// Smallest of 16 scores (NaN-ignoring).
EMB_DEV float tc_min16s(const float (&s)[16]) {
    const float a = min3f(s[0], s[1], s[2]), b = min3f(s[3], s[4], s[5]), c = min3f(s[6], s[7], s[8]);
    const float d = min3f(s[9], s[10], s[11]), e = min3f(s[12], s[13], s[14]);
    return fminf(min3f(a, b, c), min3f(d, e, s[15]));
}

// Two smallest keys of 16 scores: each score's 5 low mantissa bits replaced by
// its column jb + j (jb a multiple of 16 within a 32-column chunk; a relative
// change below 2^-18, which the error bound covers), so min/max carry the column.
EMB_DEV void tc_top2_16s(const float (&s)[16], uint32_t jb, float& k1, float& k2) {
    float lo[8], hi[8];
#pragma unroll
    for (int q = 0; q < 8; q++) {
        const float a = __uint_as_float((__float_as_uint(s[2 * q]) & ~31u) | (jb + 2 * q));
        const float b = __uint_as_float((__float_as_uint(s[2 * q + 1]) & ~31u) | (jb + 2 * q + 1));
        lo[q] = fminf(a, b);
        hi[q] = fmaxf(a, b);
    }
#pragma unroll
    for (int w = 4; w >= 1; w >>= 1) {
#pragma unroll
        for (int q = 0; q < w; q++) {
            const float a1 = lo[q], a2 = hi[q], b1 = lo[q + w], b2 = hi[q + w];
            lo[q] = fminf(a1, b1);
            hi[q] = min3f(fmaxf(a1, b1), a2, b2);
        }
    }
    k1 = lo[0];
    k2 = hi[0];
}

// The per-row state of one epilogue warp (a quarter of each tile's columns).
// s1 is the key of column i1; s2 lower-bounds the approximate score of every
// other column the warp has scored. s2 < s1 is allowed: a half-chunk whose
// smallest score cannot be the row's best (another quarter already holds a
// smaller key) only lowers s2 and costs one min, and the keyed tournament that
// tracks columns runs only where a new best is possible.
struct TcBest {
    float s1, s2;
    uint32_t i1;
};

// Persistent fused search. Grid: one CTA per SM (at most the number of work
// items). Work item w = (row tile w / nsplit, column split w % nsplit); CTA b takes
// items b, b + gridDim.x, ... A split walks centroid tiles split, split + nsplit, ...
//   warp 0      TMA producer of the centroid stages (and each tile's norms)
//   warp 1      TMEM allocation; tcgen05.mma issue (one thread)
//   warps 2-3   row loaders: the next work item's row tile into the other buffer
//               (BF16 hi/lo split or e4m3 with a per-row scale)
//   warps 4-19  epilogue, four warps per TMEM lane quarter, 64 columns of each
//               256-column tile per warp: all 64 loaded (four 16-column loads,
//               one wait), the accumulator released, then the 64 scored
// COLLECT = false: per-row (best key, column, lower bound of the rest) to part_s/part_i.
// COLLECT = true : every centroid with approximate score <= theta[row] is appended
//                  to cand[row][*] (cand_count[row] counts all, capped storage).
// Certification of one work item's 128 rows by the two row-loader warps, 16 rows
// at a time with four threads per row (k_certify16v's decisions, so every value
// has the same bits). fin[r]: the row's merged (best key, column, bound of the
// rest) as scores. valid = false (the item's results never completed: the CTA
// gave up): every row is listed for the exhaustive search instead. valid must
// be the same across each warp.
EMB_DEV void tc_fused_certify(const TcParams& p, const float* __restrict__ x, const uint32_t* __restrict__ fin,
                              int row0, int m, bool valid) {
    const int lt = (int)threadIdx.x - 32 * (kTcEpi0 - kTcLoadWarps);  // 0 .. 63
    const int q = lt & 3, lane = (int)threadIdx.x & 31;
    const int d = p.d, k = p.k;
    for (int r0 = 0; r0 < kTcBM; r0 += 8 * kTcLoadWarps) {
        const int r = r0 + (lt >> 2);
        const int row = row0 + r;
        const bool live = row < m;
        bool ok = false, redo = false;
        float theta = __int_as_float(0x7fc00000);
        if (valid) {
            const int rr = live ? row : m - 1;  // dead rows mirror a live one and write nothing
            Top2 t;
            t.init();
            if (live) {
                const uint32_t* e = fin + r * 4;
                t.push(__uint_as_float(e[0]), e[1]);
                t.push(__uint_as_float(e[2]), e[1]);
            }
            const uint32_t j1 = t.i1 < (uint32_t)k ? t.i1 : 0u;
            const float* xr = x + tc_src_row(p, rr) * (size_t)d;
            const float* c1 = p.cx + (size_t)j1 * d;
            float sq[4] = {0.0f, 0.0f, 0.0f, 0.0f}, p1[4] = {0.0f, 0.0f, 0.0f, 0.0f}, rs = 0.0f;
            for (int i = 4 * q; i < d; i += 16) {
                const float4 xv = *reinterpret_cast<const float4*>(xr + i);
                const float4 u = *reinterpret_cast<const float4*>(c1 + i);
                const float xs[4] = {xv.x, xv.y, xv.z, xv.w}, us[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    sq[j] = __fadd_rn(sq[j], __fmul_rn(xs[j], xs[j]));
                    p1[j] = __fmaf_rn(xs[j], us[j], p1[j]);
                    rs = bf16_resid_sq(xs[j], rs);
                }
            }
            rs = __fadd_ru(rs, __shfl_xor_sync(kFull, rs, 2));
            rs = __fadd_ru(rs, __shfl_xor_sync(kFull, rs, 1));
#pragma unroll
            for (int j = 0; j < 4; j++) p1[j] = __fadd_rn(p1[j], __shfl_xor_sync(kFull, p1[j], 2));
#pragma unroll
            for (int j = 0; j < 4; j++) p1[j] = __fadd_rn(p1[j], __shfl_xor_sync(kFull, p1[j], 1));
            const float a1 = __fadd_rn(__fadd_rn(p1[0], p1[2]), __fadd_rn(p1[1], p1[3]));
            float xn = -0.0f;
            const int base = lane & ~3;
#pragma unroll
            for (int qq = 0; qq < 4; qq++)
#pragma unroll
                for (int j = 0; j < 4; j++) xn = __fadd_rn(xn, __shfl_sync(kFull, sq[j], base + qq));
            if (live && q == 0) {
                // The second candidate is the first's column again (the written
                // pair), so one exact dot product serves both.
                const int no_abort = 0;
                ok = certify_decide(row, t, j1, j1, a1, a1, xn, k, p.norms, p.bounds, p.ka, p.kb, p.labels, p.dist,
                                    &no_abort, p.ka2, p.kb2, nullptr, &theta, p.kr,
                                    __fmul_ru(__fsqrt_ru(rs), 1.0000005f));
                redo = !ok;
            }
        } else {
            redo = live && q == 0;
        }
        certify_tally(ok, redo, row, theta, p.cert_count, p.redo_count, p.redo_rows, p.redo_theta);
    }
}

template <typename T, bool COLLECT, bool FP8, bool NM = false>
__global__ void __launch_bounds__(kTcPThreads, 1)
k_assign_tc(const T* __restrict__ x, const __grid_constant__ CUtensorMap map_hi,
            const __grid_constant__ CUtensorMap map_lo, const TcParams p) {
    static_assert(!NM || (!COLLECT && !FP8), "norms in the contraction: single-term BF16 fast search only");
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = smem_align1024(smem_raw);
    const TcLayout L = tc_layout(p.kpad, p.nterms, FP8, NM);
    const int S = L.stages, NB = L.nbuf;
    uint64_t* full = (uint64_t*)(smem + L.bars);          // [kTcMaxStages]
    uint64_t* empty = full + kTcMaxStages;                // [kTcMaxStages]
    uint64_t* acc_full = empty + kTcMaxStages;            // [2]
    uint64_t* acc_empty = acc_full + 2;                   // [2]
    uint64_t* norms_full = acc_empty + 2;                 // [kTcNormSlots]
    uint64_t* a_full = norms_full + kTcNormSlots;         // [2] row tile loaded
    uint64_t* a_empty = a_full + 2;                       // [2] every MMA reading the row buffer completed
    uint64_t* rs_full = a_empty + 2;                      // [kTcRowScaleSlots] FP8 row scales written
    uint64_t* mma_done = rs_full + kTcRowScaleSlots;      // every issued MMA completed (teardown)
    uint64_t* stall_bar = mma_done + 1;                   // never completed (abort-path test)
    uint64_t* nm_full = stall_bar + 1;                    // NM: [kTcNmSlots] norm slice loaded
    uint64_t* nm_empty = nm_full + kTcNmSlots;            // NM: [kTcNmSlots] the MMA reading it completed
    uint64_t* fin_full = nm_empty + kTcNmSlots;           // NM: an item's merged top-2 written (fused certify)
    uint64_t* fin_empty = fin_full + 1;                   // NM: the row loaders are done with it
    // 30 barriers: 240 of the 256 bytes; with NM 36 barriers: 288 of 512 bytes.
    uint32_t* tmem_slot = (uint32_t*)(NM ? fin_empty + 1 : stall_bar + 1);
    uint32_t* fin = (uint32_t*)(smem + L.fin);            // NM: [128 rows][4]
    volatile int* abort_flag = (volatile int*)(tmem_slot + 1);
    float* norms_s = (float*)(smem + L.norms);
    float* rscale_s = (float*)(smem + L.rscale);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int m = p.m;
    if (COLLECT && p.m_dev) {
        // Row count known only on the device (graph-captured refine).
        const int md = (int)*p.m_dev;
        m = md < m ? md : m;
    }
    const int nsplit = p.nsplit;
    const int nitems = ((m + kTcBM - 1) / kTcBM) * nsplit;
    if ((int)blockIdx.x >= nitems) return;  // no work: the whole CTA leaves before any setup
    const int my_items = (nitems - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
    const int ntiles_all = (p.k + kTcBN - 1) / kTcBN;
    auto item_of = [&](int i) { return (int)blockIdx.x + i * (int)gridDim.x; };
    auto tiles_of = [&](int split) { return split < ntiles_all ? (ntiles_all - split + nsplit - 1) / nsplit : 0; };
    const int natoms = FP8 ? p.kpad / 128 : p.kpad / 64;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kTcMaxStages; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], kTcEpiWarps);  // one arrival per epilogue warp
            mbar_init(&a_full[b], kTcLoadWarps * 32);
            mbar_init(&a_empty[b], 1);
        }
        for (int i = 0; i < kTcNormSlots; i++) mbar_init(&norms_full[i], 1);
        for (int i = 0; i < kTcRowScaleSlots; i++) mbar_init(&rs_full[i], kTcLoadWarps * 32);
        mbar_init(mma_done, 1);
        mbar_init(stall_bar, 1);
        if (NM) {
            for (int i = 0; i < kTcNmSlots; i++) {
                mbar_init(&nm_full[i], 1);
                mbar_init(&nm_empty[i], 1);
            }
            mbar_init(fin_full, 1);
            mbar_init(fin_empty, kTcLoadWarps * 32);
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) tmem_alloc(tmem_slot, kTcTmemCols);
    {  // published best keys start at +inf
        float* pub = (float*)(smem + L.pub);
        for (int i = threadIdx.x; i < 4 * kTcBM; i += blockDim.x) pub[i] = INFINITY;
    }
    if (NM) {
        // The constant row operand of the norm MMA: every row [1, 1, 1, 0, 0, 0, 0, 0]
        // in both 16-byte halves (BF16 one = 0x3F80), so whichever half the 32-byte
        // swizzle pairs with the norm slice's parts, the product is p1 + p2 + p3.
        uint4* nc = reinterpret_cast<uint4*>(smem + L.nconst);
        for (int i = threadIdx.x; i < (int)(kTcNmConstBytes / 16); i += blockDim.x)
            nc[i] = make_uint4(0x3F803F80u, 0x00003F80u, 0u, 0u);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // visible to the tensor cores
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            // ---- TMA producer: unit u = (item, tile, K atom) into stage u % S
            int u = 0, tg = 0, nissued = 0;  // units issued, tiles begun, tiles whose norms were issued
            bool ok = true;
            for (int i = 0; i < my_items && ok; i++) {
                const int w = item_of(i), split = w % nsplit;
                const int nt = tiles_of(split);
                for (int t = 0; t < nt && ok; t++, tg++) {
                    const int col = (split + t * nsplit) * kTcBN;
                    for (int a = 0; a < natoms; a++, u++) {
                        const int s = u % S;
                        if (u >= S && !mbar_wait(&empty[s], ((uint32_t)(u / S) & 1u) ^ 1u, abort_flag, kTcCtlSleepNs)) {
                            ok = false;
                            break;
                        }
                        // NM: the tile's norm slice goes into slot tg % kTcNmSlots once the
                        // MMA of tile tg - kTcNmSlots has read it (waited before any copy
                        // of this unit is issued, so an abort here leaves none untracked).
                        if (NM && a == 0 && tg >= kTcNmSlots &&
                            !mbar_wait(&nm_empty[tg % kTcNmSlots], ((uint32_t)(tg / kTcNmSlots) & 1u) ^ 1u, abort_flag,
                                       kTcCtlSleepNs)) {
                            ok = false;
                            break;
                        }
                        uint8_t* stage = smem + L.b0 + s * L.stage_bytes;
                        mbar_expect_tx(&full[s], L.stage_bytes);
                        tma_load_2d(stage, &map_hi, &full[s], a * (FP8 ? 128 : 64), col);
                        if (!FP8 && p.nterms > 1) tma_load_2d(stage + L.term_bytes, &map_lo, &full[s], a * 64, col);
                        if (a == 0) {
                            if (NM) {
                                const int ns = tg % kTcNmSlots;
                                mbar_expect_tx(&nm_full[ns], kTcNmSlotBytes);
                                bulk_load(smem + L.norms + ns * kTcNmSlotBytes, p.nrm16 + (size_t)col * 16,
                                          kTcNmSlotBytes, &nm_full[ns]);
                            } else {
                                const int ns = tg % kTcNormSlots;
                                float* dst = norms_s + ns * (L.nrm_slot_bytes / 4);
                                mbar_expect_tx(&norms_full[ns], L.nrm_slot_bytes);
                                bulk_load(dst, p.norms + (size_t)col, kTcBN * 4, &norms_full[ns]);
                                if (FP8) bulk_load(dst + kTcBN, p.wf8 + (size_t)col, kTcBN * 4, &norms_full[ns]);
                            }
                            nissued = tg + 1;
                        }
                    }
                }
            }
            // After an abort, let the copies still in flight land before the CTA
            // exits; bounded like every wait.
            if (*abort_flag) {
                for (int v = u > S ? u - S : 0; v < u; v++) mbar_drain(&full[v % S], (uint32_t)(v / S) & 1u);
                const int nslots = NM ? kTcNmSlots : kTcNormSlots;
                uint64_t* nbar = NM ? nm_full : norms_full;
                for (int t = nissued > nslots ? nissued - nslots : 0; t < nissued; t++)
                    mbar_drain(&nbar[t % nslots], (uint32_t)(t / nslots) & 1u);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // ---- MMA issuer: per unit, nterms x 4 MMAs of M=128 N=256 (K=16 BF16 / K=32 e4m3)
            const uint32_t idesc = FP8 ? idesc_e4m3(kTcBM, kTcBN) : idesc_bf16(kTcBM, kTcBN);
            const uint32_t a_atom = (kTcBM * 128) >> 4;  // descriptor units (16 B) per A atom
            int u = 0, tg = 0;
            bool ok = true;
            for (int i = 0; i < my_items && ok; i++) {
                const int w = item_of(i), split = w % nsplit;
                const int nt = tiles_of(split);
                const int ab = i % NB;
                if (!mbar_wait(&a_full[ab], (uint32_t)(i / NB) & 1u, abort_flag, kTcCtlSleepNs)) break;
                tc_fence_after();
                const uint64_t a_hi0 = sw128_desc(smem_u32(smem + ab * L.a_buf));
                const uint64_t a_lo0 = sw128_desc(smem_u32(smem + ab * L.a_buf + L.a_lo));
                for (int t = 0; t < nt && ok; t++, tg++) {
                    const int b = tg & 1;
                    if (!mbar_wait(&acc_empty[b], ((uint32_t)(tg >> 1) & 1u) ^ 1u, abort_flag, kTcCtlSleepNs) ||
                        (NM && !mbar_wait(&nm_full[tg % kTcNmSlots], (uint32_t)(tg / kTcNmSlots) & 1u, abort_flag,
                                          kTcCtlSleepNs))) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t d_tmem = tmem_base + (uint32_t)(b * kTcBN);
                    // NM: the accumulator starts as the half-norms (one K = 16 MMA).
                    if (NM)
                        mma_bf16(d_tmem, sw32_desc(smem_u32(smem + L.nconst)),
                                 sw32_desc(smem_u32(smem + L.norms + (tg % kTcNmSlots) * kTcNmSlotBytes)), idesc, 0u);
                    for (int a = 0; a < natoms; a++, u++) {
                        const int s = u % S;
                        if (!mbar_wait(&full[s], (uint32_t)(u / S) & 1u, abort_flag, kTcCtlSleepNs)) {
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                        const uint64_t bh = sw128_desc(smem_u32(smem + L.b0 + s * L.stage_bytes));
                        const uint64_t bl = bh + (L.term_bytes >> 4);
                        const uint64_t ah = a_hi0 + (uint64_t)(a * a_atom), al = a_lo0 + (uint64_t)(a * a_atom);
#pragma unroll
                        for (int kk = 0; kk < 4; kk++) {  // 32 bytes of K per MMA = 2 descriptor units
                            const uint32_t acc = (NM || a > 0 || kk > 0) ? 1u : 0u;
                            if (FP8) mma_e4m3(d_tmem, ah + 2 * kk, bh + 2 * kk, idesc, acc);
                            else mma_bf16(d_tmem, ah + 2 * kk, bh + 2 * kk, idesc, acc);
                        }
                        if (!FP8 && p.nterms > 1) {
#pragma unroll
                            for (int kk = 0; kk < 4; kk++) mma_bf16(d_tmem, ah + 2 * kk, bl + 2 * kk, idesc, 1u);
                        }
                        if (!FP8 && p.nterms > 2) {
#pragma unroll
                            for (int kk = 0; kk < 4; kk++) mma_bf16(d_tmem, al + 2 * kk, bh + 2 * kk, idesc, 1u);
                        }
                        mma_commit(&empty[s]);
                    }
                    if (ok) {
                        if (NM) mma_commit(&nm_empty[tg % kTcNmSlots]);
                        mma_commit(&acc_full[b]);
                    }
                }
                if (ok) mma_commit(&a_empty[ab]);  // the row buffer is free once these MMAs complete
            }
            // Normally every MMA has completed by now; after an abort some may still
            // run. Either way none may outlive the TMEM allocation or the stages it reads.
            mma_drain(mma_done);
        }
    } else if (warp < kTcEpi0) {
        // ---- row loaders: item i's row tile into buffer i % NB once the MMAs of
        // item i - NB have completed
        const int ltid = threadIdx.x - 64;
        // Fused certification (NM, TcParams::fuse): after loading item i's rows the
        // loaders certify item i - 1 (its merged top-2 is complete once the
        // epilogue finishes that item, while item i is searched), and the last item
        // after the loop. After an abort they load nothing more, but still list the
        // rows of every item whose results never completed for the exact search.
        // Once a wait has failed, no later item counts as complete either (its
        // barrier phases no longer line up with the items).
        const bool fuse = NM && p.fuse;
        bool fin_ok = true;
        auto certify_item = [&](int j) {
            bool valid = fin_ok && mbar_wait(fin_full, (uint32_t)(j & 1), abort_flag, kTcCtlSleepNs);
            valid = __all_sync(0xffffffffu, valid);
            fin_ok = valid;
            if constexpr (std::is_same<T, float>::value)
                tc_fused_certify(p, x, fin, (item_of(j) / nsplit) * kTcBM, m, valid);
            mbar_arrive(fin_empty);
        };
        bool loading = true;
        for (int i = 0; i < my_items; i++) {
            const int w = item_of(i);
            const int ab = i % NB;
            if (loading && !mbar_wait(&a_empty[ab], ((uint32_t)(i / NB) & 1u) ^ 1u, abort_flag, kTcCtlSleepNs))
                loading = false;
            if (loading) {
                uint8_t* a = smem + ab * L.a_buf;
                if (FP8)
                    tc_load_rows_fp8(a, rscale_s + (i % kTcRowScaleSlots) * kTcBM, x, p, (w / nsplit) * kTcBM, m,
                                     ltid);
                else
                    tc_load_rows(a, a + L.a_lo, x, p, (w / nsplit) * kTcBM, m, ltid, kTcLoadWarps * 32, NM);
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // visible to the tensor cores
                mbar_arrive(&a_full[ab]);
                // The epilogue reads slot i % 4 of the row scales at item i. The loader
                // cannot be four items ahead of it: item i + 4 needs the MMAs of item
                // i + 2 done, which need the epilogue to have released tiles of item i.
                if (FP8) mbar_arrive(&rs_full[i % kTcRowScaleSlots]);
            } else if (!fuse) {
                break;
            }
            if (fuse && i > 0) certify_item(i - 1);
        }
        if (fuse && my_items > 0) certify_item(my_items - 1);
    } else {
        // ---- epilogue: warps 4..19. Thread = row (TMEM lane); warp w takes the
        // 64-column quarter (w - 4) / 4 of every tile, as four 16-column halves.
        const int q = warp & 3;  // TMEM lane quarter this warp may access
        const int cq = (warp - kTcEpi0) >> 2;
        const int r = q * 32 + lane;
        float* pub = (float*)(smem + L.pub);
        uint32_t* mg = (uint32_t*)(smem + L.merge);
        int tg = 0;
        bool ok = true;
        for (int i = 0; i < my_items; i++) {
            const int w = item_of(i), split = w % nsplit;
            const int nt = tiles_of(split);
            const int row = (w / nsplit) * kTcBM + r;
            TcBest best{INFINITY, INFINITY, 0xffffffffu};
            float theta = 0.0f;
            if (COLLECT) theta = row < m ? p.theta[row] : __int_as_float(0x7fc00000);
            float rs = 1.0f;
            for (int t = 0; t < nt && ok; t++, tg++) {
                const int b = tg & 1;
                if (!mbar_wait(&acc_full[b], (uint32_t)(tg >> 1) & 1u, abort_flag, 20000) ||
                    (!NM && !mbar_wait(&norms_full[tg % kTcNormSlots], (uint32_t)(tg / kTcNormSlots) & 1u, abort_flag)) ||
                    (p.stall_ns && t == p.stall_tile && warp == kTcEpi0 &&
                     !mbar_wait(stall_bar, 0, abort_flag, 0, p.stall_ns))) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                if (FP8 && t == 0) {
                    if (!mbar_wait(&rs_full[i % kTcRowScaleSlots], (uint32_t)(i / kTcRowScaleSlots) & 1u, abort_flag)) {
                        ok = false;
                        break;
                    }
                    rs = rscale_s[(i % kTcRowScaleSlots) * kTcBM + r];
                }
                const float* nrm = norms_s + (tg % kTcNormSlots) * (L.nrm_slot_bytes / 4) + cq * 64;
                const uint32_t taddr = tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * kTcBN + cq * 64);
                const int cb = (split + t * nsplit) * kTcBN + cq * 64;
                // The row's best key over all four quarters so far (read once per
                // tile; keys only decrease, so a stale value is still an upper
                // bound), raised by 2^-17 relative to cover a key's column bits.
                float g1 = fminf(fminf(pub[r], pub[kTcBM + r]), fminf(pub[2 * kTcBM + r], pub[3 * kTcBM + r]));
                g1 = fmaf(fabsf(g1), 0x1p-17f, g1);
                // The warp's 64 columns into registers (four 16-column loads, one
                // wait), then the accumulator is released before they are scored.
                uint32_t v4[4][16];
                EMB_TMEM_LD16(taddr, v4[0]);
                EMB_TMEM_LD16(taddr + 16, v4[1]);
                EMB_TMEM_LD16(taddr + 32, v4[2]);
                EMB_TMEM_LD16(taddr + 48, v4[3]);
                tmem_wait_ld();
#pragma unroll
                for (int h = 0; h < 4; h++) tc_regs_ready16(v4[h]);
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&acc_empty[b]);
                float sc4[4][16], mnh[4];
#pragma unroll
                for (int h = 0; h < 4; h++) {
                    if constexpr (NM) {
                        // The accumulator is the half-score: keys and bounds stay in those
                        // units (every comparison is scale-free) until they are written.
#pragma unroll
                        for (int j = 0; j < 16; j++) sc4[h][j] = __uint_as_float(v4[h][j]);
                    } else {
                        tc_scores16<FP8>(v4[h], nrm + h * 16, nrm + kTcBN + h * 16, rs, sc4[h]);
                    }
                    mnh[h] = tc_min16s(sc4[h]);
                }
                if (!COLLECT) {
                    // One vote for the tile: when no row of the warp has a half whose
                    // minimum is below the bound at the tile's start, every half only
                    // lowers s2 (what the per-half rule below does in that case too).
                    const float thr = fminf(g1, best.s1);
                    const bool low = (mnh[0] < thr) | (mnh[1] < thr) | (mnh[2] < thr) | (mnh[3] < thr);
                    if (!__any_sync(0xffffffffu, low)) {
                        best.s2 = fminf(best.s2, fminf(fminf(mnh[0], mnh[1]), fminf(mnh[2], mnh[3])));
                    } else {
#pragma unroll
                        for (int h = 0; h < 4; h++) {
                            if (__any_sync(0xffffffffu, mnh[h] < fminf(g1, best.s1))) {
                                float k1, k2;
                                const uint32_t jb = (uint32_t)((h & 1) * 16);
                                tc_top2_16s(sc4[h], jb, k1, k2);
                                const uint32_t j1 = (uint32_t)(cb + (h >> 1) * 32) + (__float_as_uint(k1) & 31u);
                                if (k1 < best.s1) {
                                    best.s2 = min3f(best.s2, best.s1, k2);
                                    best.s1 = k1;
                                    best.i1 = j1;
                                } else {
                                    best.s2 = fminf(best.s2, k1);
                                }
                            } else {
                                best.s2 = fminf(best.s2, mnh[h]);
                            }
                        }
                    }
                } else {
#pragma unroll
                    for (int h = 0; h < 4; h++) {
                        if (mnh[h] <= theta) {
#pragma unroll
                            for (int j = 0; j < 16; j++) {
                                const int col = cb + h * 16 + j;
                                if (sc4[h][j] <= theta && col < p.k) {
                                    const uint32_t slot = atomicAdd(&p.cand_count[row], 1u);
                                    if (slot < (uint32_t)p.cand_cap)
                                        p.cand[(size_t)row * p.cand_cap + slot] = (uint32_t)col;
                                }
                            }
                        }
                    }
                }
                if (!COLLECT) pub[cq * kTcBM + r] = best.s1;  // the quarter's best key, for the other quarters
            }
            // After an abort the warp still walks every remaining item and reaches
            // both named barriers of each (bar.sync cannot time out), without waits.
            if (!COLLECT) {
                // Merge the four column quarters of each row: the best key over all,
                // and below it the smallest of everything else (the other quarters'
                // best keys and every quarter's bound of the rest).
                if (cq > 0) {
                    uint32_t* e = mg + ((cq - 1) * kTcBM + r) * 4;
                    e[0] = __float_as_uint(best.s1);
                    e[1] = best.i1;
                    e[2] = __float_as_uint(best.s2);
                }
                asm volatile("bar.sync 1, %0;" ::"n"(kTcEpiWarps * 32) : "memory");
                if (cq == 0 && row < m) {
                    float s1 = best.s1, s2 = best.s2;
                    uint32_t i1 = best.i1;
#pragma unroll
                    for (int o = 0; o < 3; o++) {
                        const uint32_t* e = mg + (o * kTcBM + r) * 4;
                        const float os1 = __uint_as_float(e[0]), os2 = __uint_as_float(e[2]);
                        const uint32_t oi1 = e[1];
                        if (lex_less(os1, oi1, s1, i1)) {
                            s2 = min3f(s2, s1, os2);
                            s1 = os1;
                            i1 = oi1;
                        } else {
                            s2 = min3f(s2, os1, os2);
                        }
                    }
                    // Written as a top-2 pair whose second entry repeats the column: a
                    // certified row always takes the first candidate, and s2 bounds
                    // every other column's approximate score from below. s2 >= s1
                    // holds by construction (every value folded into s2 is at least
                    // the final best key); were it ever violated, raising s2 to s1
                    // leaves no margin, so the row goes to the refine pass.
                    const float unit = NM ? 2.0f : 1.0f;  // NM: half-scores back to scores (exact)
                    if (NM && p.fuse) {
                        // For the row loaders' certification, once they are done with
                        // the previous item's (never after a wait that gave up).
                        if (i == 0 || mbar_wait(fin_empty, (uint32_t)((i - 1) & 1), abort_flag, kTcCtlSleepNs)) {
                            uint32_t* e = fin + r * 4;
                            e[0] = __float_as_uint(unit * s1);
                            e[1] = i1;
                            e[2] = __float_as_uint(unit * fmaxf(s2, s1));
                        }
                    } else {
                        const size_t oo = ((size_t)split * p.m + row) * 2;
                        p.part_s[oo] = unit * s1;
                        p.part_i[oo] = i1;
                        p.part_s[oo + 1] = unit * fmaxf(s2, s1);
                        p.part_i[oo + 1] = i1;
                    }
                }
                pub[cq * kTcBM + r] = INFINITY;  // the next item starts afresh
                asm volatile("bar.sync 1, %0;" ::"n"(kTcEpiWarps * 32) : "memory");
                // The item's results are complete unless some role gave up (every failed
                // wait raises the abort flag): hand them to the row loaders.
                if (NM && p.fuse && warp == kTcEpi0 && lane == 0 && !*abort_flag) mbar_arrive(fin_full);
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
