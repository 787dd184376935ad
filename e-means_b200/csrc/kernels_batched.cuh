// Batched e-means training in lockstep (emb200_train_batched): many independent
// instances of train() (src/lib.rs:348-491) over row ranges of the resident rows,
// with uneven n and k, advance together one global step at a time. Instance i
// takes part in global step s while s < its own step count; every kernel of a
// step covers all instances, reads the step's parameters from device tables
// (batch rows, epoch, last-pass flag, alpha) and leaves at once for the
// instances that are done, so one captured step replays for the whole run.
//
// A step: centroid norms and bounds -> search (a persistent kernel over a queue
// of (instance, row tile, column split) work items, FP32 SIMT with a per-row
// top-2) -> certification and exact re-search in the reference's rounding ->
// label histogram, scan, scatter -> per-cluster sums in row order -> last-pass
// labels -> batch objective -> EMA step -> revival every fifth step -> step end.
// Each per-instance computation is the single-instance one (the same device
// functions, the same operation order), so every instance's result equals its
// own train() call bit for bit.
#pragma once
#include "common.cuh"
#include "kernels_exact.cuh"
#include "kernels_update.cuh"

namespace emb {

// One instance. Offsets index the concatenated device arrays of all instances.
struct BInst {
    unsigned long long row0;     // first resident row
    unsigned long long n_off;    // last-pass labels (sum of n)
    unsigned long long ord_off;  // row orders of every epoch (sum of n * epochs)
    unsigned long long c_off;    // centroids, batch sums, pass sums (sum of k * d)
    unsigned long long g_off;    // revival stream (sum of events * k)
    unsigned long long g_cap;    // its length: events * k
    unsigned long long p_off;    // search partials, in top-2 pairs (sum of nsplit * batch)
    uint32_t n, k, batch, steps;
    uint32_t k_off;              // per-cluster arrays (sum of k)
    uint32_t b_off;              // per-batch-row arrays (sum of batch)
    uint32_t step_off;           // step table and alphas (sum of steps)
    uint32_t obj_off;            // per-epoch objective (sum of epochs)
    uint32_t kp2_off;            // revival sort scratch (sum of next_pow2(k))
    uint32_t nsplit;             // column splits of the search
    uint32_t item_off;           // first search work item
    float tau;                   // unused threshold (0: no revival)
};

// Instance step: epoch, first row of the batch in the epoch's order, batch rows,
// and whether the epoch is the last pass (src/lib.rs:403-406).
struct BStep {
    uint32_t epoch, b0, bn, last;
};

struct BCtl {
    int gstep;       // global step
    uint32_t qhead;  // search work queue head
    uint32_t redo;   // rows listed for the exhaustive search
    uint32_t redo_total;  // summed over the steps of the call
};

struct BArgs {
    const BInst* inst;
    int count, d, match;
    const BStep* steps;
    const uint32_t* orders;  // instance-local row ids
    const float* alphas;
    BCtl* ctl;
    float* c;
    float* norms;
    Bounds* bounds;
    float* usage;
    float* sums;
    uint32_t* counts;
    uint32_t* offsets;
    uint32_t* slot;
    uint32_t* list;
    uint32_t* scratch;
    uint32_t* blabels;
    float* bdist;
    uint32_t* labels_all;
    unsigned long long* pass_counts;
    float* pass_sums;
    double* pass_sums64;
    double* obj;
    const double* gstream;
    unsigned long long* cursor;
    unsigned long long* nsplits;
    double* keys;
    uint32_t* didx;
    uint32_t* unused;
    float* part_s;
    uint32_t* part_i;
    const uint32_t* item_inst;
    uint32_t total_items;
    uint32_t* redo_list;  // (instance << 24) | batch row
    float ka, kb;
};

// The instance's current step, or false once it is done.
EMB_DEV bool b_active(const BArgs& a, int i, BStep* st) {
    const BInst& I = a.inst[i];
    const int s = a.ctl->gstep;
    if (s >= (int)I.steps) return false;
    *st = a.steps[I.step_off + s];
    return true;
}

// Instance-local row ids of the current batch (src/lib.rs:408, the epoch's order).
EMB_DEV const uint32_t* b_rows(const BArgs& a, const BInst& I, const BStep& st) {
    return a.orders + I.ord_off + (size_t)st.epoch * I.n + st.b0;
}

// Initial centroids (src/lib.rs:374-379): rows init[init_off + j] of each instance.
template <typename T>
__global__ void k_b_gather_init(const T* __restrict__ x, BArgs a, const uint32_t* __restrict__ init,
                                const uint32_t* __restrict__ init_off) {
    const int i = blockIdx.y;
    const BInst& I = a.inst[i];
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (size_t)I.k * a.d) return;
    const size_t j = e / a.d, t = e - j * a.d;
    a.c[I.c_off + e] = to_f32(x[(I.row0 + init[init_off[i] + j]) * a.d + t]);
}

// set_centroids for every active instance: reference norms (src/cpu.rs:84-93) and
// the certification bounds; the batch's cluster counts start at zero.
// Grid (ceil(kmax / 8), count), one warp per centroid.
__global__ void k_b_prep(BArgs a) {
    const int i = blockIdx.y;
    BStep st;
    if (!b_active(a, i, &st)) return;
    const BInst& I = a.inst[i];
    const int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (j >= (int)I.k) return;
    const float* cj = a.c + I.c_off + (size_t)j * a.d;
    const float nrm = warp_sqnorm_ref(cj, a.d, lane);
    float ss = 0.0f;
    for (int t = lane; t < a.d; t += 32) ss = __fmaf_ru(cj[t], cj[t], ss);
    for (int o = 16; o; o >>= 1) ss = __fadd_ru(ss, __shfl_xor_sync(kFull, ss, o));
    if (lane == 0) {
        a.norms[I.k_off + j] = nrm;
        atomic_max_pos(&a.bounds[i].cmax, __fmul_ru(__fsqrt_ru(ss), 1.0000005f));
        atomic_max_pos(&a.bounds[i].nmax, fabsf(nrm));
        a.counts[I.k_off + j] = 0;
    }
}

// Loads EPT consecutive elements of a BM x 16 (or BN x 16) slab for thread t:
// row t / (16 / EPT), columns (t % (16 / EPT)) * EPT .. + EPT, zero outside.
template <typename T, int EPT>
EMB_DEV void b_slab_load(float (&r)[EPT], const T* __restrict__ base, const uint32_t* __restrict__ ids, size_t id0,
                         int row, int nrows, int d, int k0) {
    const int t = threadIdx.x;
    const int rr = row + t / (16 / EPT), col = k0 + (t % (16 / EPT)) * EPT;
#pragma unroll
    for (int q = 0; q < EPT; q++) r[q] = 0.0f;
    if (rr >= nrows) return;
    const T* p = base + (ids ? (id0 + ids[rr]) : (size_t)rr) * (size_t)d + col;
#pragma unroll
    for (int q = 0; q < EPT; q++)
        if (col + q < d) r[q] = to_f32(p[q]);
}

// The search: persistent CTAs take (instance, row tile, column split) items
// from a work queue (one atomic per item) until it is empty. An item is BM
// batch rows against the centroid tiles split, split + nsplit, ... of its
// instance: FP32 FMA tiles in registers (BM/16 x BN/16 per thread), score =
// norm - 2 acc, a running top-2 per row merged over the 16 column threads;
// partials [p_off + (split * batch + row)] as (s1, i1), (s2, i2).
template <typename T, int BM, int BN>
__global__ void __launch_bounds__(256, 1) k_b_search(const T* __restrict__ x, BArgs a) {
    constexpr int BK = 16, TM = BM / 16, TN = BN / 16, EA = BM / 16, EB = BN / 16;
    __shared__ __align__(16) float As[2][BK][BM];
    __shared__ __align__(16) float Bs[2][BK][BN];
    __shared__ uint32_t item_s;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int d = a.d;
    const int nk = (d + BK - 1) / BK;
    for (;;) {
        if (tid == 0) item_s = atomicAdd(&a.ctl->qhead, 1u);
        __syncthreads();
        const uint32_t it = item_s;
        __syncthreads();
        if (it >= a.total_items) break;
        const int i = (int)a.item_inst[it];
        BStep st;
        if (!b_active(a, i, &st)) continue;
        const BInst& I = a.inst[i];
        const uint32_t local = it - I.item_off;
        const int rt = (int)(local / I.nsplit), split = (int)(local % I.nsplit);
        const int row0 = rt * BM;
        if (row0 >= (int)st.bn) continue;
        const uint32_t* ids = b_rows(a, I, st);
        const T* xi = x + I.row0 * (size_t)d;
        const float* ci = a.c + I.c_off;
        const float* ni = a.norms + I.k_off;
        const int k = (int)I.k, m = (int)st.bn;
        const int ntiles = (k + BN - 1) / BN;
        Top2 top[TM];
#pragma unroll
        for (int q = 0; q < TM; q++) top[q].init();
        for (int tile = split; tile < ntiles; tile += (int)I.nsplit) {
            const int col0 = tile * BN;
            float acc[TM][TN];
#pragma unroll
            for (int q = 0; q < TM; q++)
#pragma unroll
                for (int j = 0; j < TN; j++) acc[q][j] = 0.0f;
            float ra[EA], rb[EB];
            b_slab_load<T, EA>(ra, xi, ids, 0, row0, m, d, 0);
            b_slab_load<float, EB>(rb, ci, (const uint32_t*)nullptr, 0, col0, k, d, 0);
            __syncthreads();  // the previous tile's readers are done with buffer 0
            {
                const int r = tid / (16 / EA), kk0 = (tid % (16 / EA)) * EA;
#pragma unroll
                for (int q = 0; q < EA; q++) As[0][kk0 + q][r] = ra[q];
                const int rbn = tid / (16 / EB), kb0 = (tid % (16 / EB)) * EB;
#pragma unroll
                for (int q = 0; q < EB; q++) Bs[0][kb0 + q][rbn] = rb[q];
            }
            __syncthreads();
            for (int kt = 0; kt < nk; kt++) {
                const int buf = kt & 1;
                if (kt + 1 < nk) {
                    b_slab_load<T, EA>(ra, xi, ids, 0, row0, m, d, (kt + 1) * BK);
                    b_slab_load<float, EB>(rb, ci, (const uint32_t*)nullptr, 0, col0, k, d, (kt + 1) * BK);
                }
#pragma unroll
                for (int kk = 0; kk < BK; kk++) {
                    float av[TM], bv[TN];
#pragma unroll
                    for (int q = 0; q < TM / 2; q++) {
                        av[q] = As[buf][kk][ty * (TM / 2) + q];
                        av[TM / 2 + q] = As[buf][kk][BM / 2 + ty * (TM / 2) + q];
                    }
#pragma unroll
                    for (int j = 0; j < TN / 2; j++) {
                        bv[j] = Bs[buf][kk][tx * (TN / 2) + j];
                        bv[TN / 2 + j] = Bs[buf][kk][BN / 2 + tx * (TN / 2) + j];
                    }
#pragma unroll
                    for (int q = 0; q < TM; q++)
#pragma unroll
                        for (int j = 0; j < TN; j++) acc[q][j] = __fmaf_rn(av[q], bv[j], acc[q][j]);
                }
                if (kt + 1 < nk) {
                    const int r = tid / (16 / EA), kk0 = (tid % (16 / EA)) * EA;
#pragma unroll
                    for (int q = 0; q < EA; q++) As[buf ^ 1][kk0 + q][r] = ra[q];
                    const int rbn = tid / (16 / EB), kb0 = (tid % (16 / EB)) * EB;
#pragma unroll
                    for (int q = 0; q < EB; q++) Bs[buf ^ 1][kb0 + q][rbn] = rb[q];
                }
                __syncthreads();
            }
#pragma unroll
            for (int j = 0; j < TN; j++) {
                const int col = col0 + (j < TN / 2 ? tx * (TN / 2) + j : BN / 2 + tx * (TN / 2) + (j - TN / 2));
                if (col < k) {
                    const float nj = ni[col];
#pragma unroll
                    for (int q = 0; q < TM; q++) top[q].push_fast(__fmaf_rn(-2.0f, acc[q][j], nj), (uint32_t)col);
                }
            }
        }
#pragma unroll
        for (int q = 0; q < TM; q++) {
            top[q].merge_shfl_xor(1);
            top[q].merge_shfl_xor(2);
            top[q].merge_shfl_xor(4);
            top[q].merge_shfl_xor(8);
        }
        if (tx == 0) {
#pragma unroll
            for (int q = 0; q < TM; q++) {
                const int row = row0 + (q < TM / 2 ? ty * (TM / 2) + q : BM / 2 + ty * (TM / 2) + (q - TM / 2));
                if (row < m) {
                    const size_t o = (I.p_off + (size_t)split * I.batch + row) * 2;
                    a.part_s[o] = top[q].s1;
                    a.part_i[o] = top[q].i1;
                    a.part_s[o + 1] = top[q].s2;
                    a.part_i[o + 1] = top[q].i2;
                }
            }
        }
    }
}

// The search with the item's row block resident in shared memory (f32 rows,
// d % 4 == 0, d <= kBResMaxD): the BM gathered rows are staged once per item
// (transposed, As[t][row]) and each BN-centroid tile once per tile (the next
// tile's values in registers while the current one is multiplied), so an
// item's rows are read once instead of once per centroid tile and a tile costs
// two block barriers instead of two per 16 dimensions. Scores, the per-row
// top-2 and the partials as k_b_search.
constexpr int kBResMaxD = 128;
template <int BM, int BN>
constexpr size_t b_res_smem() { return (size_t)kBResMaxD * (BM + BN) * sizeof(float); }

template <int BM, int BN>
__global__ void __launch_bounds__(256, 1) k_b_search_res(const float* __restrict__ x, BArgs a) {
    constexpr int TM = BM / 16, TN = BN / 16;
    constexpr int BV = BN * kBResMaxD / 4 / 256;  // float4 per thread of a centroid tile (d = kBResMaxD)
    extern __shared__ __align__(16) float res_smem[];
    float* As = res_smem;                    // [d][BM]
    float* Bs = res_smem + kBResMaxD * BM;   // [d][BN]
    __shared__ uint32_t item_s;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int d = a.d, dq = d >> 2;
    for (;;) {
        if (tid == 0) item_s = atomicAdd(&a.ctl->qhead, 1u);
        __syncthreads();
        const uint32_t it = item_s;
        __syncthreads();
        if (it >= a.total_items) break;
        const int i = (int)a.item_inst[it];
        BStep st;
        if (!b_active(a, i, &st)) continue;  // uniform: every thread read the same item
        const BInst& I = a.inst[i];
        const uint32_t local = it - I.item_off;
        const int rt = (int)(local / I.nsplit), split = (int)(local % I.nsplit);
        const int row0 = rt * BM;
        if (row0 >= (int)st.bn) continue;
        const uint32_t* ids = b_rows(a, I, st);
        const float* xi = x + I.row0 * (size_t)d;
        const float* ci = a.c + I.c_off;
        const float* ni = a.norms + I.k_off;
        const int k = (int)I.k, m = (int)st.bn;
        const int ntiles = (k + BN - 1) / BN;
        // the row block, transposed: element e = (chunk c, row r) with r fastest
        for (int e = tid; e < BM * dq; e += 256) {
            const int r = e % BM, c = e / BM;
            float4 v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            if (row0 + r < m) v = *reinterpret_cast<const float4*>(xi + (size_t)ids[row0 + r] * d + 4 * c);
            As[(4 * c + 0) * BM + r] = v.x;
            As[(4 * c + 1) * BM + r] = v.y;
            As[(4 * c + 2) * BM + r] = v.z;
            As[(4 * c + 3) * BM + r] = v.w;
        }
        auto load_b = [&](int col0, float4 (&rb)[BV]) {
#pragma unroll
            for (int q = 0; q < BV; q++) {
                const int e = tid + 256 * q, cc = e % BN, c = e / BN;
                rb[q] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                if (c < dq && col0 + cc < k) rb[q] = *reinterpret_cast<const float4*>(ci + (size_t)(col0 + cc) * d + 4 * c);
            }
        };
        auto store_b = [&](const float4 (&rb)[BV]) {
#pragma unroll
            for (int q = 0; q < BV; q++) {
                const int e = tid + 256 * q, cc = e % BN, c = e / BN;
                if (c < dq) {
                    Bs[(4 * c + 0) * BN + cc] = rb[q].x;
                    Bs[(4 * c + 1) * BN + cc] = rb[q].y;
                    Bs[(4 * c + 2) * BN + cc] = rb[q].z;
                    Bs[(4 * c + 3) * BN + cc] = rb[q].w;
                }
            }
        };
        Top2 top[TM];
#pragma unroll
        for (int q = 0; q < TM; q++) top[q].init();
        float4 rb[BV];
        if (split < ntiles) load_b(split * BN, rb);
        for (int tile = split; tile < ntiles; tile += (int)I.nsplit) {
            const int col0 = tile * BN;
            __syncthreads();  // the previous tile's readers are done with Bs (and As is written)
            store_b(rb);
            __syncthreads();
            if (tile + (int)I.nsplit < ntiles) load_b((tile + (int)I.nsplit) * BN, rb);  // in flight meanwhile
            float acc[TM][TN];
#pragma unroll
            for (int q = 0; q < TM; q++)
#pragma unroll
                for (int j = 0; j < TN; j++) acc[q][j] = 0.0f;
#pragma unroll 4
            for (int kk = 0; kk < d; kk++) {
                float av[TM], bv[TN];
#pragma unroll
                for (int q = 0; q < TM / 2; q++) {
                    av[q] = As[kk * BM + ty * (TM / 2) + q];
                    av[TM / 2 + q] = As[kk * BM + BM / 2 + ty * (TM / 2) + q];
                }
#pragma unroll
                for (int j = 0; j < TN / 2; j++) {
                    bv[j] = Bs[kk * BN + tx * (TN / 2) + j];
                    bv[TN / 2 + j] = Bs[kk * BN + BN / 2 + tx * (TN / 2) + j];
                }
#pragma unroll
                for (int q = 0; q < TM; q++)
#pragma unroll
                    for (int j = 0; j < TN; j++) acc[q][j] = __fmaf_rn(av[q], bv[j], acc[q][j]);
            }
#pragma unroll
            for (int j = 0; j < TN; j++) {
                const int col = col0 + (j < TN / 2 ? tx * (TN / 2) + j : BN / 2 + tx * (TN / 2) + (j - TN / 2));
                if (col < k) {
                    const float nj = ni[col];
#pragma unroll
                    for (int q = 0; q < TM; q++) top[q].push_fast(__fmaf_rn(-2.0f, acc[q][j], nj), (uint32_t)col);
                }
            }
        }
#pragma unroll
        for (int q = 0; q < TM; q++) {
            top[q].merge_shfl_xor(1);
            top[q].merge_shfl_xor(2);
            top[q].merge_shfl_xor(4);
            top[q].merge_shfl_xor(8);
        }
        if (tx == 0) {
#pragma unroll
            for (int q = 0; q < TM; q++) {
                const int row = row0 + (q < TM / 2 ? ty * (TM / 2) + q : BM / 2 + ty * (TM / 2) + (q - TM / 2));
                if (row < m) {
                    const size_t o = (I.p_off + (size_t)split * I.batch + row) * 2;
                    a.part_s[o] = top[q].s1;
                    a.part_i[o] = top[q].i1;
                    a.part_s[o + 1] = top[q].s2;
                    a.part_i[o + 1] = top[q].i2;
                }
            }
        }
        __syncthreads();  // As is rewritten by the next item
    }
}

// The search for small d (d <= D <= 32): one thread per batch row, an item being
// 256 rows against centroid chunks split, split + nsplit, ... of 512 centroids,
// each chunk staged in shared memory 8192 / D centroids at a time (every thread
// reads the same centroid: a broadcast). Score = norm - 2 x.c with the dot
// product as an FMA chain over the dimensions; a running top-2 per row;
// partials as k_b_search writes them.
constexpr int kBSmallRows = 256, kBSmallCols = 512;

template <typename T, int D>
__global__ void __launch_bounds__(256) k_b_search_small(const T* __restrict__ x, BArgs a) {
    constexpr int SUB = 8192 / D < kBSmallCols ? 8192 / D : kBSmallCols;  // 32 KB of staged centroids
    __shared__ __align__(16) float cs[SUB * D];
    __shared__ float ns[SUB];
    __shared__ uint32_t item_s;
    const int tid = threadIdx.x, d = a.d;
    for (;;) {
        if (tid == 0) item_s = atomicAdd(&a.ctl->qhead, 1u);
        __syncthreads();
        const uint32_t it = item_s;
        __syncthreads();
        if (it >= a.total_items) break;
        const int i = (int)a.item_inst[it];
        BStep st;
        if (!b_active(a, i, &st)) continue;
        const BInst& I = a.inst[i];
        const uint32_t local = it - I.item_off;
        const int rt = (int)(local / I.nsplit), split = (int)(local % I.nsplit);
        if (rt * kBSmallRows >= (int)st.bn) continue;
        const int row = rt * kBSmallRows + tid;
        const bool have = row < (int)st.bn;
        float xr[D];
        {
            const T* src = x + (I.row0 + b_rows(a, I, st)[have ? row : 0]) * (size_t)d;
#pragma unroll
            for (int t = 0; t < D; t++) xr[t] = (have && t < d) ? to_f32(src[t]) : 0.0f;
        }
        const int k = (int)I.k, ntiles = (k + kBSmallCols - 1) / kBSmallCols;
        const float* ci = a.c + I.c_off;
        const float* ni = a.norms + I.k_off;
        Top2 top;
        top.init();
        for (int tile = split; tile < ntiles; tile += (int)I.nsplit)
#pragma unroll 1
        for (int sub = 0; sub < kBSmallCols / SUB; sub++) {
            const int col0 = tile * kBSmallCols + sub * SUB, nc = min(SUB, k - col0);
            if (nc <= 0) break;  // uniform across the block
            __syncthreads();  // the previous chunk's readers are done
            for (int e = tid; e < nc * D; e += 256) {
                const int j = e / D, t = e - j * D;
                cs[e] = t < d ? ci[(size_t)(col0 + j) * d + t] : 0.0f;
            }
            for (int j = tid; j < nc; j += 256) ns[j] = ni[col0 + j];
            __syncthreads();
            // four centroids' dot products at a time: independent FMA chains in flight
            int j = 0;
            for (; j + 4 <= nc; j += 4) {
                float dot[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
                for (int t = 0; t < D; t++)
#pragma unroll
                    for (int u = 0; u < 4; u++) dot[u] = __fmaf_rn(xr[t], cs[(j + u) * D + t], dot[u]);
#pragma unroll
                for (int u = 0; u < 4; u++) top.push_fast(__fmaf_rn(-2.0f, dot[u], ns[j + u]), (uint32_t)(col0 + j + u));
            }
            for (; j < nc; j++) {
                float dot = 0.0f;
#pragma unroll
                for (int t = 0; t < D; t++) dot = __fmaf_rn(xr[t], cs[j * D + t], dot);
                top.push_fast(__fmaf_rn(-2.0f, dot, ns[j]), (uint32_t)(col0 + j));
            }
        }
        if (have) {
            const size_t o = (I.p_off + (size_t)split * I.batch + row) * 2;
            a.part_s[o] = top.s1;
            a.part_i[o] = top.i1;
            a.part_s[o + 1] = top.s2;
            a.part_i[o + 1] = top.i2;
        }
    }
}

// Certification for small d: one thread per batch row, the reference's rounding
// through the single-thread restatements (sqnorm_ref, dot_ref), the same decision
// as k_b_certify. Grid (ceil(max batch / 256), count).
template <typename T>
__global__ void k_b_certify_small(const T* __restrict__ x, BArgs a) {
    const int i = blockIdx.y;
    BStep st;
    if (!b_active(a, i, &st)) return;
    const BInst& I = a.inst[i];
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= (int)st.bn) return;
    const int d = a.d, k = (int)I.k;
    const T* xr = x + (I.row0 + b_rows(a, I, st)[row]) * (size_t)d;
    Top2 t;
    t.init();
    for (uint32_t s = 0; s < I.nsplit; s++) {
        const size_t o = (I.p_off + (size_t)s * I.batch + row) * 2;
        t.push(a.part_s[o], a.part_i[o]);
        t.push(a.part_s[o + 1], a.part_i[o + 1]);
    }
    const float xn = sqnorm_ref(xr, d);
    const uint32_t j1 = t.i1 < (uint32_t)k ? t.i1 : 0u;
    const uint32_t j2 = t.i2 < (uint32_t)k ? t.i2 : j1;
    const float* ci = a.c + I.c_off;
    const float d1 = dot_ref(a.match, xr, ci + (size_t)j1 * d, d);
    const float d2 = j2 == j1 ? d1 : dot_ref(a.match, xr, ci + (size_t)j2 * d, d);
    float theta = 0.0f;
    if (!certify_decide(row, t, j1, j2, d1, d2, xn, k, a.norms + I.k_off, &a.bounds[i], a.ka, a.kb,
                        a.blabels + I.b_off, a.bdist + I.b_off, nullptr, 0.0f, 0.0f, nullptr, &theta)) {
        const uint32_t slot = atomicAdd(&a.ctl->redo, 1u);
        a.redo_list[slot] = ((uint32_t)i << 24) | (uint32_t)row;
    }
}

// Exhaustive exact search with a CTA per listed row (256 threads): warp w scans
// the centroids [w k / 8, (w + 1) k / 8) in ascending order in groups as
// k_b_research does, and the warps' results merge by (score, index), finite
// scores only: the lowest index among the smallest scores, label 0 when no score
// beats +inf, as the reference's strict-< scan over all k. A row's centroid
// loads are spread over eight warps, where k_b_research walks all k in one.
template <typename T>
__global__ void __launch_bounds__(256) k_b_research_cta(const T* __restrict__ x, BArgs a) {
    __shared__ float wbest[8];
    __shared__ uint32_t wlab[8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t n = a.ctl->redo;
    const int gsz = a.match == kMatchAvx512 ? 16 : 8, gpw = 32 / gsz, g = lane / gsz;
    const int d = a.d;
    const float inf = __int_as_float(0x7f800000);
    for (uint32_t r = blockIdx.x; r < n; r += gridDim.x) {
        const uint32_t e = a.redo_list[r];
        const int i = (int)(e >> 24), row = (int)(e & 0xFFFFFFu);
        BStep st;
        b_active(a, i, &st);
        const BInst& I = a.inst[i];
        const int k = (int)I.k;
        const T* xr = x + (I.row0 + b_rows(a, I, st)[row]) * (size_t)d;
        const float* ci = a.c + I.c_off;
        const float* ni = a.norms + I.k_off;
        const int jb = (int)(((long long)k * warp) / 8), je = (int)(((long long)k * (warp + 1)) / 8);
        float best = inf;
        uint32_t lab = 0;
        for (int j0 = jb; j0 < je; j0 += gpw) {
            const int j = j0 + g, jc = j < je ? j : je - 1;
            const float dj = group_dot_ref(a.match, xr, ci + (size_t)jc * d, d, lane);
            if (j < je) {
                const float sc = score_ref(ni[j], dj);
                if (sc < best) {
                    best = sc;
                    lab = (uint32_t)j;
                }
            }
        }
        for (int o = gsz; o < 32; o <<= 1) {
            const float ob = __shfl_xor_sync(kFull, best, o);
            const uint32_t ol = __shfl_xor_sync(kFull, lab, o);
            if (ob < inf && (!(best < inf) || lex_less(ob, ol, best, lab))) {
                best = ob;
                lab = ol;
            }
        }
        if (lane == 0) {
            wbest[warp] = best;
            wlab[warp] = lab;
        }
        const float xn = warp_sqnorm_ref(xr, d, lane);
        __syncthreads();
        if (threadIdx.x == 0) {
            float b = inf;
            uint32_t l = 0;
            for (int w = 0; w < 8; w++)
                if (wbest[w] < inf && (!(b < inf) || lex_less(wbest[w], wlab[w], b, l))) {
                    b = wbest[w];
                    l = wlab[w];
                }
            a.blabels[I.b_off + row] = l;
            a.bdist[I.b_off + row] = fmaxf(__fadd_rn(b, xn), 0.0f);
        }
        __syncthreads();  // wbest / wlab are rewritten for the next row
    }
}

// Certification for f32 rows with d % 16 == 0 under the AVX-512 rounding: four
// threads per row with 16-byte loads, the 16 lanes of the reference's sums in
// the same tree as k_certify16v (the same bits as k_b_certify), a quarter of
// the warps. Grid (ceil(max batch * 4 / 256), count).
__global__ void __launch_bounds__(256) k_b_certify16v(const float* __restrict__ x, BArgs a) {
    const int i = blockIdx.y;
    BStep st;
    if (!b_active(a, i, &st)) return;
    const BInst& I = a.inst[i];
    const int lane = threadIdx.x & 31, q = lane & 3;
    const int row = (int)(((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 2);
    const int m = (int)st.bn;
    if (((int)(blockIdx.x * blockDim.x) >> 2) >= m) return;  // the whole block is past the batch
    const bool live = row < m;
    const int r = live ? row : m - 1;  // dead quarter-warps mirror a live row and write nothing
    const int d = a.d, k = (int)I.k;
    const float* xr = x + (I.row0 + b_rows(a, I, st)[r]) * (size_t)d;
    Top2 t;
    t.init();
    for (uint32_t s = 0; s < I.nsplit; s++) {
        const size_t o = (I.p_off + (size_t)s * I.batch + r) * 2;
        t.push(a.part_s[o], a.part_i[o]);
        t.push(a.part_s[o + 1], a.part_i[o + 1]);
    }
    const uint32_t j1 = t.i1 < (uint32_t)k ? t.i1 : 0u;
    const uint32_t j2 = t.i2 < (uint32_t)k ? t.i2 : j1;
    const float* ci = a.c + I.c_off;
    const float* c1 = ci + (size_t)j1 * d;
    const float* c2 = ci + (size_t)j2 * d;
    float sq[4] = {0.0f, 0.0f, 0.0f, 0.0f}, p1[4] = {0.0f, 0.0f, 0.0f, 0.0f}, p2[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    for (int e = 4 * q; e < d; e += 16) {
        const float4 xv = *reinterpret_cast<const float4*>(xr + e);
        const float4 u = *reinterpret_cast<const float4*>(c1 + e);
        const float4 w = *reinterpret_cast<const float4*>(c2 + e);
        const float xs[4] = {xv.x, xv.y, xv.z, xv.w}, us[4] = {u.x, u.y, u.z, u.w}, ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
        for (int j = 0; j < 4; j++) {
            sq[j] = __fadd_rn(sq[j], __fmul_rn(xs[j], xs[j]));
            p1[j] = __fmaf_rn(xs[j], us[j], p1[j]);
            p2[j] = __fmaf_rn(xs[j], ws[j], p2[j]);
        }
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {  // lane l with l^8, then l^4 of the reference's 16 lanes
        p1[j] = __fadd_rn(p1[j], __shfl_xor_sync(kFull, p1[j], 2));
        p2[j] = __fadd_rn(p2[j], __shfl_xor_sync(kFull, p2[j], 2));
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
        p1[j] = __fadd_rn(p1[j], __shfl_xor_sync(kFull, p1[j], 1));
        p2[j] = __fadd_rn(p2[j], __shfl_xor_sync(kFull, p2[j], 1));
    }
    const float a1 = __fadd_rn(__fadd_rn(p1[0], p1[2]), __fadd_rn(p1[1], p1[3]));
    const float a2 = __fadd_rn(__fadd_rn(p2[0], p2[2]), __fadd_rn(p2[1], p2[3]));
    float xn = -0.0f;
    const int base = lane & ~3;
#pragma unroll
    for (int qq = 0; qq < 4; qq++)
#pragma unroll
        for (int j = 0; j < 4; j++) xn = __fadd_rn(xn, __shfl_sync(kFull, sq[j], base + qq));
    if (live && q == 0) {
        float theta = 0.0f;
        if (!certify_decide(row, t, j1, j2, a1, a2, xn, k, a.norms + I.k_off, &a.bounds[i], a.ka, a.kb,
                            a.blabels + I.b_off, a.bdist + I.b_off, nullptr, 0.0f, 0.0f, nullptr, &theta)) {
            const uint32_t slot = atomicAdd(&a.ctl->redo, 1u);
            a.redo_list[slot] = ((uint32_t)i << 24) | (uint32_t)row;
        }
    }
}

// Certification of every active instance's batch rows (one warp per row, the
// reference's rounding for the selected match kernel, as k_certify); rows the
// bound cannot settle are listed for the exhaustive search.
// Grid (ceil(max batch / 8), count).
template <typename T>
__global__ void k_b_certify(const T* __restrict__ x, BArgs a) {
    const int i = blockIdx.y;
    BStep st;
    if (!b_active(a, i, &st)) return;
    const BInst& I = a.inst[i];
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (row >= (int)st.bn) return;
    const int d = a.d, k = (int)I.k;
    const T* xr = x + (I.row0 + b_rows(a, I, st)[row]) * (size_t)d;
    Top2 t;
    t.init();
    for (uint32_t s = 0; s < I.nsplit; s++) {
        const size_t o = (I.p_off + (size_t)s * I.batch + row) * 2;
        t.push(a.part_s[o], a.part_i[o]);
        t.push(a.part_s[o + 1], a.part_i[o + 1]);
    }
    const float xn = warp_sqnorm_ref(xr, d, lane);
    const uint32_t j1 = t.i1 < (uint32_t)k ? t.i1 : 0u;
    const uint32_t j2 = t.i2 < (uint32_t)k ? t.i2 : j1;
    const int gsz = a.match == kMatchAvx512 ? 16 : 8;
    const uint32_t jg = (lane / gsz) == 1 ? j2 : j1;
    const float* ci = a.c + I.c_off;
    const float dg = group_dot_ref(a.match, xr, ci + (size_t)jg * d, d, lane);
    const float d1 = __shfl_sync(kFull, dg, 0);
    const float d2 = __shfl_sync(kFull, dg, gsz);
    if (lane != 0) return;
    float theta = 0.0f;
    if (!certify_decide(row, t, j1, j2, d1, d2, xn, k, a.norms + I.k_off, &a.bounds[i], a.ka, a.kb,
                        a.blabels + I.b_off, a.bdist + I.b_off, nullptr, 0.0f, 0.0f, nullptr, &theta)) {
        const uint32_t slot = atomicAdd(&a.ctl->redo, 1u);
        a.redo_list[slot] = ((uint32_t)i << 24) | (uint32_t)row;
    }
}

// Exhaustive exact search of the listed rows (one warp per row): the reference's
// strict-< scan over ascending centroids, lowest index on ties, as
// k_research_cta; a group that never beats +inf reports (inf, 0).
template <typename T>
__global__ void k_b_research(const T* __restrict__ x, BArgs a) {
    const int lane = threadIdx.x & 31;
    const uint32_t n = a.ctl->redo;
    const int gsz = a.match == kMatchAvx512 ? 16 : 8, gpw = 32 / gsz, g = lane / gsz;
    const int d = a.d;
    for (uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += (gridDim.x * blockDim.x) >> 5) {
        const uint32_t e = a.redo_list[r];
        const int i = (int)(e >> 24), row = (int)(e & 0xFFFFFFu);
        BStep st;
        b_active(a, i, &st);
        const BInst& I = a.inst[i];
        const int k = (int)I.k;
        const T* xr = x + (I.row0 + b_rows(a, I, st)[row]) * (size_t)d;
        const float* ci = a.c + I.c_off;
        const float* ni = a.norms + I.k_off;
        float best = __int_as_float(0x7f800000);
        uint32_t lab = 0;
        for (int j0 = 0; j0 < k; j0 += gpw) {
            const int j = j0 + g, jc = j < k ? j : k - 1;
            const float dj = group_dot_ref(a.match, xr, ci + (size_t)jc * d, d, lane);
            if (j < k) {
                const float s = score_ref(ni[j], dj);
                if (s < best) {
                    best = s;
                    lab = (uint32_t)j;
                }
            }
        }
        if (!(best < __int_as_float(0x7f800000))) lab = 0;
        // Merge the groups of the warp: lowest (score, index), finite scores only.
        for (int o = gsz; o < 32; o <<= 1) {
            const float ob = __shfl_xor_sync(kFull, best, o);
            const uint32_t ol = __shfl_xor_sync(kFull, lab, o);
            if (ob < __int_as_float(0x7f800000) && (!(best < __int_as_float(0x7f800000)) || lex_less(ob, ol, best, lab))) {
                best = ob;
                lab = ol;
            }
        }
        const float xn = warp_sqnorm_ref(xr, d, lane);
        if (lane == 0) {
            a.blabels[I.b_off + row] = lab;
            a.bdist[I.b_off + row] = fmaxf(__fadd_rn(best, xn), 0.0f);
        }
    }
}

// counts[l]++ per batch row, slot = arrival order within the label.
// Grid (ceil(max batch / 256), count).
__global__ void k_b_hist(BArgs a) {
    const int i = blockIdx.y;
    BStep st;
    if (!b_active(a, i, &st)) return;
    const BInst& I = a.inst[i];
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < (int)st.bn) a.slot[I.b_off + r] = atomicAdd(&a.counts[I.k_off + a.blabels[I.b_off + r]], 1u);
}

// Exclusive prefix sum of each instance's counts (one CTA of 1024 per instance).
__global__ void __launch_bounds__(1024) k_b_scan(BArgs a) {
    __shared__ uint32_t part[1024];
    const int i = blockIdx.x;
    BStep st;
    if (!b_active(a, i, &st)) return;
    const BInst& I = a.inst[i];
    const int tid = threadIdx.x, k = (int)I.k;
    const int per = (k + 1023) / 1024;
    const int lo = tid * per, hi = min(k, lo + per);
    const uint32_t* counts = a.counts + I.k_off;
    uint32_t s = 0;
    for (int j = lo; j < hi; j++) s += counts[j];
    part[tid] = s;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        const uint32_t v = tid >= o ? part[tid - o] : 0u;
        __syncthreads();
        part[tid] += v;
        __syncthreads();
    }
    uint32_t base = tid ? part[tid - 1] : 0u;
    for (int j = lo; j < hi; j++) {
        a.offsets[I.k_off + j] = base;
        base += counts[j];
    }
}

__global__ void k_b_scatter(BArgs a) {
    const int i = blockIdx.y;
    BStep st;
    if (!b_active(a, i, &st)) return;
    const BInst& I = a.inst[i];
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < (int)st.bn)
        a.list[I.b_off + a.offsets[I.k_off + a.blabels[I.b_off + r]] + a.slot[I.b_off + r]] = (uint32_t)r;
}

// Per-cluster sums in row order, last-pass sums (one warp per cluster, the
// single-instance segment_sums_warp). Grid (ceil(kmax / 8), count).
template <typename T, int MAXG>
__global__ void k_b_segsums(const T* __restrict__ x, BArgs a, int R) {
    extern __shared__ float seg_stage[];  // R > 0: (blockDim / 32) x 2 R d floats
    const int i = blockIdx.y;
    BStep st;
    if (!b_active(a, i, &st)) return;
    const BInst& I = a.inst[i];
    const int l = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (l >= (int)I.k) return;
    const uint32_t c = a.counts[I.k_off + l];
    if (c == 0) return;
    const uint32_t off = a.offsets[I.k_off + l];
    segment_sums_warp<T, MAXG>(x + I.row0 * (size_t)a.d, b_rows(a, I, st), a.d, l, c, a.list + I.b_off + off,
                               a.scratch + 2 * ((size_t)I.b_off + off), a.sums + I.c_off, (int)st.last,
                               a.pass_counts + I.k_off, a.pass_sums ? a.pass_sums + I.c_off : nullptr,
                               a.pass_sums64 ? a.pass_sums64 + I.c_off : nullptr, lane,
                               R ? seg_stage + (size_t)(threadIdx.x >> 5) * 2 * R * a.d : nullptr, R);
}

// Last pass: the row's label (src/lib.rs:438-440).
__global__ void k_b_store_labels(BArgs a) {
    const int i = blockIdx.y;
    BStep st;
    if (!b_active(a, i, &st) || !st.last) return;
    const BInst& I = a.inst[i];
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < (int)st.bn) a.labels_all[I.n_off + b_rows(a, I, st)[r]] = a.blabels[I.b_off + r];
}

// Batch objective (src/lib.rs:442-445), the same fixed-shape f64 tree as
// k_batch_objective. One CTA of 1024 per instance.
__global__ void __launch_bounds__(1024) k_b_objective(BArgs a) {
    __shared__ double part[1024];
    const int i = blockIdx.x;
    BStep st;
    if (!b_active(a, i, &st)) return;
    const BInst& I = a.inst[i];
    double s = 0.0;
    for (int r = threadIdx.x; r < (int)st.bn; r += 1024) s += (double)a.bdist[I.b_off + r];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int o = 512; o > 0; o >>= 1) {
        if (threadIdx.x < o) part[threadIdx.x] += part[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) a.obj[I.obj_off + st.epoch] += part[0];
}

// EMA step (src/lib.rs:455-456), one warp per cluster. Grid (ceil(kmax / 8), count).
__global__ void k_b_apply(BArgs a) {
    const int i = blockIdx.y;
    BStep st;
    if (!b_active(a, i, &st)) return;
    const BInst& I = a.inst[i];
    const int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (j >= (int)I.k) return;
    apply_warp(j, a.d, a.alphas[I.step_off + a.ctl->gstep], a.c + I.c_off, a.usage + I.k_off, a.counts + I.k_off,
               a.sums + I.c_off, lane);
}

// Revival every fifth step of an instance (src/lib.rs:463-465; revive_cta), one
// CTA of 1024 per instance; donors sorted in shared memory up to smem_sort.
__global__ void __launch_bounds__(1024) k_b_revive(BArgs a, uint32_t smem_sort) {
    extern __shared__ double sort_keys[];
    const int i = blockIdx.x;
    BStep st;
    if (!b_active(a, i, &st)) return;
    const BInst& I = a.inst[i];
    if ((a.ctl->gstep + 1) % 5 != 0 || !(I.tau > 0.0f)) return;
    revive_cta((int)I.k, a.d, a.c + I.c_off, a.usage + I.k_off, I.tau, a.gstream + I.g_off, &a.cursor[i],
               a.keys + I.kp2_off, a.didx + I.kp2_off, a.unused + I.k_off, &a.nsplits[i], I.g_cap, sort_keys,
               smem_sort);
}

// End of a global step: the next step's counters and bounds start afresh.
__global__ void k_b_step_end(BArgs a) {
    for (int i = threadIdx.x; i < a.count; i += blockDim.x) a.bounds[i] = Bounds{0.0f, 0.0f, 0.0f, 0.0f};
    if (threadIdx.x == 0) {
        a.ctl->gstep += 1;
        a.ctl->qhead = 0;
        a.ctl->redo_total += a.ctl->redo;
        a.ctl->redo = 0;
    }
}

// Closing mean (src/lib.rs:481-489) of every instance. Grid (ceil(kmax d / 256), count).
__global__ void k_b_closing_mean(BArgs a) {
    const int i = blockIdx.y;
    const BInst& I = a.inst[i];
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (size_t)I.k * a.d) return;
    const size_t j = e / a.d;
    const unsigned long long n = a.pass_counts[I.k_off + j];
    if (n == 0) return;
    if (a.pass_sums64) {
        a.c[I.c_off + e] = (float)(a.pass_sums64[I.c_off + e] / (double)n);
    } else {
        const float inv = __fdiv_rn(1.0f, (float)n);
        a.c[I.c_off + e] = __fmul_rn(a.pass_sums[I.c_off + e], inv);
    }
}

}  // namespace emb
