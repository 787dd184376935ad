// Fused tcgen05 forward pass of the proposer network, d -> H -> H -> G, with the
// top-`top` group selection in its epilogue: one CTA takes 128 rows at a time
// (persistent over row tiles) and no activation or logit reaches HBM.
//
//   warp 0       TMA producer: streams the weight matrices W1, W2, W3 (BF16,
//                K-major, 128-byte swizzle) one 64-wide K slice of up to 256
//                output columns per stage, layer after layer, tile after tile
//   warp 1       allocates TMEM (512 columns), issues tcgen05.mma M=128 N<=256
//                K=16 (one thread) into FP32 accumulators, commits per layer
//   warps 2..17  input: rows -> (x - mean) * inv_std -> BF16 into the activation
//                buffer; after layers 1 and 2: TMEM -> + bias, ReLU -> BF16 back
//                into the same buffer (the next layer's A operand); after
//                layer 3: logits -> per-thread top lists, max and exp-sum over
//                a quarter of the groups, merged across the four quarters.
// The activation buffer (128 x H BF16) is shared by X0, H1 and H2: each is
// written only after the MMAs reading its predecessor have completed.
#pragma once
#include "kernels_tc.cuh"

namespace emb {

constexpr int kMlpMaxStages = 4;

struct MlpTcParams {
    int m, d, kin, H, G, top;  // kin: d rounded up to 64
    const float* x;
    const uint32_t* rows;      // optional row indices (else rows row0 + r)
    const float* mean;
    const float* istd;
    const float* b1;
    const float* b2;
    const float* b3;
    uint16_t* groups;          // [m][top]
    float* conf;               // [m]
    float* logits;             // optional [m][G]
    int* err;                  // set to 1 if a bounded wait gave up
    float mass_target;         // search the fewest groups whose mass reaches it (<= 0: all `top`)
    uint8_t* cnt;              // [m] groups to search
};

struct MlpTcSmem {
    uint32_t act, stages, bars, total;
    int nstages;
};

// The activation buffer also holds the layer-3 merge records, 4 x 128 rows x
// (2 topc + 2) floats, once the tile's last MMAs have completed.
__host__ __device__ inline MlpTcSmem mlp_tc_smem(int kin, int H, int topc) {
    MlpTcSmem s;
    const uint32_t acts = (uint32_t)kTcBM * 2 * (uint32_t)(kin > H ? kin : H);
    const uint32_t merge = 4u * kTcBM * (uint32_t)(2 * topc + 2) * 4u;
    const uint32_t act = acts > merge ? acts : merge;
    const uint32_t stage = 256u * 128u;  // 256 output columns x 64 BF16
    s.act = 0;
    s.stages = act;
    int st = 0;
    while (st < kMlpMaxStages && act + (st + 1) * stage + 256 + 1024 <= (uint32_t)kTcSmemLimit) st++;
    s.nstages = st;
    s.bars = act + st * stage;
    s.total = s.bars + 256;
    return s;
}

// Each epilogue thread keeps the TOPC best of its 64 (or 32) columns; the merge
// of the four quarters' lists gives the exact top TOPC, and for top up to 4 TOPC
// the best of what the lists hold.
// relu(a + ba), relu(b + bb) rounded to BF16 and packed (low half: a): the two
// f32 additions in one packed FMA with multiplier 1 (each rounded once, as a
// plain add), then ReLU, rounding and packing in one conversion.
EMB_DEV uint32_t bias_relu_bf16x2(float a, float b, float ba, float bb) {
    float sa, sb;
    asm("{\n .reg .b64 ra, rb, rc, rd;\n mov.b64 ra, {%2, %3};\n mov.b64 rb, {%4, %5};\n mov.b64 rc, {%6, %7};\n"
        " fma.rn.f32x2 rd, ra, rb, rc;\n mov.b64 {%0, %1}, rd;\n}\n"
        : "=f"(sa), "=f"(sb)
        : "f"(a), "f"(b), "f"(1.0f), "f"(1.0f), "f"(ba), "f"(bb));
    uint32_t r;
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(sb), "f"(sa));  // first operand -> upper half
    return r;
}

// Insert (v, j) into a descending list of length N (ties keep the earlier column first).
template <int N>
EMB_DEV void topn_insert(float (&val)[N], int (&idx)[N], float v, int j) {
    if (!(v > val[N - 1])) return;
    val[N - 1] = v;
    idx[N - 1] = j;
#pragma unroll
    for (int i = N - 1; i > 0; i--) {
        const bool sw = val[i] > val[i - 1];
        const float a = val[i], b = val[i - 1];
        const int ia = idx[i], ib = idx[i - 1];
        val[i - 1] = sw ? a : b;
        val[i] = sw ? b : a;
        idx[i - 1] = sw ? ia : ib;
        idx[i] = sw ? ib : ia;
    }
}

// Units of one row tile, in the order the producer loads and the MMA consumes them:
// layer 0: H/256 halves x kin/64 atoms; layer 1: H/256 halves x H/64 atoms; layer 2: H/64 atoms.
EMB_DEV void mlp_unit(int u, int kin, int H, int& layer, int& half, int& atom) {
    const int nh = H / 256, a0 = kin / 64, a1 = H / 64;
    if (u < nh * a0) {
        layer = 0;
        half = u / a0;
        atom = u % a0;
        return;
    }
    u -= nh * a0;
    if (u < nh * a1) {
        layer = 1;
        half = u / a1;
        atom = u % a1;
        return;
    }
    layer = 2;
    half = 0;
    atom = u - nh * a1;
}

template <int TOPC>
__global__ void __launch_bounds__(kTcThreads, 1)
k_mlp_tc(const __grid_constant__ CUtensorMap map_w1, const __grid_constant__ CUtensorMap map_w2,
         const __grid_constant__ CUtensorMap map_w3, const MlpTcParams p) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = smem_align1024(smem_raw);
    const MlpTcSmem L = mlp_tc_smem(p.kin, p.H, TOPC);
    const int S = L.nstages;
    uint64_t* full = (uint64_t*)(smem + L.bars);  // [kMlpMaxStages]
    uint64_t* empty = full + kMlpMaxStages;       // [kMlpMaxStages]
    uint64_t* acc_full = empty + kMlpMaxStages;   // MMA -> epilogue, once per layer
    uint64_t* a_ready = acc_full + 1;             // epilogue -> MMA, once per layer (16 warp arrivals)
    uint64_t* mma_done = a_ready + 1;             // every issued MMA completed (teardown)
    uint32_t* tmem_slot = (uint32_t*)(mma_done + 1);
    volatile int* abort_flag = (volatile int*)(tmem_slot + 1);
    uint8_t* act = smem + L.act;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntiles = (p.m + kTcBM - 1) / kTcBM;
    const int my_tiles = (int)blockIdx.x < ntiles ? (ntiles - (int)blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
    const int upt = (p.H / 256) * (p.kin / 64) + (p.H / 256) * (p.H / 64) + p.H / 64;  // units per tile

    if (threadIdx.x == 0) {
        for (int s = 0; s < kMlpMaxStages; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(acc_full, 1);
        mbar_init(a_ready, kTcEpiWarps);
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
            const int nunits = my_tiles * upt;
            int issued = 0;
            for (int u = 0; u < nunits; u++) {
                const int s = u % S;
                const uint32_t ph = (uint32_t)(u / S) & 1u;
                if (!mbar_wait(&empty[s], ph ^ 1u, abort_flag)) break;
                int layer, half, atom;
                mlp_unit(u % upt, p.kin, p.H, layer, half, atom);
                const uint32_t bytes = (layer == 2 ? (uint32_t)p.G : 256u) * 128u;
                uint8_t* stage = smem + L.stages + s * 256 * 128;
                mbar_expect_tx(&full[s], bytes);
                const CUtensorMap* map = layer == 0 ? &map_w1 : layer == 1 ? &map_w2 : &map_w3;
                tma_load_2d(stage, map, &full[s], atom * 64, half * 256);
                issued = u + 1;
            }
            if (*abort_flag) {
                const uint64_t t0 = global_ns();
                for (int u = issued > S ? issued - S : 0; u < issued; u++) {
                    const uint32_t ph = (uint32_t)(u / S) & 1u;
                    while (!mbar_try(&full[u % S], ph) && global_ns() - t0 < kWaitLimitNs) {
                    }
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t act_base = smem_u32(act);
            const uint32_t atom_units = (kTcBM * 128) >> 4;  // descriptor units per activation K atom
            int u = 0;
            uint32_t aph = 0;
            bool ok = true;
            for (int t = 0; t < my_tiles && ok; t++) {
                for (int layer = 0; layer < 3 && ok; layer++) {
                    if (!mbar_wait(a_ready, aph, abort_flag)) {
                        ok = false;
                        break;
                    }
                    aph ^= 1u;
                    tc_fence_after();
                    const int nh = layer < 2 ? p.H / 256 : 1;
                    const int na = layer == 0 ? p.kin / 64 : p.H / 64;
                    const uint32_t idesc = idesc_bf16(kTcBM, layer < 2 ? 256 : p.G);
                    for (int hf = 0; hf < nh && ok; hf++) {
                        const uint32_t d_tmem = tmem_base + (uint32_t)(hf * 256);
                        for (int a = 0; a < na; a++, u++) {
                            const int s = u % S;
                            const uint32_t ph = (uint32_t)(u / S) & 1u;
                            if (!mbar_wait(&full[s], ph, abort_flag)) {
                                ok = false;
                                break;
                            }
                            tc_fence_after();
                            const uint64_t bd = sw128_desc(smem_u32(smem + L.stages + s * 256 * 128));
                            const uint64_t ad = sw128_desc(act_base) + (uint64_t)(a * atom_units);
#pragma unroll
                            for (int kk = 0; kk < 4; kk++) mma_bf16(d_tmem, ad + 2 * kk, bd + 2 * kk, idesc,
                                                                    (a > 0 || kk > 0) ? 1u : 0u);
                            mma_commit(&empty[s]);
                        }
                    }
                    if (ok) mma_commit(acc_full);
                }
            }
            mma_drain(mma_done);  // no MMA may outlive the TMEM allocation (see k_assign_tc)
        }
    } else {
        const int q = warp & 3;          // TMEM lane quarter
        const int cq = (warp - 2) >> 2;  // column quarter
        const int r = q * 32 + lane;     // row of this thread in the tile
        const int et = threadIdx.x - 64; // 0..511
        uint32_t accph = 0;
        float* mg = (float*)act;         // merge area (reuses the activation buffer after layer 3)
        // After an abort every epilogue warp still walks all tiles and reaches every
        // named barrier, skipping the waits and the work, so no warp is left at one.
        bool ok = true;
        for (int t = 0; t < my_tiles; t++) {
            const int row0 = ((int)blockIdx.x + t * (int)gridDim.x) * kTcBM;
            // ---- input rows
            const int nchunk = p.kin / 8;
            for (int c = et; ok && c < kTcBM * nchunk; c += kTcEpiWarps * 32) {
                const int rr = c / nchunk, kc = c % nchunk, g = row0 + rr, k0 = kc * 8;
                float v[8];
#pragma unroll
                for (int i = 0; i < 8; i++) v[i] = 0.0f;
                if (g < p.m && k0 < p.d) {
                    // d is a multiple of 8 (fused-pass condition): whole 8-element chunks
                    const size_t src = p.rows ? (size_t)p.rows[g] : (size_t)g;
                    const float4* xr = reinterpret_cast<const float4*>(p.x + src * (size_t)p.d + k0);
                    const float4* mr = reinterpret_cast<const float4*>(p.mean + k0);
                    const float4* sr = reinterpret_cast<const float4*>(p.istd + k0);
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        const float4 xv = xr[h], mv = __ldg(mr + h), sv = __ldg(sr + h);
                        v[4 * h + 0] = (xv.x - mv.x) * sv.x;
                        v[4 * h + 1] = (xv.y - mv.y) * sv.y;
                        v[4 * h + 2] = (xv.z - mv.z) * sv.z;
                        v[4 * h + 3] = (xv.w - mv.w) * sv.w;
                    }
                }
                uint32_t w[4];
#pragma unroll
                for (int i = 0; i < 4; i++)
                    w[i] = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(v[2 * i])) |
                           ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(v[2 * i + 1])) << 16);
                *reinterpret_cast<uint4*>(act + sw128_offset(rr, kc, kTcBM)) = make_uint4(w[0], w[1], w[2], w[3]);
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            tc_fence_before();
            __syncwarp();
            if (lane == 0 && ok) mbar_arrive(a_ready);
            // ---- hidden layers: TMEM -> bias, ReLU -> BF16 activations
            for (int layer = 0; layer < 2; layer++) {
                ok = ok && mbar_wait(acc_full, accph, abort_flag, 20000);
                if (!ok) break;
                accph ^= 1u;
                tc_fence_after();
                const float* bias = layer == 0 ? p.b1 : p.b2;
                const int per = p.H / 4;
                for (int ch = 0; ch < per; ch += 32) {
                    const int c0 = cq * per + ch;
                    uint32_t v[32];
                    EMB_TMEM_LD32(tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)c0, v);
                    tmem_wait_ld();
                    tc_regs_ready(v);
#pragma unroll
                    for (int j = 0; j < 32; j += 8) {
                        const float4 b0 = __ldg(reinterpret_cast<const float4*>(bias + c0 + j));
                        const float4 b1 = __ldg(reinterpret_cast<const float4*>(bias + c0 + j + 4));
                        const float bb[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
                        uint32_t w[4];
#pragma unroll
                        for (int i = 0; i < 4; i++)
                            w[i] = bias_relu_bf16x2(__uint_as_float(v[j + 2 * i]), __uint_as_float(v[j + 2 * i + 1]),
                                                    bb[2 * i], bb[2 * i + 1]);
                        *reinterpret_cast<uint4*>(act + sw128_offset(r, (c0 + j) >> 3, kTcBM)) =
                            make_uint4(w[0], w[1], w[2], w[3]);
                    }
                }
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(a_ready);
            }
            // ---- output layer: logits -> top lists, max and exp-sum per column quarter
            ok = ok && mbar_wait(acc_full, accph, abort_flag, 20000);
            const int rec = 2 * TOPC + 2;  // floats per (quarter, row) record
            const int row = row0 + r;
            if (ok) {
                accph ^= 1u;
                tc_fence_after();
                float tv[TOPC];
                int ti[TOPC];
#pragma unroll
                for (int i = 0; i < TOPC; i++) {
                    tv[i] = -INFINITY;
                    ti[i] = 0x7fffffff;
                }
                float mx = -INFINITY, se = 0.0f;
                const int per = p.G / 4;
                for (int ch = 0; ch < per; ch += 32) {
                    const int c0 = cq * per + ch;
                    uint32_t v[32];
                    EMB_TMEM_LD32(tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)c0, v);
                    tmem_wait_ld();
                    tc_regs_ready(v);
                    float l[32];
                    float cm = -INFINITY;
#pragma unroll
                    for (int j = 0; j < 32; j++) {
                        l[j] = __uint_as_float(v[j]) + p.b3[c0 + j];
                        cm = fmaxf(cm, l[j]);
                    }
                    if (p.logits && row < p.m) {
#pragma unroll
                        for (int j = 0; j < 32; j++) p.logits[(size_t)row * p.G + c0 + j] = l[j];
                    }
                    const float nm = fmaxf(mx, cm);
                    float add = 0.0f;
#pragma unroll
                    for (int j = 0; j < 32; j++) add += __expf(l[j] - nm);
                    se = se * __expf(mx - nm) + add;
                    mx = nm;
#pragma unroll
                    for (int j = 0; j < 32; j++) topn_insert<TOPC>(tv, ti, l[j], c0 + j);
                }
                // All MMAs of this tile are complete: the activation buffer is free for the merge.
                float* e = mg + ((size_t)cq * kTcBM + r) * rec;
#pragma unroll
                for (int i = 0; i < TOPC; i++) {
                    e[i] = tv[i];
                    e[TOPC + i] = __int_as_float(ti[i]);
                }
                e[2 * TOPC] = mx;
                e[2 * TOPC + 1] = se;
            }
            tc_fence_before();
            asm volatile("bar.sync 1, %0;" ::"n"(kTcEpiWarps * 32) : "memory");
            if (ok && cq == 0 && row < p.m) {
                int head[4] = {0, 0, 0, 0};
                float M = -INFINITY;
#pragma unroll
                for (int o = 0; o < 4; o++) M = fmaxf(M, mg[((size_t)o * kTcBM + r) * rec + 2 * TOPC]);
                float Ssum = 0.0f;
#pragma unroll
                for (int o = 0; o < 4; o++) {
                    const float* f = mg + ((size_t)o * kTcBM + r) * rec;
                    Ssum += f[2 * TOPC + 1] * __expf(f[2 * TOPC] - M);
                }
                float mass = 0.0f;
                int n_search = p.top;
                for (int s = 0; s < p.top; s++) {
                    float bv = -INFINITY;
                    int bi = 0x7fffffff, bo = 0;
#pragma unroll
                    for (int o = 0; o < 4; o++) {
                        if (head[o] >= TOPC) continue;
                        const float* f = mg + ((size_t)o * kTcBM + r) * rec;
                        const float fv = f[head[o]];
                        const int fi = __float_as_int(f[TOPC + head[o]]);
                        if (fv > bv || (fv == bv && fi < bi)) {
                            bv = fv;
                            bi = fi;
                            bo = o;
                        }
                    }
                    head[bo]++;
                    if (bi < 0 || bi >= p.G) bi = 0;  // no finite logit left (a diverged network): any valid group
                    p.groups[(size_t)row * p.top + s] = (uint16_t)bi;
                    mass += __expf(bv - M);
                    if (p.mass_target > 0.0f && n_search == p.top && mass >= p.mass_target * Ssum) n_search = s + 1;
                }
                p.conf[row] = mass / Ssum;
                p.cnt[row] = (uint8_t)n_search;
            }
            // The next tile's input overwrites the merge records.
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
