// Exact integer search for i8 rows with i8 centroids, the semantics of
// CpuI8Assigner(CentroidBits::I8) (src/cpu_i8.rs:72-191). Scores are exact
// integers, so the fast kernel's argmin is the reference's label directly.
#pragma once
#include "common.cuh"

namespace emb {

// set_centroids for I8 (src/cpu_i8.rs:80-94): c8 = clamp(round half away(c)),
// off_j = sum c8^2. The reference ranks by sum(c^2 + 256 c) - 2 sum((x+128) c),
// which is the same integer as sum c^2 - 2 x.c. One warp per centroid; rows of
// c8 are padded with zeros to kpad bytes.
__global__ void k_prep_i8(const float* __restrict__ c, int k, int d, int kpad, int8_t* __restrict__ c8,
                          long long* __restrict__ off) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (warp >= k) return;
    long long s = 0;
    for (int t = lane; t < kpad; t += 32) {
        int v = 0;
        if (t < d) {
            float f = c[(size_t)warp * d + t];
            if (f == f) v = (int)fminf(fmaxf(roundf(f), -128.0f), 127.0f);  // NaN -> 0 (Rust `as` cast)
        }
        c8[(size_t)warp * kpad + t] = (int8_t)v;
        s += (long long)v * v;
    }
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) off[warp] = s;
}

// set_centroids for I16 (src/cpu_i8.rs:95-107): c16 = clamp(round half away(c *
// 2^shift), -32768, 32767) (NaN -> 0), off_j = sum c16^2. Rows padded with zeros
// to kpad elements (whole 32-element K steps of k_assign_i8<true>).
__global__ void k_prep_i16(const float* __restrict__ c, int k, int d, int kpad, float scale,
                           int16_t* __restrict__ c16, long long* __restrict__ off) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (warp >= k) return;
    long long s = 0;
    for (int t = lane; t < kpad; t += 32) {
        int v = 0;
        if (t < d) {
            float f = __fmul_rn(c[(size_t)warp * d + t], scale);
            if (f == f) v = (int)fminf(fmaxf(roundf(f), -32768.0f), 32767.0f);
        }
        c16[(size_t)warp * kpad + t] = (int16_t)v;
        s += (long long)v * v;
    }
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) off[warp] = s;
}

// set_bias in integer mode (src/cpu_i8.rs:112-117): off += (bias as f64 * unit).round()
// as i64 (saturating), unit = 2^(2 shift) score units per squared distance (1 for I8).
__global__ void k_bias_i8(long long* __restrict__ off, const float* __restrict__ bias, int k, double unit) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= k) return;
    double v = round(__dmul_rn((double)bias[j], unit));
    long long iv;
    if (v != v) iv = 0;
    else if (v >= 9.2233720368547758e18) iv = 0x7fffffffffffffffll;
    else if (v <= -9.2233720368547758e18) iv = (long long)0x8000000000000000ull;
    else iv = (long long)v;
    off[j] += iv;
}

constexpr int kI8BM = 128, kI8BN = 128, kI8BKW = 8;  // 8 words = 32 bytes of K per stage

EMB_DEV void i8_load(int (&r)[4], const int8_t* __restrict__ base, const uint32_t* __restrict__ gather, int row0,
                     int nrows, int stride, int d, int kb0, bool vec) {
    int t = threadIdx.x;
    int row = row0 + (t >> 1);
    int col = kb0 + (t & 1) * 16;
    if (row >= nrows) {
        r[0] = r[1] = r[2] = r[3] = 0;
        return;
    }
    size_t src = gather ? gather[row] : (size_t)row;
    const int8_t* p = base + src * (size_t)stride + col;
    if (vec && col + 16 <= d) {
        int4 v = *reinterpret_cast<const int4*>(p);
        r[0] = v.x; r[1] = v.y; r[2] = v.z; r[3] = v.w;
    } else {
#pragma unroll
        for (int w = 0; w < 4; w++) {
            unsigned int word = 0;
#pragma unroll
            for (int b = 0; b < 4; b++) {
                int cc = col + w * 4 + b;
                unsigned int byte = cc < d ? (unsigned int)(uint8_t)p[w * 4 + b] : 0u;
                word |= byte << (8 * b);
            }
            r[w] = (int)word;
        }
    }
}

// 32 i16 centroid elements of row (row0 + t/2) from element kb0 + 16 (t&1): eight
// words of two elements each (rows are padded to whole 32-element steps).
EMB_DEV void i16_load(int (&r)[8], const int16_t* __restrict__ base, int row0, int nrows, int kpad, int kb0) {
    int t = threadIdx.x;
    int row = row0 + (t >> 1);
    if (row >= nrows) {
#pragma unroll
        for (int w = 0; w < 8; w++) r[w] = 0;
        return;
    }
    const int4* p = reinterpret_cast<const int4*>(base + (size_t)row * kpad + kb0 + (t & 1) * 16);
    int4 v0 = p[0], v1 = p[1];
    r[0] = v0.x; r[1] = v0.y; r[2] = v0.z; r[3] = v0.w;
    r[4] = v1.x; r[5] = v1.y; r[6] = v1.z; r[7] = v1.w;
}

// Grid (ceil(m/128), nsplit). Partial top-1 per (split, row): exact int64 score
// and index; lowest index wins ties within and across threads.
// WIDE = false: I8 centroids, score off_j - 2 (x . c8) by dp4a.
// WIDE = true : I16 centroids, score off_j - mult (x . c16) by dp2a (two 16-bit
//               centroid elements times two 8-bit row elements per instruction);
//               the shift keeps x . c16 inside an int32 (src/cpu_i8.rs:96-97).
template <bool WIDE>
__global__ void __launch_bounds__(256, 1)
k_assign_i8(const int8_t* __restrict__ x, const uint32_t* __restrict__ gather, int m, int d,
            const void* __restrict__ cq, int kpad, const long long* __restrict__ off, int k, long long mult,
            long long* __restrict__ part_s, uint32_t* __restrict__ part_i, int xvec) {
    constexpr int BW = WIDE ? 2 * kI8BKW : kI8BKW;  // centroid words per 32-element step
    __shared__ __align__(16) int As[2][kI8BKW][kI8BM];
    __shared__ __align__(16) int Bs[2][BW][kI8BN];
    const int8_t* c8 = static_cast<const int8_t*>(cq);
    const int16_t* c16 = static_cast<const int16_t*>(cq);
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int row0 = blockIdx.x * kI8BM;
    const int nsplit = gridDim.y;
    const int ntiles = (k + kI8BN - 1) / kI8BN;
    const int nk = (d + 31) / 32;
    long long best[8];
    uint32_t bidx[8];
#pragma unroll
    for (int i = 0; i < 8; i++) {
        best[i] = 0x7fffffffffffffffll;
        bidx[i] = 0;
    }
    for (int tile = blockIdx.y; tile < ntiles; tile += nsplit) {
        const int col0 = tile * kI8BN;
        int acc[8][8];
#pragma unroll
        for (int i = 0; i < 8; i++)
#pragma unroll
            for (int j = 0; j < 8; j++) acc[i][j] = 0;
        int ra[4], rb[WIDE ? 8 : 4];
        auto load_b = [&](int kb0) {
            if constexpr (WIDE) i16_load(rb, c16, col0, k, kpad, kb0);
            else i8_load(rb, c8, nullptr, col0, k, kpad, kpad, kb0, true);
        };
        auto store = [&](int buf) {
            const int r = tid >> 1, w0 = (tid & 1) * 4;
#pragma unroll
            for (int w = 0; w < 4; w++) As[buf][w0 + w][r] = ra[w];
#pragma unroll
            for (int w = 0; w < (WIDE ? 8 : 4); w++) Bs[buf][(tid & 1) * (WIDE ? 8 : 4) + w][r] = rb[w];
        };
        i8_load(ra, x, gather, row0, m, d, d, 0, xvec);
        load_b(0);
        __syncthreads();
        store(0);
        __syncthreads();
        for (int kt = 0; kt < nk; kt++) {
            const int buf = kt & 1;
            if (kt + 1 < nk) {
                i8_load(ra, x, gather, row0, m, d, d, (kt + 1) * 32, xvec);
                load_b((kt + 1) * 32);
            }
#pragma unroll
            for (int w = 0; w < kI8BKW; w++) {
                int4 a0 = *reinterpret_cast<const int4*>(&As[buf][w][ty * 4]);
                int4 a1 = *reinterpret_cast<const int4*>(&As[buf][w][64 + ty * 4]);
                int a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
                if constexpr (WIDE) {
                    // word 2w: elements 4w, 4w+1; word 2w+1: elements 4w+2, 4w+3
                    int4 l0 = *reinterpret_cast<const int4*>(&Bs[buf][2 * w][tx * 4]);
                    int4 l1 = *reinterpret_cast<const int4*>(&Bs[buf][2 * w][64 + tx * 4]);
                    int4 h0 = *reinterpret_cast<const int4*>(&Bs[buf][2 * w + 1][tx * 4]);
                    int4 h1 = *reinterpret_cast<const int4*>(&Bs[buf][2 * w + 1][64 + tx * 4]);
                    int bl[8] = {l0.x, l0.y, l0.z, l0.w, l1.x, l1.y, l1.z, l1.w};
                    int bh[8] = {h0.x, h0.y, h0.z, h0.w, h1.x, h1.y, h1.z, h1.w};
#pragma unroll
                    for (int i = 0; i < 8; i++)
#pragma unroll
                        for (int j = 0; j < 8; j++)
                            acc[i][j] = __dp2a_hi(bh[j], a[i], __dp2a_lo(bl[j], a[i], acc[i][j]));
                } else {
                    int4 b0 = *reinterpret_cast<const int4*>(&Bs[buf][w][tx * 4]);
                    int4 b1 = *reinterpret_cast<const int4*>(&Bs[buf][w][64 + tx * 4]);
                    int b[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
                    for (int i = 0; i < 8; i++)
#pragma unroll
                        for (int j = 0; j < 8; j++) acc[i][j] = __dp4a(a[i], b[j], acc[i][j]);
                }
            }
            if (kt + 1 < nk) store(buf ^ 1);
            __syncthreads();
        }
#pragma unroll
        for (int j = 0; j < 8; j++) {
            int col = col0 + (j < 4 ? tx * 4 + j : 64 + tx * 4 + (j - 4));
            if (col < k) {
                long long o = off[col];
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    long long s = o - mult * (long long)acc[i][j];
                    if (s < best[i]) {
                        best[i] = s;
                        bidx[i] = (uint32_t)col;
                    }
                }
            }
        }
    }
#pragma unroll
    for (int i = 0; i < 8; i++) {
#pragma unroll
        for (int msk = 1; msk < 16; msk <<= 1) {
            long long ob = __shfl_xor_sync(0xffffffffu, best[i], msk);
            uint32_t oi = __shfl_xor_sync(0xffffffffu, bidx[i], msk);
            if (ob < best[i] || (ob == best[i] && oi < bidx[i])) {
                best[i] = ob;
                bidx[i] = oi;
            }
        }
    }
    if (tx == 0) {
#pragma unroll
        for (int i = 0; i < 8; i++) {
            int row = row0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + (i - 4));
            if (row < m) {
                size_t o = (size_t)blockIdx.y * m + row;
                part_s[o] = best[i];
                part_i[o] = bidx[i];
            }
        }
    }
}

// Merge the split partials, dist = max(|x|^2 + best * inv_unit, 0) computed in
// f64 and rounded to f32 (src/cpu_i8.rs:183-186; inv_unit = 2^(-2 shift), 1 for
// I8). One warp per row.
__global__ void k_finish_i8(const int8_t* __restrict__ x, const uint32_t* __restrict__ gather, int m, int d,
                            const long long* __restrict__ part_s, const uint32_t* __restrict__ part_i, int nsplit,
                            uint32_t* __restrict__ labels, float* __restrict__ dist, double inv_unit) {
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= m) return;
    const size_t src = gather ? gather[row] : (size_t)row;
    const int8_t* xr = x + src * (size_t)d;
    long long nrm = 0;
    for (int t = lane; t < d; t += 32) nrm += (long long)xr[t] * xr[t];
    for (int o = 16; o; o >>= 1) nrm += __shfl_xor_sync(0xffffffffu, nrm, o);
    if (lane != 0) return;
    long long b = 0x7fffffffffffffffll;
    uint32_t l = 0;
    for (int s = 0; s < nsplit; s++) {
        const long long v = part_s[(size_t)s * m + row];
        const uint32_t i = part_i[(size_t)s * m + row];
        if (v < b || (v == b && i < l)) {
            b = v;
            l = i;
        }
    }
    labels[row] = l;
    dist[row] = (float)fmax(__dadd_rn((double)nrm, __dmul_rn((double)b, inv_unit)), 0.0);
}

}  // namespace emb
