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

// set_bias for I8 (src/cpu_i8.rs:112-117): off += (bias as f64).round() as i64 (saturating).
__global__ void k_bias_i8(long long* __restrict__ off, const float* __restrict__ bias, int k) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= k) return;
    double v = round((double)bias[j]);
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

// Grid (ceil(m/128), nsplit). Partial top-1 per (split, row): exact int64 score
// and index; lowest index wins ties within and across threads.
__global__ void __launch_bounds__(256, 1)
k_assign_i8(const int8_t* __restrict__ x, const uint32_t* __restrict__ gather, int m, int d,
            const int8_t* __restrict__ c8, int kpad, const long long* __restrict__ off, int k,
            long long* __restrict__ part_s, uint32_t* __restrict__ part_i, int xvec) {
    __shared__ __align__(16) int As[2][kI8BKW][kI8BM];
    __shared__ __align__(16) int Bs[2][kI8BKW][kI8BN];
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
        int ra[4], rb[4];
        i8_load(ra, x, gather, row0, m, d, d, 0, xvec);
        i8_load(rb, c8, nullptr, col0, k, kpad, kpad, 0, true);
        __syncthreads();
        {
            int r = tid >> 1, w0 = (tid & 1) * 4;
#pragma unroll
            for (int w = 0; w < 4; w++) {
                As[0][w0 + w][r] = ra[w];
                Bs[0][w0 + w][r] = rb[w];
            }
        }
        __syncthreads();
        for (int kt = 0; kt < nk; kt++) {
            const int buf = kt & 1;
            if (kt + 1 < nk) {
                i8_load(ra, x, gather, row0, m, d, d, (kt + 1) * 32, xvec);
                i8_load(rb, c8, nullptr, col0, k, kpad, kpad, (kt + 1) * 32, true);
            }
#pragma unroll
            for (int w = 0; w < kI8BKW; w++) {
                int4 a0 = *reinterpret_cast<const int4*>(&As[buf][w][ty * 4]);
                int4 a1 = *reinterpret_cast<const int4*>(&As[buf][w][64 + ty * 4]);
                int4 b0 = *reinterpret_cast<const int4*>(&Bs[buf][w][tx * 4]);
                int4 b1 = *reinterpret_cast<const int4*>(&Bs[buf][w][64 + tx * 4]);
                int a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
                int b[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
                for (int i = 0; i < 8; i++)
#pragma unroll
                    for (int j = 0; j < 8; j++) acc[i][j] = __dp4a(a[i], b[j], acc[i][j]);
            }
            if (kt + 1 < nk) {
                int r = tid >> 1, w0 = (tid & 1) * 4;
#pragma unroll
                for (int w = 0; w < 4; w++) {
                    As[buf ^ 1][w0 + w][r] = ra[w];
                    Bs[buf ^ 1][w0 + w][r] = rb[w];
                }
            }
            __syncthreads();
        }
#pragma unroll
        for (int j = 0; j < 8; j++) {
            int col = col0 + (j < 4 ? tx * 4 + j : 64 + tx * 4 + (j - 4));
            if (col < k) {
                long long o = off[col];
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    long long s = o - 2ll * (long long)acc[i][j];
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

// Merge the split partials, dist = max(|x|^2 + best, 0) computed in f64 and
// rounded to f32 (src/cpu_i8.rs:183-186). One warp per row.
__global__ void k_finish_i8(const int8_t* __restrict__ x, const uint32_t* __restrict__ gather, int m, int d,
                            const long long* __restrict__ part_s, const uint32_t* __restrict__ part_i, int nsplit,
                            uint32_t* __restrict__ labels, float* __restrict__ dist) {
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
    dist[row] = (float)fmax((double)nrm + (double)b, 0.0);
}

}  // namespace emb
