// Exact kernels: centroid preparation, certification of the fast top-2 and the
// exact re-search, all in the reference CpuAssigner's own f32 rounding.
#pragma once
#include <cuda_bf16.h>
#include "common.cuh"

namespace emb {

constexpr unsigned kFull = 0xffffffffu;

// Device-side bounds used by the certification (filled by k_prep_centroids / k_bias).
struct Bounds {
    float cmax;  // >= max_j |c_j| (upper-rounded)
    float nmax;  // >= max_j |norms_j| (norms include the bias)
    float cmax_hi;  // >= max_j |bf16(c_j)| (three-term split bound)
    float dmax;     // >= max_j |c_j - bf16(c_j)| (single-term residual bound)
};

// Upper bound of |v - bf16(v)|^2 summed into acc (v - bf16(v) is exact in f32).
EMB_DEV float bf16_resid_sq(float v, float acc) {
    const float r = v - __bfloat162float(__float2bfloat16_rn(v));
    return __fmaf_ru(r, r, acc);
}

EMB_DEV void atomic_max_pos(float* addr, float v) {
    // Non-negative floats order like their bit patterns.
    atomicMax((unsigned int*)addr, __float_as_uint(v));
}

// Warp-cooperative sqnorm_ref (src/cpu.rs:169-180). All lanes return the value.
template <typename T>
EMB_DEV float warp_sqnorm_ref(const T* v, int d, int lane) {
    int body = d & ~15;
    float acc = 0.0f;
    if (lane < 16)
        for (int i = lane; i < body; i += 16) {
            float a = to_f32(v[i]);
            acc = __fadd_rn(acc, __fmul_rn(a, a));
        }
    float s = -0.0f;
#pragma unroll
    for (int q = 0; q < 16; q++) s = __fadd_rn(s, __shfl_sync(kFull, acc, q));
    float t = -0.0f;
    for (int i = body; i < d; i++) {
        float a = to_f32(v[i]);
        t = __fadd_rn(t, __fmul_rn(a, a));
    }
    return __fadd_rn(s, t);
}

// Group-cooperative reference dot product. The warp is split in groups of
// G = 16 lanes (AVX-512 rounding) or 8 lanes (AVX2, portable); each group
// computes x . cg for its own centroid pointer cg; every lane of the group
// returns the group's value. Must be called by all 32 lanes.
template <typename T>
EMB_DEV float group_dot_ref(int match, const T* x, const float* cg, int d, int lane) {
    if (match == kMatchAvx512) {
        int l = lane & 15;
        float acc = 0.0f;
        int dr = (d + 15) & ~15;
        for (int i = l; i < dr; i += 16) {
            float a = i < d ? to_f32(x[i]) : 0.0f, b = i < d ? cg[i] : 0.0f;
            acc = __fmaf_rn(a, b, acc);
        }
        // Lane l holds acc[l]; xor 8,4,2,1 is the tree of _mm512_reduce_add_ps.
        acc = __fadd_rn(acc, __shfl_xor_sync(kFull, acc, 8));
        acc = __fadd_rn(acc, __shfl_xor_sync(kFull, acc, 4));
        acc = __fadd_rn(acc, __shfl_xor_sync(kFull, acc, 2));
        acc = __fadd_rn(acc, __shfl_xor_sync(kFull, acc, 1));
        return acc;
    } else if (match == kMatchAvx2) {
        int l = lane & 7;
        int body = d & ~7;
        float acc = 0.0f;
        for (int i = l; i < body; i += 8) acc = __fmaf_rn(to_f32(x[i]), cg[i], acc);
        acc = __fadd_rn(acc, __shfl_xor_sync(kFull, acc, 4));
        acc = __fadd_rn(acc, __shfl_xor_sync(kFull, acc, 2));
        acc = __fadd_rn(acc, __shfl_xor_sync(kFull, acc, 1));
        for (int i = body; i < d; i++) acc = __fadd_rn(acc, __fmul_rn(to_f32(x[i]), cg[i]));
        return acc;
    } else {
        int l = lane & 7;
        int body = d & ~7;
        float acc = 0.0f;
        for (int i = l; i < body; i += 8) acc = __fadd_rn(acc, __fmul_rn(to_f32(x[i]), cg[i]));
        float s = -0.0f;
        int base = lane & ~7;
#pragma unroll
        for (int q = 0; q < 8; q++) s = __fadd_rn(s, __shfl_sync(kFull, acc, base | q));
        float tail = -0.0f;
        for (int i = body; i < d; i++) tail = __fadd_rn(tail, __fmul_rn(to_f32(x[i]), cg[i]));
        return __fadd_rn(s, tail);
    }
}

// set_centroids (src/cpu.rs:84-93): norms_j = sqnorm_ref(c_j); bounds for the
// certification; optionally the BF16 hi/lo split (hi = bf16(c), lo = bf16(c - hi)),
// written K-major into `split` with row stride `kpad` (hi at column t, lo at column kpad/2 + t).
// One warp per centroid.
__global__ void k_prep_centroids(const float* __restrict__ c, int k, int d, float* __restrict__ norms,
                                 Bounds* __restrict__ bounds, __nv_bfloat16* __restrict__ hi,
                                 __nv_bfloat16* __restrict__ lo, int kpad) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (warp >= k) return;
    const float* cj = c + (size_t)warp * d;
    float nrm = warp_sqnorm_ref(cj, d, lane);
    float ss = 0.0f, ssh = 0.0f, ssd = 0.0f;
    for (int i = lane; i < kpad; i += 32) {
        float v = i < d ? cj[i] : 0.0f;
        ss = __fmaf_ru(v, v, ss);
        ssd = bf16_resid_sq(v, ssd);
        if (hi) {
            __nv_bfloat16 h = __float2bfloat16_rn(v);
            float hf = __bfloat162float(h);
            __nv_bfloat16 l = __float2bfloat16_rn(v - hf);
            hi[(size_t)warp * kpad + i] = h;
            lo[(size_t)warp * kpad + i] = l;
            ssh = __fmaf_ru(hf, hf, ssh);
        }
    }
    for (int o = 16; o; o >>= 1) {
        ss = __fadd_ru(ss, __shfl_xor_sync(kFull, ss, o));
        ssh = __fadd_ru(ssh, __shfl_xor_sync(kFull, ssh, o));
        ssd = __fadd_ru(ssd, __shfl_xor_sync(kFull, ssd, o));
    }
    if (lane == 0) {
        norms[warp] = nrm;
        atomic_max_pos(&bounds->cmax, __fmul_ru(__fsqrt_ru(ss), 1.0000005f));
        atomic_max_pos(&bounds->nmax, fabsf(nrm));
        atomic_max_pos(&bounds->cmax_hi, __fmul_ru(__fsqrt_ru(ssh), 1.0000005f));
        atomic_max_pos(&bounds->dmax, __fmul_ru(__fsqrt_ru(ssd), 1.0000005f));
    }
}

__global__ void k_fill(float* __restrict__ p, int n, float v) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

// set_bias (src/cpu.rs:95-99): norms_j += bias_j, and refresh nmax.
__global__ void k_add_bias(float* __restrict__ norms, const float* __restrict__ bias, int k, Bounds* bounds) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= k) return;
    float v = __fadd_rn(norms[j], bias[j]);
    norms[j] = v;
    atomic_max_pos(&bounds->nmax, fabsf(v));
}

// The certify decision for one row, given the exact re-scores' dot products a1,
// a2 (candidates j1, j2) and |x|^2: true when the row is certified (its label and
// distance written), else false with the refine pass's threshold in *theta_out.
EMB_DEV bool certify_decide(int row, const Top2& t, uint32_t j1, uint32_t j2, float a1, float a2, float xn, int k,
                            const float* __restrict__ norms, const Bounds* __restrict__ bounds, float ka, float kb,
                            uint32_t* __restrict__ labels, float* __restrict__ dist,
                            const int* __restrict__ fast_err, float ka2, float kb2,
                            const float2* __restrict__ row_bounds, float* theta_out, float kr = 0.0f,
                            float xr = 0.0f) {
    bool ok = t.i1 < (uint32_t)k && (k < 2 || t.i2 < (uint32_t)k);
    const float s1 = score_ref(norms[j1], a1);
    float sb = s1;
    uint32_t jb = j1;
    if (t.i2 < (uint32_t)k) {
        const float s2 = score_ref(norms[j2], a2);
        if (lex_less(s2, j2, sb, jb)) {
            sb = s2;
            jb = j2;
        }
    }
    if (ok && k > 2) {
        const float xnorm = __fmul_ru(__fsqrt_ru(fmaxf(xn, 0.0f)), 1.0000005f);
        const float cm = row_bounds ? row_bounds[row].x : bounds->cmax;
        float E = __fadd_ru(__fmul_ru(__fmul_ru(ka, xnorm), cm),
                            __fmul_ru(kb, row_bounds ? row_bounds[row].y : bounds->nmax));
        // Single-term BF16: x.c - bf16(x).bf16(c) = (x - bf16(x)).c + bf16(x).(c - bf16(c)),
        // at most xr cmax + (|x| + xr) dmax, with xr = |x - bf16(x)| of this row.
        if (kr > 0.0f)
            E = __fadd_ru(E, __fmul_ru(kr, __fadd_ru(__fmul_ru(xr, cm), __fmul_ru(__fadd_ru(xnorm, xr), bounds->dmax))));
        const float thr = __fsub_rd(t.s2, E);
        ok = isfinite(E) && sb < thr;  // NaN-safe: any NaN fails
    }
    if (ok && !(sb < __int_as_float(0x7f800000))) ok = false;  // non-finite best: re-search
    if (fast_err && *fast_err) ok = false;  // the fast kernel gave up: trust nothing it wrote
    if (ok) {
        labels[row] = jb;
        dist[row] = fmaxf(__fadd_rn(sb, xn), 0.0f);
        return true;
    }
    // Threshold for the refine pass: the reference's best j* has s_j* <= sb, so
    // its refine-pass score is <= sb + E2. Non-finite: no candidates, so the row
    // is searched exhaustively.
    float theta = __int_as_float(0x7fc00000);
    if (t.i1 < (uint32_t)k && sb < __int_as_float(0x7f800000) && sb > -__int_as_float(0x7f800000)) {
        const float xnorm = __fmul_ru(__fsqrt_ru(fmaxf(xn, 0.0f)), 1.0000005f);
        const float E2 = __fadd_ru(__fmul_ru(__fmul_ru(ka2, xnorm), bounds->cmax), __fmul_ru(kb2, bounds->nmax));
        const float th = __fadd_ru(sb, E2);
        if (isfinite(th)) theta = th;
    }
    *theta_out = theta;
    return false;
}

// Certification of the fast top-2 (one warp per row).
//   part_s/part_i: nsplit partial top-2 lists per row, [split][row][2].
//   The approximate score of every centroid is within E of its reference
//   score, E = ka * |x| * cmax + kb * nmax. With j1, j2 re-scored exactly and
//   b their better one, every other centroid j has s_j >= s^_2 - E; if
//   b < s^_2 - E no other centroid can reach b, so b is the reference's label.
//   Rows that fail go to the exact re-search list.
template <typename T>
__global__ void k_certify(const T* __restrict__ x, const uint32_t* __restrict__ gather, int m, int d,
                          const float* __restrict__ c, const float* __restrict__ norms, int k,
                          const float* __restrict__ part_s, const uint32_t* __restrict__ part_i, int nsplit,
                          const Bounds* __restrict__ bounds, float ka, float kb, int match,
                          uint32_t* __restrict__ labels, float* __restrict__ dist,
                          uint32_t* __restrict__ redo_rows, uint32_t* __restrict__ redo_count,
                          uint32_t* __restrict__ cert_count, const int* __restrict__ fast_err,
                          float* __restrict__ redo_theta, float ka2, float kb2,
                          const float2* __restrict__ row_bounds = nullptr, float kr = 0.0f) {
    int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (row >= m) return;
    size_t src = gather ? gather[row] : (size_t)row;
    const T* xr = x + src * (size_t)d;

    Top2 t;
    t.init();
    for (int s = 0; s < nsplit; s++) {
        size_t o = ((size_t)s * m + row) * 2;
        t.push(part_s[o], part_i[o]);
        t.push(part_s[o + 1], part_i[o + 1]);
    }
    float xn = warp_sqnorm_ref(xr, d, lane);
    // Exact re-score of the two candidates: group 0 takes j1, group 1 takes j2.
    uint32_t j1 = t.i1 < (uint32_t)k ? t.i1 : 0u;
    uint32_t j2 = t.i2 < (uint32_t)k ? t.i2 : j1;
    int gsz = match == kMatchAvx512 ? 16 : 8;
    uint32_t jg = (lane / gsz) == 1 ? j2 : j1;
    float dg = group_dot_ref(match, xr, c + (size_t)jg * d, d, lane);
    float d1 = __shfl_sync(kFull, dg, 0);
    float d2 = __shfl_sync(kFull, dg, gsz);
    float xres = 0.0f;  // |x - bf16(x)|, upper-rounded (single-term BF16 bound)
    if (kr > 0.0f) {
        float acc = 0.0f;
        for (int i = lane; i < d; i += 32) acc = bf16_resid_sq(to_f32(xr[i]), acc);
        for (int o = 16; o; o >>= 1) acc = __fadd_ru(acc, __shfl_xor_sync(kFull, acc, o));
        xres = __fmul_ru(__fsqrt_ru(acc), 1.0000005f);
    }
    if (lane != 0) return;
    float theta = 0.0f;
    if (certify_decide(row, t, j1, j2, d1, d2, xn, k, norms, bounds, ka, kb, labels, dist, fast_err, ka2, kb2,
                       row_bounds, &theta, kr, xres)) {
        atomicAdd(cert_count, 1u);
    } else {
        const uint32_t slot = atomicAdd(redo_count, 1u);
        redo_rows[slot] = (uint32_t)row;
        redo_theta[slot] = theta;
    }
}

// Warp-wide tally of the certify decisions (all 32 lanes call it): one atomic
// for the warp's certified rows, one reservation of refine-list slots for its
// uncertified rows. The list's order is immaterial (each row settles alone).
EMB_DEV void certify_tally(bool ok, bool redo, int row, float theta, uint32_t* __restrict__ cert_count,
                           uint32_t* __restrict__ redo_count, uint32_t* __restrict__ redo_rows,
                           float* __restrict__ redo_theta) {
    const int lane = threadIdx.x & 31;
    const unsigned okb = __ballot_sync(kFull, ok);
    if (lane == 0 && okb) atomicAdd(cert_count, (unsigned)__popc(okb));
    const unsigned rb = __ballot_sync(kFull, redo);
    if (!rb) return;
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(redo_count, (unsigned)__popc(rb));
    base = __shfl_sync(kFull, base, 0);
    if (redo) {
        const uint32_t slot = base + (uint32_t)__popc(rb & ((1u << lane) - 1u));
        redo_rows[slot] = (uint32_t)row;
        redo_theta[slot] = theta;
    }
}

// k_certify specialised to the AVX-512 rounding (the default): one half-warp
// per row, so a warp certifies two rows, and one pass over the row computes its
// sqnorm lanes and both candidates' 16 FMA lanes. Same decisions and outputs as
// k_certify with match = AVX-512. row_bounds (optional): per row, (max |c|, max |norm|)
// over the centroids whose approximate scores were compared, in place of the
// bounds over all k; the refine threshold keeps the bounds over all k.
template <typename T>
__global__ void k_certify16(const T* __restrict__ x, const uint32_t* __restrict__ gather, int m, int d,
                            const float* __restrict__ c, const float* __restrict__ norms, int k,
                            const float* __restrict__ part_s, const uint32_t* __restrict__ part_i, int nsplit,
                            const Bounds* __restrict__ bounds, float ka, float kb,
                            uint32_t* __restrict__ labels, float* __restrict__ dist,
                            uint32_t* __restrict__ redo_rows, uint32_t* __restrict__ redo_count,
                            uint32_t* __restrict__ cert_count, const int* __restrict__ fast_err,
                            float* __restrict__ redo_theta, float ka2, float kb2,
                            const float2* __restrict__ row_bounds = nullptr, float kr = 0.0f) {
    const int lane = threadIdx.x & 31, l = lane & 15, half = lane >> 4;
    const int row = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 2 + half;
    const bool live = row < m;
    const int r = live ? row : m - 1;  // dead half-warps mirror a live row and write nothing
    const size_t src = gather ? gather[r] : (size_t)r;
    const T* xr = x + src * (size_t)d;
    Top2 t;
    t.init();
    for (int s = 0; s < nsplit; s++) {
        const size_t o = ((size_t)s * m + r) * 2;
        t.push(part_s[o], part_i[o]);
        t.push(part_s[o + 1], part_i[o + 1]);
    }
    const uint32_t j1 = t.i1 < (uint32_t)k ? t.i1 : 0u;
    const uint32_t j2 = t.i2 < (uint32_t)k ? t.i2 : j1;
    const float* c1 = c + (size_t)j1 * d;
    const float* c2 = c + (size_t)j2 * d;
    const int body = d & ~15, dr = (d + 15) & ~15;
    float sq = 0.0f, a1 = 0.0f, a2 = 0.0f, rs = 0.0f;
    for (int i = l; i < dr; i += 16) {
        const bool in = i < d;
        const float xv = in ? to_f32(xr[i]) : 0.0f;
        if (i < body) sq = __fadd_rn(sq, __fmul_rn(xv, xv));
        if (kr > 0.0f) rs = bf16_resid_sq(xv, rs);
        a1 = __fmaf_rn(xv, in ? c1[i] : 0.0f, a1);
        a2 = __fmaf_rn(xv, in ? c2[i] : 0.0f, a2);
    }
#pragma unroll
    for (int o = 8; o; o >>= 1) {
        a1 = __fadd_rn(a1, __shfl_xor_sync(kFull, a1, o));
        a2 = __fadd_rn(a2, __shfl_xor_sync(kFull, a2, o));
        rs = __fadd_ru(rs, __shfl_xor_sync(kFull, rs, o));
    }
    float xn = -0.0f;
    const int base = half * 16;
#pragma unroll
    for (int q = 0; q < 16; q++) xn = __fadd_rn(xn, __shfl_sync(kFull, sq, base + q));
    float tail = -0.0f;
    for (int i = body; i < d; i++) {
        const float v = to_f32(xr[i]);
        tail = __fadd_rn(tail, __fmul_rn(v, v));
    }
    xn = __fadd_rn(xn, tail);
    bool ok = false, redo = false;
    float theta = 0.0f;
    if (live && l == 0) {
        ok = certify_decide(row, t, j1, j2, a1, a2, xn, k, norms, bounds, ka, kb, labels, dist, fast_err, ka2, kb2,
                              row_bounds, &theta, kr, __fmul_ru(__fsqrt_ru(rs), 1.0000005f));
        redo = !ok;
    }
    certify_tally(ok, redo, row, theta, cert_count, redo_count, redo_rows, redo_theta);
}

// k_certify16 with four threads per row (eight rows per warp), for f32 rows with
// d % 16 == 0: thread q keeps AVX-512 lanes 4q .. 4q+3 and loads them as float4.
// The lane sums combine in the reference's tree order (lane l with l^8, l^4,
// l^2, l^1: threads q^2 and q^1, then in registers), and |x|^2 adds the 16 lane
// partials in lane order, so every value equals k_certify16's.
__global__ void k_certify16v(const float* __restrict__ x, const uint32_t* __restrict__ gather, int m, int d,
                             const float* __restrict__ c, const float* __restrict__ norms, int k,
                             const float* __restrict__ part_s, const uint32_t* __restrict__ part_i, int nsplit,
                             const Bounds* __restrict__ bounds, float ka, float kb, uint32_t* __restrict__ labels,
                             float* __restrict__ dist, uint32_t* __restrict__ redo_rows,
                             uint32_t* __restrict__ redo_count, uint32_t* __restrict__ cert_count,
                             const int* __restrict__ fast_err, float* __restrict__ redo_theta, float ka2, float kb2,
                             const float2* __restrict__ row_bounds = nullptr, float kr = 0.0f) {
    const int lane = threadIdx.x & 31, q = lane & 3;
    const int row = (int)(((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 2);
    const bool live = row < m;
    const int r = live ? row : m - 1;  // dead quarter-warps mirror a live row and write nothing
    const size_t src = gather ? gather[r] : (size_t)r;
    const float* xr = x + src * (size_t)d;
    Top2 t;
    t.init();
    for (int s = 0; s < nsplit; s++) {
        const size_t o = ((size_t)s * m + r) * 2;
        t.push(part_s[o], part_i[o]);
        t.push(part_s[o + 1], part_i[o + 1]);
    }
    const uint32_t j1 = t.i1 < (uint32_t)k ? t.i1 : 0u;
    const uint32_t j2 = t.i2 < (uint32_t)k ? t.i2 : j1;
    const float* c1 = c + (size_t)j1 * d;
    const float* c2 = c + (size_t)j2 * d;
    float sq[4] = {0.0f, 0.0f, 0.0f, 0.0f}, p1[4] = {0.0f, 0.0f, 0.0f, 0.0f}, p2[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    float rs = 0.0f;
    for (int i = 4 * q; i < d; i += 16) {
        const float4 xv = *reinterpret_cast<const float4*>(xr + i);
        const float4 u = *reinterpret_cast<const float4*>(c1 + i);
        const float4 w = *reinterpret_cast<const float4*>(c2 + i);
        const float xs[4] = {xv.x, xv.y, xv.z, xv.w}, us[4] = {u.x, u.y, u.z, u.w}, ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
        for (int j = 0; j < 4; j++) {
            sq[j] = __fadd_rn(sq[j], __fmul_rn(xs[j], xs[j]));
            p1[j] = __fmaf_rn(xs[j], us[j], p1[j]);
            p2[j] = __fmaf_rn(xs[j], ws[j], p2[j]);
            if (kr > 0.0f) rs = bf16_resid_sq(xs[j], rs);
        }
    }
    rs = __fadd_ru(rs, __shfl_xor_sync(kFull, rs, 2));
    rs = __fadd_ru(rs, __shfl_xor_sync(kFull, rs, 1));
#pragma unroll
    for (int j = 0; j < 4; j++) {  // lane l with l^8, then l^4
        p1[j] = __fadd_rn(p1[j], __shfl_xor_sync(kFull, p1[j], 2));
        p2[j] = __fadd_rn(p2[j], __shfl_xor_sync(kFull, p2[j], 2));
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
        p1[j] = __fadd_rn(p1[j], __shfl_xor_sync(kFull, p1[j], 1));
        p2[j] = __fadd_rn(p2[j], __shfl_xor_sync(kFull, p2[j], 1));
    }
    // l^2 and l^1 within the thread
    const float a1 = __fadd_rn(__fadd_rn(p1[0], p1[2]), __fadd_rn(p1[1], p1[3]));
    const float a2 = __fadd_rn(__fadd_rn(p2[0], p2[2]), __fadd_rn(p2[1], p2[3]));
    float xn = -0.0f;
    const int base = lane & ~3;
#pragma unroll
    for (int qq = 0; qq < 4; qq++)
#pragma unroll
        for (int j = 0; j < 4; j++) xn = __fadd_rn(xn, __shfl_sync(kFull, sq[j], base + qq));
    bool ok = false, redo = false;
    float theta = 0.0f;
    if (live && q == 0) {
        ok = certify_decide(row, t, j1, j2, a1, a2, xn, k, norms, bounds, ka, kb, labels, dist, fast_err, ka2, kb2,
                              row_bounds, &theta, kr, __fmul_ru(__fsqrt_ru(rs), 1.0000005f));
        redo = !ok;
    }
    certify_tally(ok, redo, row, theta, cert_count, redo_count, redo_rows, redo_theta);
}

// Exact re-score of the refine pass's candidates (one warp per refined row):
// the reference's label is the lowest-index minimum of the exact scores of the
// candidates, because every centroid whose exact score could reach sb was
// collected. Rows with no candidates or more than cap go to the exhaustive list.
template <typename T>
__global__ void k_rescore_cands(const T* __restrict__ x, const uint32_t* __restrict__ gather, int d,
                                const float* __restrict__ c, const float* __restrict__ norms, int match,
                                const uint32_t* __restrict__ redo_rows, const uint32_t* __restrict__ redo_count,
                                const uint32_t* __restrict__ cand, const uint32_t* __restrict__ cand_count, int cap,
                                const int* __restrict__ refine_err, uint32_t* __restrict__ labels,
                                float* __restrict__ dist, uint32_t* __restrict__ redo2_rows,
                                uint32_t* __restrict__ redo2_count) {
    int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (i >= (int)*redo_count) return;
    uint32_t row = redo_rows[i];
    uint32_t cnt = cand_count[i];
    if (cnt == 0 || cnt > (uint32_t)cap || *refine_err) {
        if (lane == 0) redo2_rows[atomicAdd(redo2_count, 1u)] = row;
        return;
    }
    size_t src = gather ? gather[row] : (size_t)row;
    const T* xr = x + src * (size_t)d;
    const int gsz = match == kMatchAvx512 ? 16 : 8;
    const int ngroups = 32 / gsz, g = lane / gsz;
    float best = __int_as_float(0x7f800000);
    uint32_t lab = 0xffffffffu;
    for (uint32_t c0 = 0; c0 < cnt; c0 += ngroups) {
        uint32_t ci = c0 + g < cnt ? c0 + g : cnt - 1;
        uint32_t j = cand[(size_t)i * cap + ci];
        float dg = group_dot_ref(match, xr, c + (size_t)j * d, d, lane);
        float s = score_ref(norms[j], dg);
        if (lex_less(s, j, best, lab)) {
            best = s;
            lab = j;
        }
    }
    for (int q = 1; q < ngroups; q++) {
        float ob = __shfl_sync(kFull, best, q * gsz);
        uint32_t ol = __shfl_sync(kFull, lab, q * gsz);
        if (lex_less(ob, ol, best, lab)) {
            best = ob;
            lab = ol;
        }
    }
    float xn = warp_sqnorm_ref(xr, d, lane);
    if (lane == 0) {
        if (best < __int_as_float(0x7f800000)) {
            labels[row] = lab;
            dist[row] = fmaxf(__fadd_rn(best, xn), 0.0f);
        } else {
            redo2_rows[atomicAdd(redo2_count, 1u)] = row;
        }
    }
}

// Exhaustive exact search with one CTA per row (persistent over the list):
// 8 warps x (32 / G) lane groups score interleaved centroids, two per group in
// flight, then the groups are merged in (score, index) order.
template <typename T>
__global__ void __launch_bounds__(256) k_research_cta(const T* __restrict__ x, const uint32_t* __restrict__ gather,
                                                      int d, const float* __restrict__ c,
                                                      const float* __restrict__ norms, int k, int match,
                                                      const uint32_t* __restrict__ rows,
                                                      const uint32_t* __restrict__ count,
                                                      uint32_t* __restrict__ labels, float* __restrict__ dist) {
    __shared__ float sb[32];
    __shared__ uint32_t sl[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int gsz = match == kMatchAvx512 ? 16 : 8;
    const int gpw = 32 / gsz;                 // groups per warp
    const int G = 8 * gpw;                    // groups per CTA
    const int g = warp * gpw + lane / gsz;    // this lane's group
    const uint32_t n = *count;
    for (uint32_t r = blockIdx.x; r < n; r += gridDim.x) {
        uint32_t row = rows[r];
        size_t src = gather ? gather[row] : (size_t)row;
        const T* xr = x + src * (size_t)d;
        float best = __int_as_float(0x7f800000);
        uint32_t lab = 0;
        for (int j0 = 0; j0 < k; j0 += 2 * G) {
            int ja = j0 + g, jb = j0 + G + g;
            int jac = ja < k ? ja : k - 1, jbc = jb < k ? jb : k - 1;
            float da = group_dot_ref(match, xr, c + (size_t)jac * d, d, lane);
            float db = group_dot_ref(match, xr, c + (size_t)jbc * d, d, lane);
            if (ja < k) {
                float s = score_ref(norms[ja], da);
                if (s < best) {
                    best = s;
                    lab = (uint32_t)ja;
                }
            }
            if (jb < k) {
                float s = score_ref(norms[jb], db);
                if (s < best) {
                    best = s;
                    lab = (uint32_t)jb;
                }
            }
        }
        // A group that never beat +inf reports (inf, 0): it loses to any finite
        // score, and if every group is at +inf the reference's label 0 results.
        if ((lane & (gsz - 1)) == 0) {
            sb[g] = best;
            sl[g] = best < __int_as_float(0x7f800000) ? lab : 0u;
        }
        __syncthreads();
        if (warp == 0) {
            float rb = __int_as_float(0x7f800000);
            uint32_t rl = 0;
            for (int q = 0; q < G; q++)
                if (sb[q] < __int_as_float(0x7f800000) && lex_less(sb[q], sl[q], rb, rl)) {
                    rb = sb[q];
                    rl = sl[q];
                }
            float xn = warp_sqnorm_ref(xr, d, lane);
            if (lane == 0) {
                labels[row] = rl;
                dist[row] = fmaxf(__fadd_rn(rb, xn), 0.0f);
            }
        }
        __syncthreads();
    }
}

// Exhaustive exact search spread over many CTAs per row: CTA p takes row
// p / slices and the centroids [span (p % slices), span (p % slices + 1)), scores
// them as k_research_cta does, and folds its best into keys[r] with a 64-bit
// atomicMin on (order-preserving score bits, index), so the lowest index wins
// exact ties as in the reference's strict-< scan. keys start at (+inf, 0): a
// row whose scores never beat +inf keeps label 0, the reference's result.
EMB_DEV unsigned long long research_key(float s, uint32_t j) {
    const uint32_t b = __float_as_uint(__fadd_rn(s, 0.0f));  // -0 -> +0: the two compare equal
    const uint32_t o = (b & 0x80000000u) ? ~b : (b | 0x80000000u);
    return ((unsigned long long)o << 32) | j;
}
EMB_DEV float research_key_score(unsigned long long key) {
    const uint32_t o = (uint32_t)(key >> 32);
    return __uint_as_float((o & 0x80000000u) ? (o & 0x7fffffffu) : ~o);
}

__global__ void k_research_keys_init(unsigned long long* __restrict__ keys, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) keys[i] = ((unsigned long long)0xff800000u << 32);  // (+inf, label 0)
}

template <typename T>
__global__ void __launch_bounds__(256) k_research_split(const T* __restrict__ x, const uint32_t* __restrict__ gather,
                                                        int d, const float* __restrict__ c,
                                                        const float* __restrict__ norms, int k, int match,
                                                        const uint32_t* __restrict__ rows,
                                                        const uint32_t* __restrict__ count, int slices, int span,
                                                        unsigned long long* __restrict__ keys) {
    __shared__ unsigned long long sk[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int gsz = match == kMatchAvx512 ? 16 : 8;
    const int gpw = 32 / gsz;
    const int G = 8 * gpw;
    const int g = warp * gpw + lane / gsz;
    const size_t total = (size_t)*count * (size_t)slices;
    for (size_t p = blockIdx.x; p < total; p += gridDim.x) {
        const uint32_t r = (uint32_t)(p / slices);
        const int j_lo = (int)(p % slices) * span;
        const int j_hi = j_lo + span < k ? j_lo + span : k;
        const uint32_t row = rows[r];
        const size_t src = gather ? gather[row] : (size_t)row;
        const T* xr = x + src * (size_t)d;
        unsigned long long best = ~0ull;
        for (int j0 = j_lo; j0 < j_hi; j0 += 2 * G) {
            const int ja = j0 + g, jb = j0 + G + g;
            const int jac = ja < j_hi ? ja : j_hi - 1, jbc = jb < j_hi ? jb : j_hi - 1;
            const float da = group_dot_ref(match, xr, c + (size_t)jac * d, d, lane);
            const float db = group_dot_ref(match, xr, c + (size_t)jbc * d, d, lane);
            if (ja < j_hi) {
                const float s = score_ref(norms[ja], da);
                if (s < __int_as_float(0x7f800000)) best = min(best, research_key(s, (uint32_t)ja));
            }
            if (jb < j_hi) {
                const float s = score_ref(norms[jb], db);
                if (s < __int_as_float(0x7f800000)) best = min(best, research_key(s, (uint32_t)jb));
            }
        }
        if ((lane & (gsz - 1)) == 0) sk[g] = best;
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned long long b = ~0ull;
            for (int q = 0; q < G; q++) b = min(b, sk[q]);
            if (b != ~0ull) atomicMin(&keys[r], b);
        }
        __syncthreads();
    }
}

// Labels and distances of the split search: dist = max(best + sqnorm(x), 0). One warp per row.
template <typename T>
__global__ void k_research_finish(const T* __restrict__ x, const uint32_t* __restrict__ gather, int d,
                                  const uint32_t* __restrict__ rows, const uint32_t* __restrict__ count,
                                  const unsigned long long* __restrict__ keys, uint32_t* __restrict__ labels,
                                  float* __restrict__ dist) {
    const uint32_t r = (uint32_t)(((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (r >= *count) return;
    const uint32_t row = rows[r];
    const size_t src = gather ? gather[row] : (size_t)row;
    const float xn = warp_sqnorm_ref(x + src * (size_t)d, d, lane);
    if (lane == 0) {
        const unsigned long long key = keys[r];
        labels[row] = (uint32_t)(key & 0xffffffffu);
        dist[row] = fmaxf(__fadd_rn(research_key_score(key), xn), 0.0f);
    }
}


}  // namespace emb
