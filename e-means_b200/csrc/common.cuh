// Shared device helpers of the B200 e-means engine.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define EMB_DEV __device__ __forceinline__

namespace emb {

constexpr int kF32 = 0, kI8 = 1, kU8 = 2;
constexpr int kMatchAvx512 = 0, kMatchAvx2 = 1, kMatchPortable = 2;

template <typename T> EMB_DEV float to_f32(T v) { return (float)v; }
template <> EMB_DEV float to_f32<float>(float v) { return v; }

// ---- the reference's f32 arithmetic, restated with non-contracting intrinsics

// sqnorm, src/cpu.rs:169-180: lane l of 16 accumulates v[i]*v[i] for i = l mod 16
// (multiply, then add: Rust does not fuse), then the 16 lanes and the tail are
// summed sequentially from -0.0.
template <typename T>
EMB_DEV float sqnorm_ref(const T* v, int d) {
    float acc[16];
#pragma unroll
    for (int l = 0; l < 16; l++) acc[l] = 0.0f;
    int body = d & ~15;
    for (int i = 0; i < body; i += 16) {
#pragma unroll
        for (int l = 0; l < 16; l++) {
            float a = to_f32(v[i + l]);
            acc[l] = __fadd_rn(acc[l], __fmul_rn(a, a));
        }
    }
    float s = -0.0f;
#pragma unroll
    for (int l = 0; l < 16; l++) s = __fadd_rn(s, acc[l]);
    float t = -0.0f;
    for (int i = body; i < d; i++) {
        float a = to_f32(v[i]);
        t = __fadd_rn(t, __fmul_rn(a, a));
    }
    return __fadd_rn(s, t);
}

// Score of one row against one centroid in the reference's rounding:
// norms[j] - 2 * dot (src/cpu.rs:148), where dot follows the selected kernel:
//   AVX-512 (src/cpu.rs:200-231): 16 FMA lanes (i = l mod 16), masked tail, tree (l,l+8),(l,l+4),(l,l+2),(0,1)
//   AVX2    (src/cpu.rs:233-266): 8 FMA lanes over d & ~7, tree (l,l+4),(l,l+2),(0,1), then the tail
//                                  added one product at a time (multiply, add)
//   portable(src/cpu.rs:182-198): 8 lanes of multiply-then-add over d/8*8, lanes summed in order,
//                                  plus the tail's products summed in order
// Used by the serial (single-thread) re-score of a few candidates.
template <typename T>
EMB_DEV float dot_ref(int match, const T* x, const float* c, int d) {
    if (match == kMatchAvx512) {
        float acc[16];
#pragma unroll
        for (int l = 0; l < 16; l++) acc[l] = 0.0f;
        for (int i = 0; i < d; i += 16) {
#pragma unroll
            for (int l = 0; l < 16; l++) {
                // Masked tail lanes load zeros (src/cpu.rs:217-227).
                float a = (i + l < d) ? to_f32(x[i + l]) : 0.0f, b = (i + l < d) ? c[i + l] : 0.0f;
                acc[l] = __fmaf_rn(a, b, acc[l]);
            }
        }
        float t8[8], t4[4];
#pragma unroll
        for (int l = 0; l < 8; l++) t8[l] = __fadd_rn(acc[l], acc[l + 8]);
#pragma unroll
        for (int l = 0; l < 4; l++) t4[l] = __fadd_rn(t8[l], t8[l + 4]);
        return __fadd_rn(__fadd_rn(t4[0], t4[2]), __fadd_rn(t4[1], t4[3]));
    } else if (match == kMatchAvx2) {
        float acc[8];
#pragma unroll
        for (int l = 0; l < 8; l++) acc[l] = 0.0f;
        int body = d & ~7;
        for (int i = 0; i < body; i += 8) {
#pragma unroll
            for (int l = 0; l < 8; l++) acc[l] = __fmaf_rn(to_f32(x[i + l]), c[i + l], acc[l]);
        }
        float t4[4];
#pragma unroll
        for (int l = 0; l < 4; l++) t4[l] = __fadd_rn(acc[l], acc[l + 4]);
        float r = __fadd_rn(__fadd_rn(t4[0], t4[2]), __fadd_rn(t4[1], t4[3]));
        for (int i = body; i < d; i++) r = __fadd_rn(r, __fmul_rn(to_f32(x[i]), c[i]));
        return r;
    } else {
        float acc[8];
#pragma unroll
        for (int l = 0; l < 8; l++) acc[l] = 0.0f;
        int body = d & ~7;
        for (int i = 0; i < body; i += 8) {
#pragma unroll
            for (int l = 0; l < 8; l++) acc[l] = __fadd_rn(acc[l], __fmul_rn(to_f32(x[i + l]), c[i + l]));
        }
        float s = -0.0f;
#pragma unroll
        for (int l = 0; l < 8; l++) s = __fadd_rn(s, acc[l]);
        float tail = -0.0f;
        for (int i = body; i < d; i++) tail = __fadd_rn(tail, __fmul_rn(to_f32(x[i]), c[i]));
        return __fadd_rn(s, tail);
    }
}

EMB_DEV float score_ref(float norm, float dot) { return __fsub_rn(norm, __fmul_rn(2.0f, dot)); }

// (score, index) lexicographic order: lower score, then lower index.
EMB_DEV bool lex_less(float s, uint32_t i, float t, uint32_t j) { return s < t || (s == t && i < j); }

// Running top-2 of (score, index) pairs in lexicographic order.
struct Top2 {
    float s1, s2;
    uint32_t i1, i2;
    EMB_DEV void init() {
        s1 = s2 = __int_as_float(0x7f800000);
        i1 = i2 = 0xffffffffu;
    }
    EMB_DEV void push(float s, uint32_t i) {
        if (lex_less(s, i, s2, i2)) {
            if (lex_less(s, i, s1, i1)) {
                s2 = s1;
                i2 = i1;
                s1 = s;
                i1 = i;
            } else {
                s2 = s;
                i2 = i;
            }
        }
    }
    // Branch-free insertion for an approximate search: strict <, so the earlier
    // index keeps a tie and +inf / NaN scores are never inserted. The exact
    // certification and re-search settle every row whatever the partials are,
    // so only their values as bounds matter, not the tie order.
    EMB_DEV void push_fast(float s, uint32_t i) {
        const bool b1 = s < s1, b2 = s < s2;
        s2 = b1 ? s1 : (b2 ? s : s2);
        i2 = b1 ? i1 : (b2 ? i : i2);
        s1 = b1 ? s : s1;
        i1 = b1 ? i : i1;
    }
    EMB_DEV void merge(const Top2& o) {
        push(o.s1, o.i1);
        push(o.s2, o.i2);
    }
    EMB_DEV void merge_shfl_xor(int mask) {
        Top2 o;
        o.s1 = __shfl_xor_sync(0xffffffffu, s1, mask);
        o.s2 = __shfl_xor_sync(0xffffffffu, s2, mask);
        o.i1 = __shfl_xor_sync(0xffffffffu, i1, mask);
        o.i2 = __shfl_xor_sync(0xffffffffu, i2, mask);
        merge(o);
    }
};

}  // namespace emb
