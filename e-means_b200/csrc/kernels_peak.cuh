// FP32 SIMT throughput microbenchmark: the measured denominator of the FP32
// search's roofline (k_assign_simt). Each thread runs 8 independent FMA chains
// (scalar fma.rn.f32, or fma.rn.f32x2 on register pairs), enough to cover the
// FMA latency at a full SM's worth of warps.
#pragma once
#include "common.cuh"

namespace emb {

template <bool PAIRED>
__global__ void __launch_bounds__(256) k_simt_peak(float* __restrict__ out, int iters, float b, float c) {
    float a[8];
#pragma unroll
    for (int j = 0; j < 8; j++) a[j] = (float)(threadIdx.x + j) * 1e-3f;
    for (int i = 0; i < iters; i++) {
        if (PAIRED) {
#pragma unroll
            for (int j = 0; j < 8; j += 2)
                asm("{\n .reg .b64 ra, rb, rc;\n mov.b64 ra, {%0, %1};\n mov.b64 rb, {%2, %2};\n mov.b64 rc, {%3, %3};\n"
                    " fma.rn.f32x2 ra, ra, rb, rc;\n mov.b64 {%0, %1}, ra;\n}\n"
                    : "+f"(a[j]), "+f"(a[j + 1])
                    : "f"(b), "f"(c));
        } else {
#pragma unroll
            for (int j = 0; j < 8; j++) a[j] = fmaf(a[j], b, c);
        }
    }
    float s = 0.0f;
#pragma unroll
    for (int j = 0; j < 8; j++) s += a[j];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keeps the chains live
}

}  // namespace emb
