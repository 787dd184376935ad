// libemb200: C ABI (include/emb200.h) and host orchestration of the B200
// e-means engine. Every computation runs in the CUDA kernels included below;
// host code only sizes buffers, launches and copies.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <atomic>
#include <cstring>
#include <map>
#include <mutex>
#include <thread>
#include <string>
#include <vector>

#include "../../include/emb200.h"
#include "common.cuh"
#include "host_recipe.hpp"
#include "kernels_exact.cuh"
#include "kernels_i8.cuh"
#include "kernels_simt.cuh"
#include "kernels_tc.cuh"
#include "kernels_tc_i8.cuh"
#include "kernels_tc_grouped.cuh"
#include "kernels_update.cuh"
#include "kernels_mlp.cuh"
#include "kernels_mlp_tc.cuh"
#include "kernels_gemm_tc.cuh"
#include "kernels_proposer.cuh"
#include "kernels_quant.cuh"
#include "kernels_report.cuh"
#include "kernels_peak.cuh"
#include "kernels_peak_tc.cuh"
#include "kernels_batched.cuh"

constexpr int kRefineCap = 32;  // candidates kept per refined row
constexpr size_t kMaxSearchRows = (size_t)1 << 26;  // rows per search pass (32-bit row indexing inside)

using namespace emb;

namespace {

struct Proposer;
void proposer_release(emb200_handle* h);
struct ReportState;
void report_release(emb200_handle* h);

// Device buffer owned by a handle.
template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaError_t ensure(size_t want) {
        if (want <= n && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        cudaError_t e = cudaMalloc((void**)&p, std::max(want, (size_t)1) * sizeof(T));
        if (e == cudaSuccess) n = std::max(want, (size_t)1);
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

// Device state of a training run (filled by emb200_train).
struct TrainState {
    DevBuf<float> usage, sums, pass_sums, batch_dist, alphas, xbatch;
    DevBuf<int> ctl;  // [0] step, [1] epoch, [2] last pass
    DevBuf<double> pass_sums64, keys, scalars, obj, gstream;
    DevBuf<uint32_t> counts, offsets, slot, list, scratch, batch_labels, labels_all, order, didx, unused;
    DevBuf<unsigned long long> pass_counts;
    uint32_t* order_host = nullptr;  // pinned staging of the epoch's row order
    size_t order_host_n = 0;
    void release() {
        if (order_host) cudaFreeHost(order_host);
        order_host = nullptr;
        order_host_n = 0;
        usage.release(); sums.release(); pass_sums.release(); batch_dist.release(); alphas.release(); ctl.release();
        xbatch.release();
        pass_sums64.release(); keys.release(); scalars.release(); obj.release(); gstream.release();
        counts.release(); offsets.release(); slot.release(); list.release(); scratch.release();
        batch_labels.release(); labels_all.release(); order.release(); didx.release(); unused.release();
        pass_counts.release();
    }
};

// Device state of a batched lockstep run (emb200_train_batched).
struct BatchState {
    DevBuf<uint8_t> inst, steps, ctl;
    DevBuf<uint32_t> orders, counts, offsets, slot, list, scratch, blabels, labels_all, didx, unused, part_i, items,
        redo, init, init_off;
    DevBuf<float> alphas, c, norms, usage, sums, bdist, pass_sums, part_s;
    DevBuf<Bounds> bounds;
    DevBuf<unsigned long long> pass_counts, cursor, nsplits;
    DevBuf<double> pass_sums64, obj, gstream, keys;
    void release() {
        inst.release(); steps.release(); ctl.release(); orders.release(); counts.release(); offsets.release();
        slot.release(); list.release(); scratch.release(); blabels.release(); labels_all.release(); didx.release();
        unused.release(); part_i.release(); items.release(); redo.release(); init.release(); init_off.release();
        alphas.release(); c.release(); norms.release(); usage.release(); sums.release(); bdist.release();
        pass_sums.release(); part_s.release(); bounds.release(); pass_counts.release(); cursor.release();
        nsplits.release(); pass_sums64.release(); obj.release(); gstream.release(); keys.release();
    }
};

}  // namespace

struct emb200_handle {
    int device = 0;
    cudaStream_t stream = nullptr;
    emb200_opts opts{};
    std::string err;
    emb200_stats stats{};
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t evk0 = nullptr, evk1 = nullptr;  // around the fast contraction kernel
    int sm_count = 148;

    // centroids
    size_t k = 0, d = 0;
    bool have_centroids = false;
    DevBuf<float> c, norms, bias;
    DevBuf<Bounds> bounds;
    DevBuf<__nv_bfloat16> c_hi, c_lo;  // K-major BF16 split, row stride kpad
    size_t kpad = 0;
    CUtensorMap map_hi{}, map_lo{};  // TMA descriptors of c_hi / c_lo (128B swizzle, 64 x 128 boxes)
    bool maps_ok = false;
    // Half-norms split into BF16 parts for the single-term search that sums the
    // norms inside the contraction ([whole tiles][16], k_prep_nrm16)
    DevBuf<__nv_bfloat16> nrm16;
    DevBuf<int8_t> c8;   // I8 centroids (CpuI8Assigner)
    DevBuf<int16_t> c16; // I16 centroids: round(c * 2^ishift)
    int ishift = 0;      // I16 scale exponent (src/cpu_i8.rs:97)
    DevBuf<long long> off8;  // integer offsets: sum c8^2 or sum c16^2 (+ bias in score units)
    bool bias_set = false;
    double bias_absmax = 0.0;  // largest |bias| added since set_centroids (inf: unknown, device-computed)
    CUtensorMap map_c8{};      // TMA descriptor of c8 (128B swizzle, 128 x 256 boxes)
    bool map_c8_ok = false;
    DevBuf<int> pkeys;         // per-centroid integer keys of the kind::i8 epilogue
    // FP8 (e4m3) search operands: codes [k][kp8], column factors and scoring norms
    // (padded to whole tiles), TMA descriptor of the codes
    DevBuf<uint8_t> c_f8;
    DevBuf<float> wf8, nf8;
    CUtensorMap map_f8{};
    bool f8_ok = false;

    // resident rows
    DevBuf<uint8_t> rows;
    const void* rows_view = nullptr;  // rows owned by another handle (batched instances)
    int rows_dtype = -1;
    size_t rows_n = 0, rows_d = 0;
    DevBuf<uint32_t> res_labels;
    DevBuf<float> res_dist;
    size_t res_n = 0;            // rows of the last emb200_assign_resident (0: none valid)
    uint64_t res_version = 0;    // centroid version those results belong to

    // scratch for assign
    DevBuf<uint8_t> stage;  // host-path staging of rows (two chunk buffers)
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_copied[2] = {nullptr, nullptr};
    cudaEvent_t ev_done[2] = {nullptr, nullptr};  // a staging buffer's search is complete
    DevBuf<uint32_t> st_labels;
    DevBuf<float> st_dist;
    // largest split partials of any batch of up to part_size_m rows (no-host-read mode)
    size_t part_size_m = 0, part_size_k = 0, part_size_rows = 0;
    bool part_size_tc = false;
    DevBuf<float> part_s;
    DevBuf<uint32_t> part_i;
    DevBuf<uint32_t> redo_rows;
    DevBuf<float> redo_theta;
    DevBuf<uint32_t> cand, cand_count, redo2_rows;  // refine pass
    DevBuf<uint32_t> counters;  // see assign_rows_dev
    DevBuf<unsigned long long> rkeys;  // exhaustive search: per listed row (score, index) keys

    // training state
    TrainState train;
    BatchState bat;       // batched lockstep training (emb200_train_batched)
    int bat_variant = -1; // search variant of the last lockstep run (autotuner's choice)

    // learned proposer (emb200_proposer_*), and a counter of centroid changes it tracks
    Proposer* prop = nullptr;
    uint64_t centroid_version = 0;

    // int8 quantizer scratch (emb200_quantizer_*)
    DevBuf<float> qshift;
    DevBuf<QuantSelect> qsel;
    DevBuf<unsigned long long> qclip;
    DevBuf<uint8_t> qx, qcodes;

    // report() state (emb200_report*)
    ReportState* rep = nullptr;

    // abort-path test (emb200_set_abort_test): stall of the fast tensor-core kernels
    int stall_tile = 0;
    uint64_t stall_ns = 0;
};

namespace {

int fail(emb200_handle* h, int code, const char* fmt, ...) {
    // The error is reported here: clear the runtime's last-error state, so that a
    // later call's launch checks do not report this one again (a sticky error,
    // such as an illegal address, still fails every later call by itself).
    cudaGetLastError();
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (h) h->err = buf;
    return code;
}

#define CK(call)                                                                                      \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess) return fail(h, e_ == cudaErrorMemoryAllocation ? EMB200_ENOMEM : EMB200_ECUDA, \
                                           "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

#define CKL()                                                                                         \
    do {                                                                                              \
        h->stats.kernel_launches++;                                                                   \
        cudaError_t e_ = cudaGetLastError();                                                          \
        if (e_ != cudaSuccess) return fail(h, EMB200_ECUDA, "kernel launch: %s (%s:%d)", cudaGetErrorString(e_), \
                                           __FILE__, __LINE__);                                       \
    } while (0)

// cudaFuncSetAttribute(MaxDynamicSharedMemorySize) once per kernel and device:
// the attribute belongs to the device context, so a flag per call site and
// device (bit `device` of `done`) covers handles on several GPUs in one process.
int smem_attr_once(emb200_handle* h, std::atomic<uint64_t>& done, const void* fn, int bytes) {
    const uint64_t bit = 1ull << (h->device & 63);
    if (done.load() & bit) return EMB200_OK;
    CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    done.fetch_or(bit);
    return EMB200_OK;
}

#define SMEM_ATTR_ONCE(fn, bytes)                                               \
    do {                                                                        \
        static std::atomic<uint64_t> done_{0};                                  \
        int rc_ = smem_attr_once(h, done_, (const void*)(fn), (int)(bytes));    \
        if (rc_) return rc_;                                                    \
    } while (0)

size_t elt_size(int dtype) { return dtype == EMB200_F32 ? 4 : 1; }

// Error-bound coefficients of the certification, E = ka |x| cmax + kb nmax
// (see k_certify). u = 2^-24 (f32 rounding), ub = 2^-8 (bf16 rounding: 8
// significant bits, round to nearest); the
// tensor-core accumulation is allowed one f32 truncation (2u) per product term.
//
// The single-term BF16 search of f32 rows (norm_mma) sums the half-norm's three
// BF16 parts in the same tensor-core accumulation as the d products: three more
// truncated terms, whose magnitudes add |norm| / 2 to the sum they are relative to,
// so the score (twice the accumulator) gains gamma(d + 5, 2u) |norm|.
//
// kr (single-term BF16, when the caller asks for it): the operands' rounding is
// bounded per row instead, by kr (xr cmax + (|x| + xr) dmax) with xr = |x - bf16(x)|
// of the row and dmax >= max_j |c_j - bf16(c_j)| (exact identity plus Cauchy-Schwarz,
// in score units), and leaves ka.
void bound_coefficients(int precision, int dtype, size_t d, bool packed, float* ka, float* kb, bool norm_mma = false,
                        float* kr = nullptr) {
    if (kr) *kr = 0.0f;
    const double u = std::ldexp(1.0, -24), ub = std::ldexp(1.0, -8);
    auto gamma = [](double n, double unit) { return n * unit / (1.0 - n * unit); };
    double g_ref = gamma((double)d + 2, u);  // reference dot vs exact
    double a;
    if (precision == EMB200_PREC_FP32) {
        a = 2.0 * (gamma((double)d + 2, u) + g_ref) + 4.02 * u;
    } else if (precision == EMB200_PREC_FP8) {
        // e4m3 rounding of both operands: relative u8 = 2^-4 for elements in the
        // binades below the scaled maximum (224, 448], and for the small ones a
        // floor of 2^-10 / scale <= 2^-10 max / 224 per element, at most
        // sqrt(d) 2^-10 / 224 |x||c| over a dot product, for each operand.
        const double u8 = std::ldexp(1.0, -4);
        const double rep = 2.0 * u8 + u8 * u8 + 2.0 * (1.0 + u8) * std::sqrt((double)d) * std::ldexp(1.0, -10) / 224.0;
        a = 2.0 * (rep + 1.02 * gamma((double)d + 2, 2 * u) + g_ref) + 4.02 * u;
    } else if (precision == EMB200_PREC_BF16) {
        double terms = dtype == EMB200_F32 ? 3.0 : 2.0;
        double rep = dtype == EMB200_F32 ? 3.2 * ub * ub : 1.1 * ub * ub;  // dropped split terms
        a = 2.0 * (rep + 1.02 * gamma(terms * (double)d + 2, 2 * u) + g_ref) + 4.02 * u;
    } else {
        double rep = dtype == EMB200_F32 ? 2.0 * ub + ub * ub : ub;
        if (kr) {
            // The identity is exact and the norms it uses are rounded up; the
            // 2^-10 margin covers |x| from the reference's rounded sqnorm.
            rep = 0.0;
            *kr = 2.0f * (1.0f + 0x1p-10f);
        }
        a = 2.0 * (rep + 1.02 * gamma((double)d + (norm_mma ? 5 : 2), 2 * u) + g_ref) + 4.02 * u;
    }
    double b = 2.0 * u;
    if (norm_mma) b += 1.02 * gamma((double)d + 5, 2 * u);
    if (packed) {  // tensor-core top-2 keys carry the column in 5 mantissa bits: |key - s| <= 2^-18 |s|
        const double t = std::ldexp(1.0, -18);
        a += 2.01 * t;
        b += t;
    }
    *ka = (float)(1.25 * a);
    *kb = (float)(1.25 * b);
}

bool use_i8_mode(const emb200_handle* h, int dtype) {
    return dtype == EMB200_I8 &&
           (h->opts.centroid_bits == EMB200_CENTROIDS_I8 || h->opts.centroid_bits == EMB200_CENTROIDS_I16);
}


// cuTensorMapEncodeTiled from the driver, fetched at run time (no libcuda link).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled_fn() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    });
    return fn;
}

// 2-D map over a k x kpad BF16 matrix (row stride kpad), boxes of 64 x 256
// (one 128-byte swizzle atom wide); rows past k read as zeros.
int encode_bf16_map(emb200_handle* h, CUtensorMap* map, void* base) {
    EncodeTiledFn fn = encode_tiled_fn();
    if (!fn) return fail(h, EMB200_ECUDA, "cuTensorMapEncodeTiled unavailable");
    cuuint64_t dims[2] = {(cuuint64_t)h->kpad, (cuuint64_t)h->k};
    cuuint64_t strides[1] = {(cuuint64_t)h->kpad * 2};
    cuuint32_t box[2] = {64, (cuuint32_t)kTcBN};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, base, dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(h, EMB200_ECUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return EMB200_OK;
}

// set_centroids on the device: reference norms, certification bounds, and the
// forms the selected search needs (BF16 split for tcgen05, i8 for I8 mode).
int prepare_centroids(emb200_handle* h) {
    cudaStream_t st = h->stream;
    const int k = (int)h->k, d = (int)h->d;
    CK(cudaMemsetAsync(h->bounds.p, 0, sizeof(Bounds), st));
    // Norms are padded to whole tiles with 3e38 (never a candidate, and finite
    // so the packed top-2 keys of the padding stay numbers).
    const size_t kp = (h->k + kTcBN - 1) / kTcBN * kTcBN;
    k_fill<<<(unsigned)((kp + 255) / 256), 256, 0, st>>>(h->norms.p, (int)kp, 3.0e38f);
    CKL();
    h->kpad = (h->d + 63) / 64 * 64;
    __nv_bfloat16 *hi = nullptr, *lo = nullptr;
    h->maps_ok = false;
    if (h->kpad <= 256) {
        // BF16 hi/lo split for the tensor-core search and refine passes.
        if (h->c_hi.ensure((size_t)k * h->kpad) || h->c_lo.ensure((size_t)k * h->kpad))
            return fail(h, EMB200_ENOMEM, "BF16 centroid allocation failed");
        hi = h->c_hi.p;
        lo = h->c_lo.p;
        int rc = encode_bf16_map(h, &h->map_hi, hi);
        if (rc) return rc;
        rc = encode_bf16_map(h, &h->map_lo, lo);
        if (rc) return rc;
        // Allocated here, outside any captured epoch; filled before each search.
        if (h->nrm16.ensure(kp * 16)) return fail(h, EMB200_ENOMEM, "BF16 norm allocation failed");
        h->maps_ok = true;
    }
    k_prep_centroids<<<(unsigned)((k + 7) / 8), 256, 0, st>>>(h->c.p, k, d, h->norms.p, h->bounds.p, hi, lo,
                                                              (int)h->kpad);
    CKL();
    h->f8_ok = false;
    if (h->opts.precision == EMB200_PREC_FP8 && h->d <= 256) {
        // e4m3 codes in rows of one or two 128-byte swizzle atoms; scoring norms are
        // the reference norms, -3e38 for a centroid outside the FP8 range (so it can
        // only be a row's first candidate, which the certification re-scores
        // exactly), 3e38 for the padding.
        const size_t kp8 = (h->d + 127) / 128 * 128;
        if (h->c_f8.ensure((size_t)k * kp8) || h->wf8.ensure(kp) || h->nf8.ensure(kp))
            return fail(h, EMB200_ENOMEM, "FP8 centroid allocation failed");
        CK(cudaMemcpyAsync(h->nf8.p, h->norms.p, kp * sizeof(float), cudaMemcpyDeviceToDevice, st));
        k_prep_fp8<<<(unsigned)((kp * 32 + 255) / 256), 256, 0, st>>>(h->c.p, k, d, (int)kp8, (int)kp, h->c_f8.p,
                                                                      h->wf8.p, h->nf8.p);
        CKL();
        EncodeTiledFn fn = encode_tiled_fn();
        if (!fn) return fail(h, EMB200_ECUDA, "cuTensorMapEncodeTiled unavailable");
        cuuint64_t dims[2] = {(cuuint64_t)kp8, (cuuint64_t)h->k};
        cuuint64_t strides[1] = {(cuuint64_t)kp8};
        cuuint32_t box[2] = {128, (cuuint32_t)kTcBN};
        cuuint32_t estr[2] = {1, 1};
        CUresult r = fn(&h->map_f8, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, h->c_f8.p, dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return fail(h, EMB200_ECUDA, "cuTensorMapEncodeTiled (fp8) failed (%d)", (int)r);
        h->f8_ok = true;
    }
    if (h->opts.centroid_bits == EMB200_CENTROIDS_I8) {
        // Rows of c8 padded to whole 128-byte swizzle atoms (the kind::i8 K atom).
        const size_t kp8 = (h->d + 127) / 128 * 128;
        if (h->c8.ensure((size_t)k * kp8) || h->off8.ensure(k)) return fail(h, EMB200_ENOMEM, "i8 centroid allocation failed");
        k_prep_i8<<<(unsigned)((k + 7) / 8), 256, 0, st>>>(h->c.p, k, d, (int)kp8, h->c8.p, h->off8.p);
        CKL();
        h->map_c8_ok = false;
        if (h->d <= 512) {
            EncodeTiledFn fn = encode_tiled_fn();
            if (!fn) return fail(h, EMB200_ECUDA, "cuTensorMapEncodeTiled unavailable");
            cuuint64_t dims[2] = {(cuuint64_t)kp8, (cuuint64_t)h->k};
            cuuint64_t strides[1] = {(cuuint64_t)kp8};
            cuuint32_t box[2] = {128, (cuuint32_t)kTcBN};
            cuuint32_t estr[2] = {1, 1};
            CUresult r = fn(&h->map_c8, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, h->c8.p, dims, strides, box, estr,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            if (r != CUDA_SUCCESS) return fail(h, EMB200_ECUDA, "cuTensorMapEncodeTiled (i8) failed (%d)", (int)r);
            h->map_c8_ok = true;
        }
    }
    if (h->opts.centroid_bits == EMB200_CENTROIDS_I16) {
        // The largest s <= 7 with d 128 (128 2^s) < 2^31 (src/cpu_i8.rs:96-98).
        int s = 7;
        while (s > 0 && ((uint64_t)h->d << (14 + s)) >= ((uint64_t)1 << 31)) s--;
        h->ishift = s;
        const size_t kp16 = (h->d + 31) / 32 * 32;
        if (h->c16.ensure((size_t)k * kp16) || h->off8.ensure(k)) return fail(h, EMB200_ENOMEM, "i16 centroid allocation failed");
        k_prep_i16<<<(unsigned)((k + 7) / 8), 256, 0, st>>>(h->c.p, k, d, (int)kp16, (float)(1u << s), h->c16.p,
                                                            h->off8.p);
        CKL();
    }
    h->bias_set = false;
    h->bias_absmax = 0.0;
    return EMB200_OK;
}

// set_bias on the device (bias already in device memory).
int apply_bias(emb200_handle* h, const float* bias_dev) {
    cudaStream_t st = h->stream;
    const int k = (int)h->k;
    k_add_bias<<<(unsigned)((k + 255) / 256), 256, 0, st>>>(h->norms.p, bias_dev, k, h->bounds.p);
    CKL();
    if (h->f8_ok) {
        k_add_bias_f8<<<(unsigned)((k + 255) / 256), 256, 0, st>>>(h->nf8.p, bias_dev, k);
        CKL();
    }
    if (h->opts.centroid_bits == EMB200_CENTROIDS_I8 || h->opts.centroid_bits == EMB200_CENTROIDS_I16) {
        const double unit = h->opts.centroid_bits == EMB200_CENTROIDS_I16 ? std::ldexp(1.0, 2 * h->ishift) : 1.0;
        k_bias_i8<<<(unsigned)((k + 255) / 256), 256, 0, st>>>(h->off8.p, bias_dev, k, unit);
        CKL();
    }
    h->bias_set = true;
    h->bias_absmax = INFINITY;  // device-computed bias: magnitude unknown on the host
    return EMB200_OK;
}

// CpuI8Assigner(I8) semantics: exact integer search, no certification needed.
// The kind::i8 tensor-core kernel serves d <= 512 with |bias| small enough for
// its 32-bit keys (see kernels_tc_i8.cuh); other cases use the dp4a kernel.
int launch_i8_assign(emb200_handle* h, const int8_t* x, const uint32_t* gather, size_t m, uint32_t* labels,
                     float* dist, cudaStream_t st, bool graph = false) {
    const int k = (int)h->k, d = (int)h->d;
    const size_t kp8 = (h->d + 127) / 128 * 128;
    const bool wide = h->opts.centroid_bits == EMB200_CENTROIDS_I16;
    const bool tc = !wide && h->map_c8_ok && h->d <= 512 && h->bias_absmax <= 8.0e6;
    const double inv_unit = wide ? std::ldexp(1.0, -2 * h->ishift) : 1.0;
    int nsplit = 1;
    const int target = tc ? h->sm_count : 2 * h->sm_count;
    const int row_tiles = (int)((m + 127) / 128);
    const int ntiles = tc ? (k + kTcBN - 1) / kTcBN : (k + kI8BN - 1) / kI8BN;
    if (row_tiles < target) nsplit = std::min(ntiles, (target + row_tiles - 1) / row_tiles);
    nsplit = std::max(nsplit, 1);
    // As in assign_rows_dev: in the training loop, size the split partials for every
    // batch of up to m rows (a smaller batch may use more splits).
    size_t part_rows = (size_t)nsplit * m;
    if (graph) {
        for (size_t rt = 1; rt * 128 < m + 128; rt++) {
            const size_t mm = std::min(rt * 128, m);
            const int ns = (int)rt < target ? std::max(1, std::min(ntiles, (target + (int)rt - 1) / (int)rt)) : 1;
            part_rows = std::max(part_rows, (size_t)ns * mm);
        }
    }
    // part_s holds int64 scores here: 2 floats per entry.
    if (h->part_s.ensure(part_rows * 2) || h->part_i.ensure(part_rows) || h->counters.ensure(8))
        return fail(h, EMB200_ENOMEM, "scratch allocation failed for %zu rows", m);
    if (!graph) CK(cudaEventRecord(h->evk0, st));
    if (tc) {
        const size_t kp = (h->k + kTcBN - 1) / kTcBN * kTcBN;
        if (h->pkeys.ensure(kp)) return fail(h, EMB200_ENOMEM, "key allocation failed");
        k_i8_keys<<<(unsigned)((kp + 255) / 256), 256, 0, st>>>(h->off8.p, k, (int)kp, h->pkeys.p);
        CKL();
        // Graph replay keeps the flag sticky: the training loop clears it once and reads it at the end.
        if (!graph) CK(cudaMemsetAsync(h->counters.p + 2, 0, sizeof(uint32_t), st));
        TcI8Params p{};
        p.m = (int)m;
        p.d = d;
        p.k = k;
        p.kpad = (int)kp8;
        p.gather = gather;
        p.pkeys = h->pkeys.p;
        p.part_s = (long long*)h->part_s.p;
        p.part_i = h->part_i.p;
        p.err = (int*)(h->counters.p + 2);
        p.stall_tile = h->stall_tile;
        p.stall_ns = h->stall_ns;
        const TcSmem L = tc_i8_smem_layout(p.kpad);
        const size_t smem = std::max<size_t>(L.total + 1024, 120 * 1024);
        SMEM_ATTR_ONCE(k_assign_tc_i8, kTcSmemLimit);
        k_assign_tc_i8<<<dim3((unsigned)row_tiles, (unsigned)nsplit), kTcThreads, smem, st>>>(x, h->map_c8, p);
        CKL();
    } else {
        const int xvec = (d % 16 == 0 && ((uintptr_t)x & 15) == 0) ? 1 : 0;
        if (wide) {
            k_assign_i8<true><<<dim3((unsigned)row_tiles, (unsigned)nsplit), 256, 0, st>>>(
                x, gather, (int)m, d, h->c16.p, (int)((h->d + 31) / 32 * 32), h->off8.p, k, 2ll << h->ishift,
                (long long*)h->part_s.p, h->part_i.p, xvec);
        } else {
            k_assign_i8<false><<<dim3((unsigned)row_tiles, (unsigned)nsplit), 256, 0, st>>>(
                x, gather, (int)m, d, h->c8.p, (int)kp8, h->off8.p, k, 2ll, (long long*)h->part_s.p, h->part_i.p,
                xvec);
        }
        CKL();
    }
    if (!graph) CK(cudaEventRecord(h->evk1, st));
    h->stats.fast_kernel = tc ? 3 : 2;
    k_finish_i8<<<(unsigned)((m + 7) / 8), 256, 0, st>>>(x, gather, (int)m, d, (const long long*)h->part_s.p,
                                                         h->part_i.p, nsplit, labels, dist, inv_unit);
    CKL();
    if (tc && !graph) {  // the bounded waits gave up: redo the call with the exact dp4a kernel
        uint32_t err = 0;
        CK(cudaMemcpyAsync(&err, h->counters.p + 2, sizeof err, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        float kms = 0.0f;
        CK(cudaEventElapsedTime(&kms, h->evk0, h->evk1));
        h->stats.fast_ms += kms;
        h->stats.fast_launches += 1;
        if (err) {
            h->stats.fast_aborted = 1;
            const int xvec = (d % 16 == 0 && ((uintptr_t)x & 15) == 0) ? 1 : 0;
            const int ns = std::max(1, std::min((k + kI8BN - 1) / kI8BN, (2 * h->sm_count + row_tiles - 1) / row_tiles));
            if (h->part_s.ensure((size_t)ns * m * 2) || h->part_i.ensure((size_t)ns * m))
                return fail(h, EMB200_ENOMEM, "scratch allocation failed for %zu rows", m);
            k_assign_i8<false><<<dim3((unsigned)row_tiles, (unsigned)ns), 256, 0, st>>>(
                x, gather, (int)m, d, h->c8.p, (int)kp8, h->off8.p, k, 2ll, (long long*)h->part_s.p, h->part_i.p,
                xvec);
            CKL();
            k_finish_i8<<<(unsigned)((m + 7) / 8), 256, 0, st>>>(x, gather, (int)m, d, (const long long*)h->part_s.p,
                                                                 h->part_i.p, ns, labels, dist, 1.0);
            CKL();
        }
    }
    return EMB200_OK;
}

// Product terms of the tensor-core search: three for f32 rows (their BF16 split
// has a low part), two for integer rows (exact in BF16), one for BF16X1 and FP8.
int tc_terms(int precision, int dtype) {
    if (precision == EMB200_PREC_BF16X1 || precision == EMB200_PREC_FP8) return 1;
    return dtype == EMB200_F32 ? 3 : 2;
}

// K width of the operands in elements: one 128-byte atom per 64 BF16 or 128 e4m3.
int tc_kpad(const emb200_handle* h, bool fp8) { return fp8 ? (int)((h->d + 127) / 128 * 128) : (int)h->kpad; }

bool tc_supported(const emb200_handle* h, int nterms, bool fp8 = false) {
    if (fp8 ? !h->f8_ok : !h->maps_ok) return false;
    const TcLayout L = tc_layout(tc_kpad(h, fp8), nterms, fp8);
    return L.stages >= 2 && L.total + 1024 <= (uint32_t)kTcSmemLimit;
}

// Column splits of the tensor-core search: the one with the fewest waves of CTAs
// times the tiles a CTA takes (plus half a tile of per-CTA setup), a larger
// split only when it saves 3%. 394 row tiles on 148 SMs: 3 splits, 8 waves of 22
// tiles, against 3 waves of 64 unsplit.
//
// Splits with the same tiles per CTA form runs of consecutive counts, and within
// a run the waves never decrease with the count, so only the first count of each
// run can be chosen: visiting those (O(sqrt(tiles)) of them) picks the same split
// as trying every count from 1 to the number of tiles.
int tc_nsplit(const emb200_handle* h, size_t m) {
    const long row_tiles = (long)((m + kTcBM - 1) / kTcBM);
    const int ntiles = (int)((h->k + kTcBN - 1) / kTcBN);
    const long sms = std::max(1, h->sm_count);
    int best = 1;
    double best_cost = 0.0;
    for (int ns = 1; ns <= ntiles;) {
        const int per_cta = (ntiles + ns - 1) / ns;
        const double waves = (double)((row_tiles * ns + sms - 1) / sms);
        const double cost = waves * ((double)per_cta + 0.5);
        if (ns == 1 || cost < 0.97 * best_cost) {
            best = ns;
            best_cost = cost;
        }
        if (per_cta == 1) break;
        ns = (ntiles + per_cta - 2) / (per_cta - 1);  // first count with fewer tiles per CTA
    }
    return best;
}

template <typename T, bool COLLECT, bool FP8, bool NM = false>
int launch_tc_kernel(emb200_handle* h, const T* x, const TcParams& p, int nsplit, cudaStream_t st) {
    const TcLayout L = tc_layout(p.kpad, p.nterms, FP8, NM);
    // At least 120 KB so that two CTAs never share an SM: each holds all 512 TMEM columns.
    const size_t smem = std::max<size_t>(L.total + 1024, 120 * 1024);
    SMEM_ATTR_ONCE((k_assign_tc<T, COLLECT, FP8, NM>), 227 * 1024);  // one flag per instantiation
    // Persistent: one CTA per SM, or one per work item when there are fewer.
    const size_t items = (p.m + (size_t)kTcBM - 1) / kTcBM * (size_t)nsplit;
    const unsigned grid = (unsigned)std::max<size_t>(1, std::min(items, (size_t)h->sm_count));
    k_assign_tc<T, COLLECT, FP8, NM><<<grid, kTcPThreads, smem, st>>>(x, FP8 ? h->map_f8 : h->map_hi, h->map_lo, p);
    CKL();
    return EMB200_OK;
}

template <typename T, bool COLLECT>
int launch_tc(emb200_handle* h, const T* x, const uint32_t* gather, const uint32_t* gather2, size_t m, int nterms,
              const float* theta, uint32_t* cand, uint32_t* cand_count, int cap, int* err, cudaStream_t st,
              const uint32_t* m_dev = nullptr, int nsplit_override = 0, bool fp8 = false,
              const TcParams* fuse = nullptr, bool* fused = nullptr) {
    TcParams p{};
    p.m = (int)m;
    p.d = (int)h->d;
    p.k = (int)h->k;
    p.kpad = tc_kpad(h, fp8);
    p.nterms = nterms;
    p.gather = gather;
    p.gather2 = gather2;
    p.norms = fp8 ? h->nf8.p : h->norms.p;
    p.wf8 = fp8 ? h->wf8.p : nullptr;
    p.part_s = h->part_s.p;
    p.part_i = h->part_i.p;
    p.err = err;
    p.xvec = (h->d % 4 == 0 && ((uintptr_t)x & 15) == 0) ? 1 : 0;
    p.theta = theta;
    p.cand = cand;
    p.cand_count = cand_count;
    p.cand_cap = cap;
    p.m_dev = m_dev;
    if (!COLLECT) {  // the abort-path test stalls the fast search only
        p.stall_tile = h->stall_tile;
        p.stall_ns = h->stall_ns;
    }
    const int nsplit = nsplit_override > 0 ? nsplit_override : tc_nsplit(h, m);
    p.nsplit = nsplit;
    if constexpr (!COLLECT && std::is_same<T, float>::value) {
        if (fp8) return launch_tc_kernel<T, false, true>(h, x, p, nsplit, st);
        // Single-term BF16 search of f32 rows: norms summed inside the contraction
        // (the certification bound allows for it whenever this mode is searched).
        const size_t kp = (h->k + kTcBN - 1) / kTcBN * kTcBN;
        if (nterms == 1 && h->nrm16.n >= kp * 16) {
            k_prep_nrm16<<<(unsigned)((kp + 255) / 256), 256, 0, st>>>(h->norms.p, (int)kp, h->nrm16.p);
            CKL();
            p.nrm16 = h->nrm16.p;
            if (fuse && nsplit == 1) {  // certification at the end of each item
                p.fuse = 1;
                p.cx = fuse->cx;
                p.bounds = fuse->bounds;
                p.ka = fuse->ka;
                p.kb = fuse->kb;
                p.kr = fuse->kr;
                p.ka2 = fuse->ka2;
                p.kb2 = fuse->kb2;
                p.labels = fuse->labels;
                p.dist = fuse->dist;
                p.redo_rows = fuse->redo_rows;
                p.redo_theta = fuse->redo_theta;
                p.redo_count = fuse->redo_count;
                p.cert_count = fuse->cert_count;
                if (fused) *fused = true;
            }
            return launch_tc_kernel<T, false, false, true>(h, x, p, nsplit, st);
        }
    }
    return launch_tc_kernel<T, COLLECT, false>(h, x, p, nsplit, st);
}

// Fold the device counters of one pipeline run into the handle's stats.
int finish_counters(emb200_handle* h, cudaStream_t st, bool refined) {
    uint32_t c[5];
    CK(cudaMemcpyAsync(c, h->counters.p, sizeof c, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    h->stats.rows_certified += c[1];
    h->stats.rows_researched += refined ? c[3] : c[0];
    if (c[2] || c[4]) h->stats.fast_aborted = 1;
    return EMB200_OK;
}

// Full pipeline of one assign over m rows already on the device (x, or
// gathered through `gather`), results to device labels/dist:
//   1. fast contraction (tcgen05 BF16 or FP32 SIMT): top-2 per row with an error bound
//   2. certify: exact re-score of the two candidates; rows whose margin the bound
//      certifies are final
//   3. refine (uncertified rows): a three-term BF16 tensor-core pass collects every
//      centroid whose score could reach the exact best, then exact re-score of those
//   4. exhaustive exact search for rows the refine pass could not settle
// Counters (device): [0] uncertified rows, [1] certified rows, [2] fast-kernel abort,
// [3] exhaustive rows, [4] refine abort.
template <typename T>
int settle_rows(emb200_handle* h, const T* x, const uint32_t* gather, size_t m, uint32_t* labels, float* dist,
                cudaStream_t st, bool graph, int nsplit, int fast_prec, bool tc,
                const float2* row_bounds = nullptr, bool certified = false);

template <typename T>
int assign_rows_dev(emb200_handle* h, const T* x, const uint32_t* gather, size_t m, uint32_t* labels, float* dist,
                    cudaStream_t st, bool graph = false) {
    const int dtype = std::is_same<T, float>::value ? EMB200_F32 : (std::is_same<T, int8_t>::value ? EMB200_I8 : EMB200_U8);
    const int k = (int)h->k, d = (int)h->d;
    if (m == 0) return EMB200_OK;
    if (m > kMaxSearchRows) {
        // Pieces of at most 2^26 rows: the search kernels index rows (up to 32
        // threads each) in 32 bits.
        for (size_t r0 = 0; r0 < m; r0 += kMaxSearchRows) {
            const size_t mc = std::min(kMaxSearchRows, m - r0);
            const T* xs = gather ? x : x + r0 * (size_t)d;
            int rc = assign_rows_dev(h, xs, gather ? gather + r0 : nullptr, mc, labels + r0, dist + r0, st, graph);
            if (rc) return rc;
        }
        return EMB200_OK;
    }
    if (use_i8_mode(h, dtype)) {
        h->stats.fast_kernel = 2;
        return launch_i8_assign(h, (const int8_t*)x, gather, m, labels, dist, st, graph);
    }
    int prec = h->opts.precision;
    // FP8 operands for f32 rows when prepared (d <= 256); otherwise the single-term BF16 search.
    const bool fp8 = prec == EMB200_PREC_FP8 && dtype == EMB200_F32 && tc_supported(h, 1, true);
    if (prec == EMB200_PREC_FP8 && !fp8) prec = EMB200_PREC_BF16X1;
    const int row_tiles = (int)((m + kSimtBM - 1) / kSimtBM);
    const int ntiles = (k + kSimtBN - 1) / kSimtBN;
    const int fast_terms = tc_terms(prec, dtype);
    const bool tc = prec != EMB200_PREC_FP32 && (fp8 || tc_supported(h, fast_terms));
    int nsplit = 1;
    if (tc) {
        nsplit = tc_nsplit(h, m);
    } else {
        int target = 2 * h->sm_count;
        if (row_tiles < target) nsplit = std::min(ntiles, (target + row_tiles - 1) / row_tiles);
    }
    // Inside the training loop (graph = true) nothing may allocate while an epoch is
    // captured, and a smaller batch can need more split partials than a full one
    // (fewer row tiles, more splits): size them for every batch of up to m rows.
    size_t part_rows = (size_t)nsplit * m;
    if (graph && m <= h->part_size_m && h->part_size_k == h->k && h->part_size_tc == tc) {
        // Sized before for every batch of up to part_size_m rows, which covers this one.
        part_rows = std::max(part_rows, h->part_size_rows);
    } else if (graph) {
        for (size_t rt = 1; rt * kTcBM < m + kTcBM; rt++) {
            const size_t mm = std::min(rt * kTcBM, m);
            int ns = 1;
            if (tc) {
                ns = tc_nsplit(h, mm);
            } else {
                const int rtiles = (int)((mm + kSimtBM - 1) / kSimtBM), target = 2 * h->sm_count;
                if (rtiles < target) ns = std::min(ntiles, (target + rtiles - 1) / rtiles);
            }
            part_rows = std::max(part_rows, (size_t)ns * mm);
        }
        h->part_size_m = m;
        h->part_size_k = h->k;
        h->part_size_tc = tc;
        h->part_size_rows = part_rows;
    }
    if (h->part_s.ensure(part_rows * 2) || h->part_i.ensure(part_rows * 2) || h->redo_rows.ensure(m) ||
        h->redo_theta.ensure(m) || h->counters.ensure(8))
        return fail(h, EMB200_ENOMEM, "scratch allocation failed for %zu rows", m);
    uint32_t* ctr = h->counters.p;
    CK(cudaMemsetAsync(ctr, 0, 8 * sizeof(uint32_t), st));
    h->stats.fast_kernel = fp8 ? 4 : tc ? 1 : 0;
    if (!graph) CK(cudaEventRecord(h->evk0, st));
    bool fused = false;
    if (tc) {
        // Single-term search of aligned f32 rows in the AVX-512 rounding: the fast
        // kernel certifies each row tile itself (when it also sums the norms in its
        // contraction and searches all columns in one split).
        TcParams fz{};
        const TcParams* fzp = nullptr;
        if constexpr (std::is_same<T, float>::value) {
            if (!fp8 && fast_terms == 1 && h->opts.match_kernel == kMatchAvx512 && d % 16 == 0 &&
                ((uintptr_t)x & 15) == 0 && ((uintptr_t)h->c.p & 15) == 0) {
                bound_coefficients(prec, dtype, h->d, true, &fz.ka, &fz.kb, prec == EMB200_PREC_BF16X1, &fz.kr);
                bound_coefficients(EMB200_PREC_BF16, dtype, h->d, false, &fz.ka2, &fz.kb2);
                fz.cx = h->c.p;
                fz.bounds = h->bounds.p;
                fz.labels = labels;
                fz.dist = dist;
                fz.redo_rows = h->redo_rows.p;
                fz.redo_theta = h->redo_theta.p;
                fz.redo_count = ctr;
                fz.cert_count = ctr + 1;
                fzp = &fz;
            }
        }
        int rc = launch_tc<T, false>(h, x, gather, nullptr, m, fast_terms, nullptr, nullptr, nullptr, 0,
                                     (int*)(ctr + 2), st, nullptr, 0, fp8, fzp, &fused);
        if (rc) return rc;
    } else {
        dim3 grid(row_tiles, nsplit);
        int vec4 = (d % 4 == 0 && ((uintptr_t)x & 15) == 0) ? 1 : 0;
        k_assign_simt<T><<<grid, kSimtThreads, 0, st>>>(x, gather, (int)m, d, h->c.p, h->norms.p, k, h->part_s.p,
                                                         h->part_i.p, vec4);
        CKL();
    }
    if (!graph) CK(cudaEventRecord(h->evk1, st));
    return settle_rows(h, x, gather, m, labels, dist, st, graph, nsplit, tc ? prec : EMB200_PREC_FP32, tc, nullptr,
                       fused);
}

// Exhaustive exact search of the rows listed in rows[0 .. *count) (count on the
// device, at most m): each row's centroids are split over several CTAs.
template <typename T>
int launch_research(emb200_handle* h, const T* x, const uint32_t* gather, size_t m, const uint32_t* rows,
                    const uint32_t* count, uint32_t* labels, float* dist, cudaStream_t st) {
    const int k = (int)h->k;
    const int slices = std::max(1, std::min(64, (k + 2047) / 2048));
    const int span = (k + slices - 1) / slices;
    if (h->rkeys.ensure(m)) return fail(h, EMB200_ENOMEM, "scratch allocation failed for %zu rows", m);
    k_research_keys_init<<<(unsigned)((m + 255) / 256), 256, 0, st>>>(h->rkeys.p, m);
    CKL();
    k_research_split<T><<<h->sm_count * 4, 256, 0, st>>>(x, gather, (int)h->d, h->c.p, h->norms.p, k,
                                                          h->opts.match_kernel, rows, count, slices, span, h->rkeys.p);
    CKL();
    k_research_finish<T><<<(unsigned)((m * 32 + 255) / 256), 256, 0, st>>>(x, gather, (int)h->d, rows, count,
                                                                           h->rkeys.p, labels, dist);
    CKL();
    return EMB200_OK;
}

// Steps 2-4 of the pipeline for m rows whose fast-contraction top-2 partials are
// in h->part_s / h->part_i (nsplit splits), with the device counters zeroed before
// the fast kernel (which may have set the abort flag, counter 2).
template <typename T>
int settle_rows(emb200_handle* h, const T* x, const uint32_t* gather, size_t m, uint32_t* labels, float* dist,
                cudaStream_t st, bool graph, int nsplit, int fast_prec, bool tc, const float2* row_bounds,
                bool certified) {
    const int dtype = std::is_same<T, float>::value ? EMB200_F32 : (std::is_same<T, int8_t>::value ? EMB200_I8 : EMB200_U8);
    const int k = (int)h->k, d = (int)h->d;
    const int refine_terms = tc_terms(EMB200_PREC_BF16, dtype);
    if (h->redo_rows.ensure(m) || h->redo_theta.ensure(m) || h->counters.ensure(8))
        return fail(h, EMB200_ENOMEM, "scratch allocation failed for %zu rows", m);
    uint32_t* ctr = h->counters.p;
    float ka, kb, ka2, kb2, kr;
    bound_coefficients(fast_prec, dtype, h->d, tc, &ka, &kb,
                       tc && fast_prec == EMB200_PREC_BF16X1 && dtype == EMB200_F32, &kr);
    bound_coefficients(EMB200_PREC_BF16, dtype, h->d, false, &ka2, &kb2);
    const int match = h->opts.match_kernel;
    bool vec4 = false;
    if constexpr (std::is_same<T, float>::value)
        vec4 = d % 16 == 0 && ((uintptr_t)x & 15) == 0 && ((uintptr_t)h->c.p & 15) == 0;
    if (certified) {
        // the fast kernel certified its rows itself (TcParams::fuse)
    } else if (match == kMatchAvx512 && vec4) {
        k_certify16v<<<(unsigned)((m + 63) / 64), 256, 0, st>>>(
            (const float*)x, gather, (int)m, d, h->c.p, h->norms.p, k, h->part_s.p, h->part_i.p, nsplit, h->bounds.p,
            ka, kb, labels, dist, h->redo_rows.p, ctr, ctr + 1, tc ? (const int*)(ctr + 2) : nullptr, h->redo_theta.p,
            ka2, kb2, row_bounds, kr);
    } else if (match == kMatchAvx512) {
        k_certify16<T><<<(unsigned)((m + 15) / 16), 256, 0, st>>>(
            x, gather, (int)m, d, h->c.p, h->norms.p, k, h->part_s.p, h->part_i.p, nsplit, h->bounds.p, ka, kb, labels,
            dist, h->redo_rows.p, ctr, ctr + 1, tc ? (const int*)(ctr + 2) : nullptr, h->redo_theta.p, ka2, kb2,
            row_bounds, kr);
    } else {
        k_certify<T><<<(unsigned)((m + 7) / 8), 256, 0, st>>>(x, gather, (int)m, d, h->c.p, h->norms.p, k, h->part_s.p,
                                                               h->part_i.p, nsplit, h->bounds.p, ka, kb, match, labels,
                                                               dist, h->redo_rows.p, ctr, ctr + 1,
                                                               tc ? (const int*)(ctr + 2) : nullptr, h->redo_theta.p,
                                                               ka2, kb2, row_bounds, kr);
    }
    CKL();
    if (graph) {
        // No host reads: every later launch takes its row count from the device
        // counters (grids sized for all m rows, surplus CTAs leave at once).
        const uint32_t* exhaustive = h->redo_rows.p;
        const uint32_t* exhaustive_count = ctr;
        if (tc_supported(h, refine_terms)) {
            const int cap = kRefineCap;
            if (h->cand.ensure(m * cap) || h->cand_count.ensure(m) || h->redo2_rows.ensure(m))
                return fail(h, EMB200_ENOMEM, "refine allocation failed for %zu rows", m);
            CK(cudaMemsetAsync(h->cand_count.p, 0, m * sizeof(uint32_t), st));
            const int ntl = (int)((h->k + kTcBN - 1) / kTcBN);
            int rc = launch_tc<T, true>(h, x, gather, h->redo_rows.p, m, refine_terms, h->redo_theta.p, h->cand.p,
                                        h->cand_count.p, cap, (int*)(ctr + 4), st, ctr, std::min(ntl, 4));
            if (rc) return rc;
            k_rescore_cands<T><<<(unsigned)((m + 7) / 8), 256, 0, st>>>(
                x, gather, d, h->c.p, h->norms.p, match, h->redo_rows.p, ctr, h->cand.p, h->cand_count.p, cap,
                (const int*)(ctr + 4), labels, dist, h->redo2_rows.p, ctr + 3);
            CKL();
            exhaustive = h->redo2_rows.p;
            exhaustive_count = ctr + 3;
        }
        return launch_research(h, x, gather, m, exhaustive, exhaustive_count, labels, dist, st);
    }
    uint32_t nredo = 0;
    CK(cudaMemcpyAsync(&nredo, ctr, sizeof nredo, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    float kms = 0.0f;
    CK(cudaEventElapsedTime(&kms, h->evk0, h->evk1));
    h->stats.fast_ms += kms;
    h->stats.fast_launches += 1;
    h->stats.rows_refined += nredo;
    if (nredo == 0) return finish_counters(h, st, false);
    const uint32_t* exhaustive = h->redo_rows.p;
    const uint32_t* exhaustive_count = ctr;
    if (tc_supported(h, refine_terms)) {
        const int cap = kRefineCap;
        if (h->cand.ensure((size_t)nredo * cap) || h->cand_count.ensure(nredo) || h->redo2_rows.ensure(nredo))
            return fail(h, EMB200_ENOMEM, "refine allocation failed for %u rows", nredo);
        CK(cudaMemsetAsync(h->cand_count.p, 0, nredo * sizeof(uint32_t), st));
        int rc = launch_tc<T, true>(h, x, gather, h->redo_rows.p, nredo, refine_terms, h->redo_theta.p, h->cand.p,
                                    h->cand_count.p, cap, (int*)(ctr + 4), st);
        if (rc) return rc;
        k_rescore_cands<T><<<(nredo + 7) / 8, 256, 0, st>>>(x, gather, d, h->c.p, h->norms.p, match, h->redo_rows.p,
                                                           ctr, h->cand.p, h->cand_count.p, cap,
                                                           (const int*)(ctr + 4), labels, dist, h->redo2_rows.p,
                                                           ctr + 3);
        CKL();
        exhaustive = h->redo2_rows.p;
        exhaustive_count = ctr + 3;
    }
    // at most nredo rows reach the exhaustive list: grids sized by it, not by m
    const int rc = launch_research(h, x, gather, nredo, exhaustive, exhaustive_count, labels, dist, st);
    if (rc) return rc;
    return finish_counters(h, st, exhaustive_count == ctr + 3);
}

int assign_dispatch(emb200_handle* h, int dtype, const void* x, const uint32_t* gather, size_t m, uint32_t* labels,
                    float* dist, cudaStream_t st) {
    switch (dtype) {
        case EMB200_F32: return assign_rows_dev(h, (const float*)x, gather, m, labels, dist, st);
        case EMB200_I8: return assign_rows_dev(h, (const int8_t*)x, gather, m, labels, dist, st);
        case EMB200_U8: return assign_rows_dev(h, (const uint8_t*)x, gather, m, labels, dist, st);
    }
    return fail(h, EMB200_EINVAL, "unknown dtype %d", dtype);
}

int check_ready(emb200_handle* h, int dtype) {
    if (!h) return EMB200_EINVAL;
    if (!h->have_centroids) return fail(h, EMB200_ESTATE, "set_centroids must be called first");
    if (dtype < 0 || dtype > 2) return fail(h, EMB200_EINVAL, "unknown dtype %d", dtype);
    if (use_i8_mode(h, dtype) && h->d > 32768)
        return fail(h, EMB200_EINVAL, "integer assignment supports d <= 32768");
    return EMB200_OK;
}

// Host-memory assign (the trait call). Rows go through two staging buffers in
// chunks: the copy of chunk i+1 (its own stream) overlaps the search of chunk i,
// and each chunk's labels and distances are copied back as soon as they are final.
// With pinned host memory the transfers run at full PCIe speed.
int assign_host(emb200_handle* h, int dtype, const void* x, size_t m, uint32_t* labels, float* dist) {
    int rc = check_ready(h, dtype);
    if (rc) return rc;
    if (m && (!x || !labels || !dist)) return fail(h, EMB200_EINVAL, "null buffer");
    if (m > 0xFFFFFFFFull) return fail(h, EMB200_EINVAL, "more than 2^32 - 1 rows in one call");
    h->stats = emb200_stats{};
    cudaStream_t st = h->stream;
    if (!h->copy_stream) CK(cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking));
    if (!h->ev_copied[0]) {
        for (int b = 0; b < 2; b++) {
            CK(cudaEventCreateWithFlags(&h->ev_copied[b], cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&h->ev_done[b], cudaEventDisableTiming));
            CK(cudaEventRecord(h->ev_done[b], st));
        }
    }
    CK(cudaEventRecord(h->ev0, st));
    const size_t esz = elt_size(dtype);
    const size_t row_bytes = h->d * esz;
    // 64 MB chunks. The copies bound the call (the last chunk's search is the part no
    // copy overlaps), but each chunk's search reads its counters on the host, so more
    // chunks cost more than they hide: on 1M x 128 rows, 16 MB chunks took 13.4 ms
    // and 64 MB chunks halving over the last two took 11.0 ms, against 10.6 ms here.
    const size_t chunk = std::max<size_t>(1, std::min(m, ((size_t)64 << 20) / row_bytes));
    std::vector<size_t> starts;
    for (size_t r0 = 0; r0 < m; r0 += chunk) starts.push_back(r0);
    starts.push_back(m);
    const size_t nch = starts.size() - 1;
    if (h->stage.ensure(2 * chunk * row_bytes) || h->st_labels.ensure(chunk) || h->st_dist.ensure(chunk))
        return fail(h, EMB200_ENOMEM, "staging allocation failed");
    auto stage_of = [&](size_t i) { return h->stage.p + (i & 1) * chunk * row_bytes; };
    auto copy_in = [&](size_t i) -> int {
        const size_t r0 = starts[i], mc = starts[i + 1] - r0;
        CK(cudaStreamWaitEvent(h->copy_stream, h->ev_done[i & 1], 0));  // buffer no longer read
        CK(cudaMemcpyAsync(stage_of(i), (const uint8_t*)x + r0 * row_bytes, mc * row_bytes, cudaMemcpyHostToDevice,
                           h->copy_stream));
        CK(cudaEventRecord(h->ev_copied[i & 1], h->copy_stream));
        return EMB200_OK;
    };
    if (m) {
        rc = copy_in(0);
        if (rc) return rc;
    }
    for (size_t i = 0; i < nch; i++) {
        const size_t r0 = starts[i], mc = starts[i + 1] - r0;
        // Chunk i + 1 goes into the buffer of chunk i - 1 once that search is done.
        if (i + 1 < nch) {
            rc = copy_in(i + 1);
            if (rc) return rc;
        }
        CK(cudaStreamWaitEvent(st, h->ev_copied[i & 1], 0));
        rc = assign_dispatch(h, dtype, stage_of(i), nullptr, mc, h->st_labels.p, h->st_dist.p, st);
        if (rc) return rc;
        CK(cudaEventRecord(h->ev_done[i & 1], st));
        CK(cudaMemcpyAsync(labels + r0, h->st_labels.p, mc * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(dist + r0, h->st_dist.p, mc * sizeof(float), cudaMemcpyDeviceToHost, st));
    }
    CK(cudaEventRecord(h->ev1, st));
    CK(cudaEventSynchronize(h->ev1));
    float ms = 0;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    h->stats.rows = m;
    if (use_i8_mode(h, dtype)) h->stats.rows_certified = m;
    h->stats.ms_total = ms;
    return EMB200_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
extern "C" {

int emb200_create(int ordinal, const emb200_opts* opts, emb200_handle** out) {
    if (!out) return EMB200_EINVAL;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return EMB200_EDEVICE;
    if (ordinal < 0 || ordinal >= n) return EMB200_EINVAL;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, ordinal) != cudaSuccess) return EMB200_EDEVICE;
    if (prop.major != 10) return EMB200_EDEVICE;  // built for sm_100a only
    emb200_handle* h = new emb200_handle();
    h->device = ordinal;
    h->sm_count = prop.multiProcessorCount;
    if (opts) h->opts = *opts;
    if (cudaSetDevice(ordinal) != cudaSuccess || cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) ||
        cudaEventCreate(&h->ev0) || cudaEventCreate(&h->ev1) || cudaEventCreate(&h->evk0) ||
        cudaEventCreate(&h->evk1) || h->bounds.ensure(1)) {
        delete h;
        return EMB200_ECUDA;
    }
    *out = h;
    return EMB200_OK;
}

int emb200_destroy(emb200_handle* h) {
    if (!h) return EMB200_OK;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    h->c.release(); h->norms.release(); h->bias.release(); h->bounds.release(); h->nrm16.release();
    h->c_hi.release(); h->c_lo.release(); h->c8.release(); h->c16.release(); h->off8.release();
    h->rows.release(); h->res_labels.release(); h->res_dist.release();
    h->stage.release(); h->st_labels.release(); h->st_dist.release();
    h->part_s.release(); h->part_i.release(); h->redo_rows.release(); h->counters.release();
    h->redo_theta.release(); h->cand.release(); h->cand_count.release(); h->redo2_rows.release();
    h->rkeys.release();
    h->qshift.release(); h->qsel.release(); h->qclip.release(); h->qx.release(); h->qcodes.release();
    h->train.release();
    h->bat.release();
    proposer_release(h);
    report_release(h);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->evk0) cudaEventDestroy(h->evk0);
    if (h->evk1) cudaEventDestroy(h->evk1);
    if (h->copy_stream) {
        cudaStreamSynchronize(h->copy_stream);
        cudaStreamDestroy(h->copy_stream);
    }
    for (int b = 0; b < 2; b++) {
        if (h->ev_copied[b]) cudaEventDestroy(h->ev_copied[b]);
        if (h->ev_done[b]) cudaEventDestroy(h->ev_done[b]);
    }
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return EMB200_OK;
}

const char* emb200_last_error(const emb200_handle* h) {
    if (!h) return "null handle";
    return h->err.c_str();
}

int emb200_set_opts(emb200_handle* h, const emb200_opts* opts) {
    if (!h || !opts) return EMB200_EINVAL;
    if (opts->precision < 0 || opts->precision > 3 || opts->match_kernel < 0 || opts->match_kernel > 2 ||
        (opts->centroid_bits != 0 && opts->centroid_bits != 8 && opts->centroid_bits != 16))
        return fail(h, EMB200_EINVAL, "invalid options");
    bool rebuild = h->opts.centroid_bits != opts->centroid_bits || h->opts.precision != opts->precision;
    h->opts = *opts;
    if (rebuild && h->have_centroids) h->have_centroids = false;  // centroid forms depend on the options
    return EMB200_OK;
}

int emb200_get_stats(const emb200_handle* h, emb200_stats* out) {
    if (!h || !out) return EMB200_EINVAL;
    *out = h->stats;
    return EMB200_OK;
}

int emb200_name(emb200_handle* h, char* buf, size_t len) {
    if (!h || !buf || len == 0) return EMB200_EINVAL;
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, h->device);
    const char* prec = h->opts.precision == EMB200_PREC_FP32   ? "FP32 SIMT"
                       : h->opts.precision == EMB200_PREC_BF16 ? "BF16x3 tcgen05"
                       : h->opts.precision == EMB200_PREC_FP8  ? "FP8 e4m3 tcgen05"
                                                               : "BF16 tcgen05";
    const char* match = h->opts.match_kernel == 0 ? "AVX-512" : h->opts.match_kernel == 1 ? "AVX2" : "portable";
    char ib[64] = "";
    if (h->opts.centroid_bits == 8) snprintf(ib, sizeof ib, ", int8 centroids for i8 rows");
    if (h->opts.centroid_bits == 16) snprintf(ib, sizeof ib, ", int16 centroids (1/%u unit) for i8 rows", 1u << h->ishift);
    snprintf(buf, len, "B200 fused assign (%s search, exact re-score in %s rounding%s), %s", prec, match, ib,
             prop.name);
    return EMB200_OK;
}

int emb200_set_centroids(emb200_handle* h, const float* centroids, size_t k, size_t d) {
    if (!h) return EMB200_EINVAL;
    if (!centroids || k == 0 || d == 0) return fail(h, EMB200_EINVAL, "centroids must be a non-empty k x d array");
    if (k > 0x7FFFFFFF || d > 0x7FFFFFFF) return fail(h, EMB200_EINVAL, "k and d must fit in 31 bits");
    CK(cudaSetDevice(h->device));
    if (h->c.ensure(k * d) || h->norms.ensure((k + kTcBN - 1) / kTcBN * kTcBN) || h->bias.ensure(k))
        return fail(h, EMB200_ENOMEM, "centroid allocation failed");
    h->k = k;
    h->d = d;
    CK(cudaMemcpyAsync(h->c.p, centroids, k * d * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    int rc = prepare_centroids(h);
    if (rc) return rc;
    CK(cudaStreamSynchronize(h->stream));
    h->have_centroids = true;
    h->centroid_version++;
    return EMB200_OK;
}

int emb200_set_bias(emb200_handle* h, const float* bias, size_t k) {
    if (!h) return EMB200_EINVAL;
    if (!h->have_centroids) return fail(h, EMB200_ESTATE, "set_centroids must be called first");
    if (!bias || k != h->k) return fail(h, EMB200_EINVAL, "bias must have k = %zu entries", h->k);
    h->res_n = 0;  // resident results no longer match the biased centroids
    CK(cudaMemcpyAsync(h->bias.p, bias, k * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    double amax = 0.0;
    for (size_t j = 0; j < k; j++) amax = std::max(amax, std::fabs((double)bias[j]));
    if (!(amax < INFINITY)) amax = INFINITY;
    const double prev = h->bias_absmax;
    int rc = apply_bias(h, h->bias.p);
    h->bias_absmax = prev + amax;  // biases accumulate until the next set_centroids
    if (rc) return rc;
    CK(cudaStreamSynchronize(h->stream));
    return EMB200_OK;
}

int emb200_assign_f32(emb200_handle* h, const float* x, size_t m, uint32_t* labels, float* dist) {
    return assign_host(h, EMB200_F32, x, m, labels, dist);
}
int emb200_assign_i8(emb200_handle* h, const int8_t* x, size_t m, uint32_t* labels, float* dist) {
    return assign_host(h, EMB200_I8, x, m, labels, dist);
}
int emb200_assign_u8(emb200_handle* h, const uint8_t* x, size_t m, uint32_t* labels, float* dist) {
    return assign_host(h, EMB200_U8, x, m, labels, dist);
}

int emb200_assign_device(emb200_handle* h, int dtype, const void* x_dev, size_t m, uint32_t* labels_dev,
                         float* dist_dev, void* stream) {
    int rc = check_ready(h, dtype);
    if (rc) return rc;
    if (m > 0xFFFFFFFFull) return fail(h, EMB200_EINVAL, "more than 2^32 - 1 rows in one call");
    if (m && (!x_dev || !labels_dev || !dist_dev)) return fail(h, EMB200_EINVAL, "null buffer");
    cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
    return assign_dispatch(h, dtype, x_dev, nullptr, m, labels_dev, dist_dev, st);
}

int emb200_load_rows(emb200_handle* h, int dtype, const void* x, size_t n, size_t d) {
    if (!h) return EMB200_EINVAL;
    if (dtype < 0 || dtype > 2) return fail(h, EMB200_EINVAL, "unknown dtype %d", dtype);
    if (!x || n == 0 || d == 0) return fail(h, EMB200_EINVAL, "x must be a non-empty row-major n x d array");
    if (n > 0xFFFFFFFFull) return fail(h, EMB200_EINVAL, "more than 2^32 - 1 rows: subsample or shard the input");
    CK(cudaSetDevice(h->device));
    size_t bytes = n * d * elt_size(dtype);
    if (h->rows.ensure(bytes)) return fail(h, EMB200_ENOMEM, "cannot hold %zu bytes of rows", bytes);
    CK(cudaMemcpyAsync(h->rows.p, x, bytes, cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->rows_dtype = dtype;
    h->rows_n = n;
    h->rows_d = d;
    h->res_n = 0;
    return EMB200_OK;
}

int emb200_assign_resident(emb200_handle* h, uint32_t* labels, float* dist) {
    if (!h) return EMB200_EINVAL;
    if (h->rows_dtype < 0) return fail(h, EMB200_ESTATE, "load_rows must be called first");
    int rc = check_ready(h, h->rows_dtype);
    if (rc) return rc;
    if (h->rows_d != h->d) return fail(h, EMB200_EINVAL, "rows have d = %zu, centroids d = %zu", h->rows_d, h->d);
    if (h->res_labels.ensure(h->rows_n) || h->res_dist.ensure(h->rows_n))
        return fail(h, EMB200_ENOMEM, "result allocation failed");
    h->res_n = 0;
    h->stats = emb200_stats{};
    cudaStream_t st = h->stream;
    CK(cudaEventRecord(h->ev0, st));
    rc = assign_dispatch(h, h->rows_dtype, h->rows.p, nullptr, h->rows_n, h->res_labels.p, h->res_dist.p, st);
    if (rc) return rc;
    CK(cudaEventRecord(h->ev1, st));
    if (labels) CK(cudaMemcpyAsync(labels, h->res_labels.p, h->rows_n * 4, cudaMemcpyDeviceToHost, st));
    if (dist) CK(cudaMemcpyAsync(dist, h->res_dist.p, h->rows_n * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    float ms = 0;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    h->stats.rows = h->rows_n;
    if (use_i8_mode(h, h->rows_dtype)) h->stats.rows_certified = h->rows_n;
    h->stats.ms_total = ms;
    h->res_n = h->rows_n;
    h->res_version = h->centroid_version;
    return EMB200_OK;
}

int emb200_resolve_recipe(size_t n, size_t d, size_t k, const emb200_config* cfg, emb200_recipe* out,
                          uint64_t* epoch_rows, size_t max_epochs) {
    if (!cfg || !out) return EMB200_EINVAL;
    Recipe r = resolve_recipe(n, d, k, *cfg);
    out->batch_size = r.batch_size;
    out->alpha0 = r.alpha0;
    out->n_epochs = r.epoch_rows.size();
    out->total_steps = r.total_steps;
    out->unused_threshold = r.unused_threshold;
    if (epoch_rows)
        for (size_t i = 0; i < r.epoch_rows.size() && i < max_epochs; i++) epoch_rows[i] = r.epoch_rows[i];
    return EMB200_OK;
}

double emb200_scheduled_alpha(double alpha0, size_t step, size_t total) { return scheduled_alpha(alpha0, step, total); }

int emb200_measure_simt_peak(int ordinal, double* tflops, double* tflops_paired) {
    if (!tflops || !tflops_paired) return EMB200_EINVAL;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || ordinal < 0 || ordinal >= n) return EMB200_EDEVICE;
    if (cudaSetDevice(ordinal) != cudaSuccess) return EMB200_ECUDA;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ordinal) != cudaSuccess) return EMB200_ECUDA;
    const int blocks = sms * 8, threads = 256, iters = 1 << 14;  // 64 warps per SM
    float* out = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = EMB200_OK;
    if (cudaMalloc(&out, (size_t)blocks * threads * sizeof(float)) != cudaSuccess) return EMB200_ENOMEM;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) rc = EMB200_ECUDA;
    const double flops = 2.0 * 8.0 * (double)iters * blocks * threads;
    for (int paired = 0; paired < 2 && rc == EMB200_OK; paired++) {
        float best = 1e30f;
        for (int rep = 0; rep < 6; rep++) {  // the first launches warm up; the best of the rest
            cudaEventRecord(e0);
            if (paired) k_simt_peak<true><<<blocks, threads>>>(out, iters, 0.999999f, 1e-7f);
            else k_simt_peak<false><<<blocks, threads>>>(out, iters, 0.999999f, 1e-7f);
            cudaEventRecord(e1);
            if (cudaEventSynchronize(e1) != cudaSuccess) {
                rc = EMB200_ECUDA;
                break;
            }
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep >= 2) best = std::min(best, ms);
        }
        (paired ? *tflops_paired : *tflops) = flops / (best * 1e-3) / 1e12;
    }
    if (cudaGetLastError() != cudaSuccess) rc = EMB200_ECUDA;
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(out);
    return rc;
}

int emb200_measure_mma_peak(int ordinal, double* tflops_1sm, double* tflops_2sm) {
    if (!tflops_1sm || !tflops_2sm) return EMB200_EINVAL;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || ordinal < 0 || ordinal >= n) return EMB200_EDEVICE;
    if (cudaSetDevice(ordinal) != cudaSuccess) return EMB200_ECUDA;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ordinal) != cudaSuccess) return EMB200_ECUDA;
    const int iters = 1 << 16;
    int* err = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = EMB200_OK;
    if (cudaMalloc(&err, sizeof(int)) != cudaSuccess) return EMB200_ENOMEM;
    cudaMemset(err, 0, sizeof(int));
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) rc = EMB200_ECUDA;
    if (cudaFuncSetAttribute(k_mma_peak<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPeakSmem) !=
            cudaSuccess ||
        cudaFuncSetAttribute(k_mma_peak<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPeakSmem) !=
            cudaSuccess)
        rc = EMB200_ECUDA;
    for (int pair = 0; pair < 2 && rc == EMB200_OK; pair++) {
        // 2 x 128 x 256 x 16 flops per CTA and MMA step either way (a pair's
        // M = 256 instruction covers two SMs)
        const int ctas = pair ? sms / 2 * 2 : sms;
        const double flops = 2.0 * 128 * 256 * 16 * 4.0 * iters * ctas;
        float best = 1e30f;
        for (int rep = 0; rep < 5 && rc == EMB200_OK; rep++) {
            cudaEventRecord(e0);
            if (pair) {
                cudaLaunchConfig_t lc = {};
                lc.gridDim = dim3((unsigned)ctas);
                lc.blockDim = dim3(128);
                lc.dynamicSmemBytes = kPeakSmem;
                cudaLaunchAttribute at[1];
                at[0].id = cudaLaunchAttributeClusterDimension;
                at[0].val.clusterDim.x = 2;
                at[0].val.clusterDim.y = 1;
                at[0].val.clusterDim.z = 1;
                lc.attrs = at;
                lc.numAttrs = 1;
                if (cudaLaunchKernelEx(&lc, k_mma_peak<true>, iters, err) != cudaSuccess) rc = EMB200_ECUDA;
            } else {
                k_mma_peak<false><<<ctas, 128, kPeakSmem>>>(iters, err);
            }
            cudaEventRecord(e1);
            if (cudaEventSynchronize(e1) != cudaSuccess) {
                rc = EMB200_ECUDA;
                break;
            }
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep >= 1) best = std::min(best, ms);
        }
        (pair ? *tflops_2sm : *tflops_1sm) = flops / (best * 1e-3) / 1e12;
    }
    int e = 0;
    if (rc == EMB200_OK && (cudaMemcpy(&e, err, sizeof e, cudaMemcpyDeviceToHost) != cudaSuccess || e)) rc = EMB200_ECUDA;
    if (cudaGetLastError() != cudaSuccess) rc = EMB200_ECUDA;
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(err);
    return rc;
}

int emb200_set_abort_test(emb200_handle* h, int stall_tile, uint64_t stall_ns) {
    if (!h) return EMB200_EINVAL;
    if (stall_tile < 0 || stall_ns == 0) {
        h->stall_tile = 0;
        h->stall_ns = 0;
        return EMB200_OK;
    }
    h->stall_tile = stall_tile;
    h->stall_ns = stall_ns;
    return EMB200_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Search without allocation: emb200_assign_f32_noalloc.
//
// Some callers cannot call cudaMalloc at the moment they need a search: a host
// program whose GPU memory is owned by its own pool or budget (a database or
// serving runtime that forbids allocations outside its allocator), or code on a
// latency-critical path where an allocation could stall, fragment memory or fail
// under a full device. For them this entry point takes every input and output
// from the caller and keeps its own working memory (centroid norms, error
// bounds, per-row candidate pairs, the list of rows to re-search) in one static
// device array of kNoAllocScratchBytes, which exists once per GPU that loads the
// library and is held until the process exits. It runs the FP32 search with the
// exact certification and re-search (CpuAssigner's bits, like every other entry
// point), all enqueued on the caller's stream with no host synchronisation.
//
// Every call shares that array and finds it as the previous call left it: the
// counters that must start at zero are cleared by each call. Two calls that
// overlap on the GPU (concurrent streams, or several host threads) race on it;
// the caller must order them.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t kNoAllocMaxRows = 65536;    // EMB200_NOALLOC_MAX_ROWS
constexpr size_t kNoAllocMaxK = 262144;      // EMB200_NOALLOC_MAX_K
constexpr size_t kNoAllocPartBytes = (size_t)8 << 20;  // per-row candidate pairs of all column splits
constexpr size_t kNoAllocScratchBytes = 256 + 256 + kNoAllocMaxK * 4 + kNoAllocPartBytes + kNoAllocMaxRows * 8;

__device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch in the current device's context. Host code
// must not use the symbol itself as an address. The lookup is repeated on every
// call (a host-side query, no allocation): a cached address would go stale when
// the caller resets the device or switches to another context on the same
// device, where the module's array can sit elsewhere.
int noalloc_scratch(void** out) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return EMB200_ECUDA;
    *out = p;
    return EMB200_OK;
}

}  // namespace

extern "C" int emb200_assign_f32_noalloc(const float* x_dev, size_t m, size_t d, const float* centroids_dev,
                                         size_t k, uint32_t* labels_dev, float* dist_dev, int match_kernel,
                                         void* stream) {
    if (m > kNoAllocMaxRows || k > kNoAllocMaxK) return EMB200_ELIMIT;
    // d rounded up to 64 (the padded width the centroid preparation takes) must fit in an int.
    if (d == 0 || k == 0 || d > (size_t)0x7FFFFFFF - 63) return EMB200_EINVAL;
    if (match_kernel < 0 || match_kernel > 2) return EMB200_EINVAL;
    if (m == 0) return EMB200_OK;
    if (!x_dev || !centroids_dev || !labels_dev || !dist_dev) return EMB200_EINVAL;
    cudaGetLastError();  // the launch check below reports this call's launches only
    void* base = nullptr;
    int rc = noalloc_scratch(&base);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    uint8_t* p = (uint8_t*)base;
    Bounds* bounds = (Bounds*)p;
    uint32_t* ctr = (uint32_t*)(p + 256);  // [0] rows to re-search, [1] certified rows
    float* norms = (float*)(p + 512);
    float* part_s = (float*)(p + 512 + kNoAllocMaxK * 4);
    const int row_tiles = (int)((m + kSimtBM - 1) / kSimtBM);
    const int ntiles = (int)((k + kSimtBN - 1) / kSimtBN);
    const size_t pair_bytes = 2 * sizeof(float) + 2 * sizeof(uint32_t);
    int nsplit = 1;
    int sms = 148;
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (row_tiles < 2 * sms) nsplit = std::min(ntiles, (2 * sms + row_tiles - 1) / row_tiles);
    nsplit = (int)std::max<size_t>(1, std::min<size_t>((size_t)nsplit, kNoAllocPartBytes / (m * pair_bytes)));
    uint32_t* part_i = (uint32_t*)(part_s + (size_t)nsplit * m * 2);
    uint32_t* redo = (uint32_t*)(p + 512 + kNoAllocMaxK * 4 + kNoAllocPartBytes);
    float* redo_theta = (float*)(redo + kNoAllocMaxRows);  // written by the certification, unused without refine
    if (cudaMemsetAsync(p, 0, 512, st) != cudaSuccess) return EMB200_ECUDA;  // bounds and counters start at zero
    // Norms and the certification bounds (no BF16 split: the search here is FP32).
    k_prep_centroids<<<(unsigned)((k + 7) / 8), 256, 0, st>>>(centroids_dev, (int)k, (int)d, norms, bounds, nullptr,
                                                              nullptr, (int)((d + 63) / 64 * 64));
    const int vec4 = (d % 4 == 0 && ((uintptr_t)x_dev & 15) == 0 && ((uintptr_t)centroids_dev & 15) == 0) ? 1 : 0;
    k_assign_simt<float><<<dim3(row_tiles, nsplit), kSimtThreads, 0, st>>>(
        x_dev, nullptr, (int)m, (int)d, centroids_dev, norms, (int)k, part_s, part_i, vec4);
    float ka, kb;
    bound_coefficients(EMB200_PREC_FP32, EMB200_F32, d, false, &ka, &kb);
    // No refine pass here: uncertified rows (rare with FP32 scores) go straight to the exact search.
    k_certify<float><<<(unsigned)((m + 7) / 8), 256, 0, st>>>(
        x_dev, nullptr, (int)m, (int)d, centroids_dev, norms, (int)k, part_s, part_i, nsplit, bounds, ka, kb,
        match_kernel, labels_dev, dist_dev, redo, ctr, ctr + 1, nullptr, redo_theta, 0.0f, 0.0f);
    k_research_cta<float><<<sms * 2, 256, 0, st>>>(x_dev, nullptr, (int)d, centroids_dev, norms, (int)k,
                                                    match_kernel, redo, ctr, labels_dev, dist_dev);
    return cudaGetLastError() == cudaSuccess ? EMB200_OK : EMB200_ECUDA;
}

#include "engine_batched.inc"
#include "engine_train.inc"
#include "engine_proposer.inc"
#include "engine_quant.inc"
#include "engine_report.inc"
