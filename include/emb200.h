/*
 * emb200.h - C ABI of the B200 e-means engine (libemb200.so).
 *
 * The engine is a drop-in backend for the nearest-centroid search and the
 * training loop of the Rust crate `emeans` (andrewluetgers/e-means). Each
 * entry point names the reference interface it replaces (paths inside the
 * reference project). Conventions:
 *   - every call returns 0 on success and a negative EMB200_E* code on error;
 *     emb200_last_error() then describes it. No call aborts or throws;
 *   - host pointers are caller-owned and only read or written during the call;
 *     device memory is owned by the handle and freed by emb200_destroy;
 *   - one thread at a time per handle (the trait methods take &mut self);
 *     distinct handles are independent;
 *   - every computation runs on the GPU; there is no CPU fallback. A missing
 *     or unsupported GPU is reported by emb200_create.
 */
#ifndef EMB200_H
#define EMB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct emb200_handle emb200_handle;

/* Error codes. */
#define EMB200_OK 0
#define EMB200_EINVAL -1  /* bad argument or shape (the reference asserts or returns Err) */
#define EMB200_ECUDA -2   /* CUDA runtime or driver error */
#define EMB200_ENOMEM -3  /* device allocation failed */
#define EMB200_ESTATE -4  /* call out of order (e.g. assign before set_centroids) */
#define EMB200_EDEVICE -5 /* no usable sm_100 device */
#define EMB200_ELIMIT -6  /* size beyond the limits of emb200_assign_f32_noalloc */

/* Row element types (src/lib.rs:47-71, trait Scalar: f32, i8, u8). */
#define EMB200_F32 0
#define EMB200_I8 1
#define EMB200_U8 2

/* Search precision of the main contraction. Every mode returns the labels and
 * distances of the reference CpuAssigner bit for bit: the fast contraction
 * keeps the top-2 candidates per row with a rigorous error bound, both are
 * re-scored with the reference's own f32 arithmetic, and rows the bound cannot
 * certify are searched again exactly. */
#define EMB200_PREC_FP32 0  /* FP32 SIMT contraction */
#define EMB200_PREC_BF16 1  /* tcgen05 BF16, three-term split (hi*hi + hi*lo + lo*hi), FP32 accumulate */
#define EMB200_PREC_BF16X1 2 /* tcgen05 BF16 single term, FP32 accumulate (wider bound, more re-search) */
#define EMB200_PREC_FP8 3    /* tcgen05 FP8 e4m3 operands (kind::f8f6f4), a power-of-two scale per row and per
                                centroid, FP32 accumulate; f32 rows with d <= 256 (else as BF16X1). Its error
                                bound (e4m3 unit roundoff 2^-4) is wide: most rows go on to the refine pass */

/* Centroid representation for i8 rows (src/cpu_i8.rs:21-25). */
#define EMB200_CENTROIDS_F32 0 /* CpuAssigner semantics: rows widened to f32 */
#define EMB200_CENTROIDS_I8 8  /* CpuI8Assigner(CentroidBits::I8): centroids rounded to i8, exact integer ranking */
#define EMB200_CENTROIDS_I16 16 /* CpuI8Assigner(CentroidBits::I16): centroids rounded to 1/2^s of a unit
                                   (s <= 7 from d, src/cpu_i8.rs:95-107), exact integer ranking */

/* Which CpuAssigner kernel's f32 rounding the exact re-score reproduces
 * (src/cpu.rs:13-33: AVX-512 on CPUs that have it, else AVX2+FMA, else portable). */
#define EMB200_MATCH_AVX512 0
#define EMB200_MATCH_AVX2 1
#define EMB200_MATCH_PORTABLE 2

typedef struct {
    int precision;     /* EMB200_PREC_* (default FP32) */
    int centroid_bits; /* EMB200_CENTROIDS_* (default F32) */
    int match_kernel;  /* EMB200_MATCH_* (default AVX512) */
    int train_eager;   /* 1: launch the training loop's kernels one by one instead of
                          capturing each epoch as a CUDA graph and replaying it (default 0) */
    int batched_streams; /* emb200_train_batched: 0 (default) runs the instances in lockstep with
                            batched kernels where supported; 1 gives each instance its own stream */
    int reserved[3];
} emb200_opts;

/* Config, src/lib.rs:104-124. Optional fields use sentinels:
 * batch_size 0 = None, alpha0 <= 0 = None, unused_threshold < 0 = None. */
typedef struct {
    double nepochs;
    int batch_law; /* 0 Auto, 1 Throughput, 2 Quality (src/lib.rs:94-101) */
    uint64_t batch_size;
    double alpha0;
    float unused_threshold;
    float balance;
    uint64_t seed;
    int verbose;
    int closing_f64; /* 0: f32 pass sums as the reference (bit-exact); 1: FP64 pass sums */
} emb200_config;

/* Recipe, src/lib.rs:143-149 (epoch_rows written to a caller array). */
typedef struct {
    uint64_t batch_size;
    double alpha0;
    uint64_t n_epochs;
    uint64_t total_steps;
    float unused_threshold;
} emb200_recipe;

/* Counters of the last assign / train call. */
typedef struct {
    uint64_t rows;           /* rows searched */
    uint64_t rows_certified; /* rows whose fast top-2 the error bound certified */
    uint64_t rows_researched; /* rows searched exhaustively with exact arithmetic */
    uint64_t kernel_launches; /* kernels launched by the call */
    double ms_total;          /* device time of the call (CUDA events) */
    int32_t fast_kernel;      /* fast contraction used: 0 FP32 SIMT, 1 tcgen05 BF16, 2 exact int8 (dp4a),
                                 3 exact int8 (tcgen05 kind::i8), 4 tcgen05 FP8 e4m3 */
    int32_t fast_aborted;     /* 1 if a bounded wait in the fast kernel gave up (rows then re-searched) */
    uint64_t rows_refined;    /* uncertified rows sent through the candidate-collecting refine pass (lockstep
                                 batched training: batch rows settled by the exhaustive search, all steps) */
    double fast_ms;           /* device time of the fast contraction kernel(s) (CUDA events, summed) */
    uint64_t fast_launches;   /* launches of the fast contraction kernel */
    uint64_t rows_proposed;   /* proposer assign: rows searched in their proposed groups only */
    uint64_t rows_lowconf;    /* proposer assign: rows below the confidence threshold (full search) */
    double propose_ms;        /* proposer assign: device time of the proposals (network or group centroids) */
    uint64_t groups_searched; /* proposer assign: (row, group) pairs scored by the grouped search */
    double update_ms;         /* train with opts.train_eager: device time of the per-batch update kernels
                                 (label histogram to revival; CUDA events around each batch's chain) */
    uint64_t update_bytes;    /* their algorithmic bytes: each batch row re-read once, per-row and
                                 per-cluster arrays, centroids and sums read and written once */
    double late_fit_ms;       /* emb200_train_proposed: host time of building and fitting the proposer */
    double late_epochs_ms;    /* emb200_train_proposed: device time of the epochs searched through it */
} emb200_stats;

/* ---- lifecycle ---------------------------------------------------------- */

/* Replaces CudaAssigner::new (src/cuda.rs:69-91). opts may be NULL (defaults). */
int emb200_create(int ordinal, const emb200_opts* opts, emb200_handle** out);
int emb200_destroy(emb200_handle* h);
/* Description of the last error on this handle (never NULL). */
const char* emb200_last_error(const emb200_handle* h);
/* Assigner::name, src/lib.rs:83. */
int emb200_name(emb200_handle* h, char* buf, size_t len);
/* Set or read options after creation (takes effect at the next call). */
int emb200_set_opts(emb200_handle* h, const emb200_opts* opts);
int emb200_get_stats(const emb200_handle* h, emb200_stats* out);

/* ---- Assigner trait (src/lib.rs:75-91) ---------------------------------- */

/* Assigner::set_centroids, src/lib.rs:77 (CpuAssigner src/cpu.rs:84-93,
 * CpuI8Assigner src/cpu_i8.rs:73-110): k x d row-major f32, host memory. */
int emb200_set_centroids(emb200_handle* h, const float* centroids, size_t k, size_t d);
/* Assigner::set_bias, src/lib.rs:81 (src/cpu.rs:95-99, src/cpu_i8.rs:112-117):
 * adds bias[j] to centroid j's score until the next set_centroids. */
int emb200_set_bias(emb200_handle* h, const float* bias, size_t k);
/* AssignRows<T>::assign, src/lib.rs:90 (src/cpu.rs:108-167, src/cpu_i8.rs:130-191):
 * m rows of d elements (host, row-major) -> labels[m], dist[m] (host). */
int emb200_assign_f32(emb200_handle* h, const float* x, size_t m, uint32_t* labels, float* dist);
int emb200_assign_i8(emb200_handle* h, const int8_t* x, size_t m, uint32_t* labels, float* dist);
int emb200_assign_u8(emb200_handle* h, const uint8_t* x, size_t m, uint32_t* labels, float* dist);

/* Same as emb200_assign_* with device pointers, enqueued on `stream`
 * (cudaStream_t, or NULL for the handle's stream); no host copies, no sync. */
int emb200_assign_device(emb200_handle* h, int dtype, const void* x_dev, size_t m, uint32_t* labels_dev,
                         float* dist_dev, void* stream);

/* ---- resident rows (rows uploaded once, src/cuda.rs:8-9 streamed them) ---- */

/* Upload n x d rows of dtype once; they stay in HBM for assign_resident/train. */
int emb200_load_rows(emb200_handle* h, int dtype, const void* x, size_t n, size_t d);
/* assign() (src/lib.rs:512-520) over the resident rows with the current
 * centroids. labels/dist: host arrays of n, or NULL to keep results on device. */
int emb200_assign_resident(emb200_handle* h, uint32_t* labels, float* dist);

/* Test of the bounded-wait abort path (no counterpart in the reference: its
 * CudaAssigner has no device-side waits). With stall_tile >= 0 and stall_ns > 0,
 * the next fast tensor-core searches on this handle (BF16 and int8 kind::i8)
 * make their first epilogue warp wait, at that centroid tile of each CTA, on a
 * barrier that nothing completes, bounded by stall_ns. The wait runs out, the
 * kernel lets its copies and MMAs in flight finish, frees its TMEM and flags the
 * abort; the call then settles every row with the exact search (the same labels
 * and distances) and reports stats.fast_aborted = 1. stall_tile < 0 or
 * stall_ns = 0 turns it off (the default). */
int emb200_set_abort_test(emb200_handle* h, int stall_tile, uint64_t stall_ns);

/* FP32 SIMT throughput of device `ordinal` (no counterpart in the reference): the
 * measured denominator of the FP32 search's roofline. Runs 8 independent FMA
 * chains per thread over 64 warps per SM, scalar fma.rn.f32 (tflops) and paired
 * fma.rn.f32x2 (tflops_paired); best of four timed launches each, CUDA events. */
int emb200_measure_simt_peak(int ordinal, double* tflops, double* tflops_paired);

/* tcgen05 BF16 MMA throughput of this device (TF/s) with operands resident in
 * shared memory: cta_group::1 M=128 N=256 (the shape k_assign_tc issues) and a
 * CTA pair's cta_group::2 M=256 N=256. A measurement for rooflines; no
 * counterpart in the reference. */
int emb200_measure_mma_peak(int ordinal, double* tflops_1sm, double* tflops_2sm);

/* ---- training (src/lib.rs:201-225 and 348-491) --------------------------- */

/* resolve_recipe, src/lib.rs:201-225. epoch_rows: array of max_epochs. */
int emb200_resolve_recipe(size_t n, size_t d, size_t k, const emb200_config* cfg, emb200_recipe* out,
                          uint64_t* epoch_rows, size_t max_epochs);
/* scheduled_alpha, src/lib.rs:194-198. */
double emb200_scheduled_alpha(double alpha0, size_t step, size_t total);

/* train (src/lib.rs:348-491) on the resident rows, entirely on the device.
 * Outputs (host, caller-allocated, any may be NULL): centroids k*d, labels n
 * (last-pass labels, UINT32_MAX where unset), objective n_epochs, n_splits.
 * The trained centroids also become the handle's current centroids. */
int emb200_train(emb200_handle* h, const emb200_config* cfg, size_t k, float* centroids, uint32_t* labels,
                 double* objective, uint64_t* n_splits, emb200_recipe* recipe);

/* ---- batched instances (PQ sub-codebooks, per-list IVF refinements) ----------
 *
 * train() (src/lib.rs:348-491) run for `count` independent instances at once,
 * each over rows [row0, row0 + n) of the resident rows (same d and dtype, same
 * config) with its own k. By default the instances advance in lockstep, one
 * global step at a time: each step is a chain of batched kernels over all
 * instances (the search a persistent kernel over an (instance, row tile, column
 * split) work queue, FP32 SIMT, with its tile shape and split policy picked by a
 * measured sweep cached in $EMB200_AUTOTUNE_CACHE or
 * $HOME/.cache/emb200/autotune.txt), captured once as a CUDA graph and replayed
 * until the longest instance is done. This covers CpuAssigner semantics
 * (centroid_bits 0), balance 0 and up to 256 instances; otherwise, or with
 * opts.batched_streams = 1, each instance runs on its own stream with its epochs
 * replayed as CUDA graphs, at most max_concurrency at a time (0: 16). Outputs
 * are concatenated in instance order: centroids sum(k_i) x d, labels sum(n_i)
 * (instance-local row order), objective sum(n_epochs_i), n_splits[count]. Each
 * instance's results equal a single train() call's. */
typedef struct {
    uint64_t row0;
    uint64_t n;
    uint64_t k;
} emb200_instance;
int emb200_train_batched(emb200_handle* h, const emb200_config* cfg, const emb200_instance* inst, size_t count,
                         size_t max_concurrency, float* centroids, uint32_t* labels, double* objective,
                         uint64_t* n_splits);
/* The search tile the autotuner chose for the last lockstep emb200_train_batched
 * call on this handle (no counterpart in the reference): rows x centroids per
 * work item, and whether an item covers one centroid tile (split_all = 1) or all
 * of them. EMB200_ESTATE before any lockstep run. */
int emb200_batched_search_choice(const emb200_handle* h, int* rows, int* centroids, int* split_all);

/* ---- learned proposer (no counterpart in the reference's code) -----------
 *
 * For large k: the centroids are partitioned into G groups by e-means on the
 * centroids themselves (this engine's own train(), k = G), and a small BF16
 * network d -> H -> H -> G (ReLU, FP32 accumulation, trained on the GPU with
 * this library's forward and backward kernels and Adam) predicts from a row the
 * group of its nearest centroid. The proposer assign scores each row exactly
 * against the centroids of its `top` most likely groups only (tcgen05, over a
 * group-sorted copy of the centroids), re-scores the two best in the
 * reference's f32 rounding, and certifies the label against the error bound of
 * the fast contraction. Rows whose top-`top` softmax mass is below `confidence`,
 * or whose margin among the candidates the bound cannot certify, take the full
 * exact search instead. Labels are therefore the exact argmin over the
 * proposed groups, and equal the full search's wherever the nearest centroid
 * lies in them (recall@1 is measured, not guaranteed).
 *
 * mode EMB200_PROPOSER_CENTROIDS replaces the network by the nearest `top`
 * group centroids (the method without a learned part). */
#define EMB200_PROPOSER_MLP 0
#define EMB200_PROPOSER_CENTROIDS 1
typedef struct {
    uint32_t groups;      /* G <= 512; 0 = 256 */
    uint32_t hidden;      /* H, a multiple of 8; 0 = 512 */
    uint32_t top;         /* groups searched per row, <= 32 and <= G; 0 = 8 */
    uint32_t mode;        /* EMB200_PROPOSER_* */
    float confidence;     /* MLP mode: rows below this top-`top` softmax mass take the full search */
    uint32_t batch;       /* training mini-batch rows; 0 = 4096 */
    float lr;             /* Adam learning rate (decays linearly to lr/10 over a train call); 0 = 2e-3 */
    float group_epochs;   /* e-means epochs of the grouping; 0 = 5 */
    uint64_t seed;        /* grouping and initialisation seed */
    float mass;           /* MLP mode: search only the fewest of the `top` groups whose softmax mass
                             reaches this (<= 0: all `top`) */
    uint32_t reserved[3];
} emb200_proposer_config;

/* Groups the current centroids, builds the group-sorted copy and initialises the
 * network (input standardisation from the resident rows when present). d <= 128. */
int emb200_proposer_init(emb200_handle* h, const emb200_proposer_config* cfg);
/* train() (src/lib.rs:348-491) with the learned proposer in its last
 * `late_epochs` epochs (no counterpart in the reference; at least one
 * full-search epoch always comes first). The epochs before run as emb200_train;
 * the labels the full search gives in the epoch just before the late ones train
 * the network (emb200_proposer_init with *pcfg over the centroids of that moment,
 * then emb200_proposer_train for net_steps Adam steps), and each late batch is
 * searched through the proposer: the exact kernel scores each row against its
 * proposed groups' centroids only, with the certification, the refine pass over
 * all k and the full search for low-confidence rows as in
 * emb200_assign_proposed_*. A label then differs from train()'s only where the
 * nearest centroid lies outside the proposed groups. Resident f32 rows, d <= 128,
 * balance 0. Outputs as emb200_train; stats count the proposed rows. The
 * proposer stays on the handle for later emb200_assign_proposed_* calls. */
int emb200_train_proposed(emb200_handle* h, const emb200_config* cfg, size_t k, const emb200_proposer_config* pcfg,
                          uint32_t late_epochs, uint32_t net_steps, float* centroids, uint32_t* labels,
                          double* objective, uint64_t* n_splits, emb200_recipe* recipe);
/* Adam steps on mini-batches of resident rows with known labels (host array of
 * rows_n labels, e.g. train()'s output; UINT32_MAX rows are skipped): targets
 * are the labels' groups. losses: optional host array of `steps` mean losses. */
int emb200_proposer_train(emb200_handle* h, const uint32_t* labels, size_t n, uint32_t steps, float* losses);
/* Mode, groups per row, confidence threshold and mass target for later assigns. */
int emb200_proposer_set(emb200_handle* h, uint32_t mode, uint32_t top, float confidence, float mass);
/* Network parameters as one f32 array: input mean[d], input 1/std[d], W1[H][d],
 * b1[H], W2[H][H], b2[H], W3[G][H], b3[G], each block starting at a multiple of 8. */
size_t emb200_proposer_param_count(const emb200_handle* h);
int emb200_proposer_get_params(emb200_handle* h, float* params, size_t count);
int emb200_proposer_set_params(emb200_handle* h, const float* params, size_t count);
/* Mean cross-entropy loss of m host rows against target groups, and its gradient
 * in the parameter layout (input statistics entries zero). */
int emb200_proposer_grad(emb200_handle* h, const float* x, const uint32_t* targets, size_t m, float* grads,
                         float* loss);
/* Network logits of m host rows (m <= 65536), [m][G]: fused = 1 from the fused
 * tcgen05 forward pass (H of 256 or 512, G of 128 or 256, d a multiple of 8),
 * fused = 0 from the GEMM forward pass used in training. */
int emb200_proposer_logits(emb200_handle* h, const float* x, size_t m, float* logits, int fused);
/* Group of every centroid (k entries). */
int emb200_proposer_groups(emb200_handle* h, uint32_t* group_of);
/* Proposals for m host rows: groups[m][top] (most likely first), confidence[m]
 * and counts[m] (how many of them the proposer assign searches); confidence and
 * counts may be NULL. */
int emb200_propose(emb200_handle* h, const float* x, size_t m, uint32_t* groups, float* confidence,
                   uint32_t* counts);
/* The proposer assign over the resident f32 rows (labels/dist host arrays of n,
 * or NULL to keep them on the device), or over m device rows on `stream`. */
int emb200_assign_proposed_resident(emb200_handle* h, uint32_t* labels, float* dist);
int emb200_assign_proposed_device(emb200_handle* h, const float* x_dev, size_t m, uint32_t* labels_dev,
                                  float* dist_dev, void* stream);

/* ---- int8 quantizer (src/quantize.rs) ------------------------------------
 *
 * Int8Quantizer on the GPU, bit-exact with the reference: shift = per-dimension
 * mean (f64 sums in row order, then f32), peak = the centred magnitude
 * |x - shift| at rank round((n d - 1) quantile) in f32::total_cmp order, scale =
 * target_peak / peak (1 if peak is not > 0), rounded down to a power of two if
 * asked; code = clamp(round_half_away((x - shift) * scale), -128, 127), NaN -> 0.
 * A quantizer is (d, shift[d], scale), held by the caller. Device pointers
 * (x_dev, sample_dev, codes_dev) must be 16-byte aligned. */

/* Calibration, src/quantize.rs:17-34 (faiss(): {112, 1, 1.0}; clipped(q): {127, 0, q}). */
typedef struct emb200_calibration {
    float target_peak;     /* code magnitude the peak maps to */
    int32_t power_of_two;  /* non-zero: round the scale down to a power of two */
    double quantile;       /* which centred magnitude is the peak: 1.0 = the largest */
} emb200_calibration;

/* Int8Quantizer::fit, src/quantize.rs:45-62, on a host sample (n x d row-major
 * f32, n > 0): writes shift[d] and *scale. */
int emb200_quantizer_fit(emb200_handle* h, const float* sample, size_t n, size_t d, const emb200_calibration* cal,
                         float* shift, float* scale);
/* The same on a sample in device memory. */
int emb200_quantizer_fit_device(emb200_handle* h, const float* sample_dev, size_t n, size_t d,
                                const emb200_calibration* cal, float* shift, float* scale);
/* The same on the resident f32 rows (emb200_load_rows). */
int emb200_quantizer_fit_resident(emb200_handle* h, const emb200_calibration* cal, float* shift, float* scale);
/* Int8Quantizer::encode (src/quantize.rs:65-73) of host rows into host codes
 * (n x d), and the count of values that clip, the numerator of clipped_fraction
 * (:87-95). codes or clipped may be NULL: encode only, or count only. */
int emb200_quantizer_encode(emb200_handle* h, const float* x, size_t n, size_t d, const float* shift, float scale,
                            int8_t* codes, uint64_t* clipped);
/* The same on device rows into device codes, enqueued on `stream` (NULL: the
 * handle's stream); returns when the work is done. */
int emb200_quantizer_encode_device(emb200_handle* h, const float* x_dev, size_t n, size_t d, const float* shift,
                                   float scale, int8_t* codes_dev, uint64_t* clipped, void* stream);
/* Replace the resident f32 rows by their int8 codes: the resident rows become
 * EMB200_I8 rows for emb200_train / emb200_assign_resident. */
int emb200_quantize_resident(emb200_handle* h, const float* shift, float scale, uint64_t* clipped);
/* Int8Quantizer::decode, src/quantize.rs:76-79: out = codes * (1 / scale) + shift
 * (codes and out host n x d f32, e.g. centroids learned on codes). */
int emb200_quantizer_decode(emb200_handle* h, const float* codes, size_t n, size_t d, const float* shift, float scale,
                            float* out);

/* ---- report (src/report.rs) ----------------------------------------------
 *
 * report() on the GPU: per-cluster statistics of the member distances, the
 * nearest other live centroid, prototype families and per-row robust z-scores,
 * from each row's label and squared distance (what assign returns) and the
 * centroids. Values are bit-identical to the reference's, with one rule where
 * the reference leaves the order to its unstable sort: clusters of equal size
 * are taken in index order when families form, and families of equal size
 * keep the order in which they formed. k <= 131072. */

/* ReportConfig, src/report.rs:21-34 (default {1.25, 0, 30}). family_pass picks
 * how families are formed, with the same result either way: 0 = parallel rounds
 * unless their neighbour lists would be too large, 1 = parallel rounds, 2 = the
 * sequential greedy pass. */
typedef struct emb200_report_config {
    float family_radius;
    uint32_t family_pass;
    uint64_t min_local_size;
} emb200_report_config;

/* ClusterStats, src/report.rs:37-56 (distances plain L2; an empty cluster has
 * size 0 and zero statistics, but its nearest centroid is still filled). */
typedef struct emb200_cluster_stats {
    uint32_t size;
    float rms, median, mad, p90, p99, max, looseness;
    uint32_t nearest_centroid;
    float nearest_dist, isolation;
    uint32_t family;
} emb200_cluster_stats;

/* Report's scalars (src/report.rs:78-80), and the sizes of the family arrays. */
typedef struct emb200_report_summary {
    float median_dist, median_rms, median_nearest_dist;
    uint32_t n_families;  /* families, largest first */
    uint32_t n_live;      /* non-empty clusters = total family members */
    uint32_t reserved[3];
} emb200_report_summary;

/* report(labels, sqdist, centroids, d, cfg), src/report.rs:121-241, on host
 * arrays: labels[n] (< k), sqdist[n], centroids k x d. Writes clusters[k],
 * local_z[n], global_z[n] (either may be NULL) and the summary. */
int emb200_report(emb200_handle* h, const uint32_t* labels, const float* sqdist, size_t n, const float* centroids,
                  size_t k, size_t d, const emb200_report_config* cfg, emb200_cluster_stats* clusters,
                  float* local_z, float* global_z, emb200_report_summary* summary);
/* The same on the labels and distances of the last emb200_assign_resident (or
 * emb200_assign_proposed_resident) and the handle's centroids, all in HBM. */
int emb200_report_resident(emb200_handle* h, const emb200_report_config* cfg, emb200_cluster_stats* clusters,
                           float* local_z, float* global_z, emb200_report_summary* summary);
/* Families of the last report (Family, src/report.rs:58-66): leader[F],
 * size[F], share[F], offsets[F + 1] into members[n_live] (members of family f,
 * in decreasing cluster size, are members[offsets[f] .. offsets[f + 1])).
 * F = summary.n_families. Any pointer may be NULL. */
int emb200_report_families(emb200_handle* h, uint32_t* leader, uint64_t* size, double* share, uint32_t* offsets,
                           uint32_t* members);

/* ---- search without allocation (no counterpart in the reference) --------
 *
 * For callers that cannot allocate device memory when they search: programs
 * whose GPU memory belongs to their own pool or budget (a database or serving
 * runtime that forbids cudaMalloc outside its allocator), or latency-critical
 * code where an allocation could stall, fragment memory or fail on a full
 * device. The caller passes everything in device memory: x_dev (m x d f32
 * rows), centroids_dev (k x d f32), labels_dev[m], dist_dev[m]; the work is
 * enqueued on `stream` (cudaStream_t, NULL = the legacy default stream) with no
 * host synchronisation, no handle and no allocation of any kind. Results are
 * those of the FP32 search: labels and distances equal to CpuAssigner's.
 *
 * Working memory is one static device array (9.5 MiB) that every GPU
 * loading the library holds until the process exits. Its device address in the
 * current context is looked up on every call (a host-side query that allocates
 * nothing), so the call stays valid after the caller resets the device or
 * switches contexts. All calls share the array and find the previous call's
 * contents (each call clears what must start at zero): calls that overlap on
 * the GPU race on it and must be ordered by the caller.
 *
 * Limits: m <= EMB200_NOALLOC_MAX_ROWS, k <= EMB200_NOALLOC_MAX_K; larger
 * sizes return EMB200_ELIMIT without doing anything. d must be at most
 * 2^31 - 64 (EMB200_EINVAL beyond). match_kernel: EMB200_MATCH_*. */
#define EMB200_NOALLOC_MAX_ROWS 65536
#define EMB200_NOALLOC_MAX_K 262144
int emb200_assign_f32_noalloc(const float* x_dev, size_t m, size_t d, const float* centroids_dev, size_t k,
                              uint32_t* labels_dev, float* dist_dev, int match_kernel, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* EMB200_H */
