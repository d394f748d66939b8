/*
 * C ABI of the B200 fastPLS fitting library (libfastpls_b200.so).
 *
 * The first block keeps, symbol for symbol, the CUDA ABI that the fastPLS R
 * package links against (fastPLS src/cuda_resident_api.h), so the package's
 * .Call glue (src/cuda_resident_r.cpp) links to this library unchanged.
 * Conventions (unchanged from the reference):
 *   - precision is 32 or 64; FP32 data are IEEE-754 floats;
 *   - matrices are column-major with leading dimension = rows;
 *   - labels are one-based (1..classes); folds are one-based (1..K);
 *   - component paths are strictly increasing and <= the fitted count;
 *   - scaling: 1 = centre, 2 = autoscale (sd with n-1), 3 = none;
 *   - regression metric: 2 = R2, 3 = Q2, 4 = RMSD;
 *   - every pointer is host memory borrowed for the call; outputs are
 *     caller-allocated; functions return 0 (or a handle) on success and 1
 *     (or NULL) on error, writing a NUL-terminated message into `error`
 *     (capacity `error_capacity`); nothing throws across the boundary;
 *   - a handle owns one CUDA stream; calls are synchronous and a handle is
 *     not safe for concurrent calls. Every handle, whatever the method, is
 *     released with fastpls_resident_simpls_destroy.
 * Addition: the four _create functions also take precision 16. The
 * predictors x (and the rows later given to that handle's predict, classify,
 * project and response-sums calls) are then BF16 bit patterns (uint16, the
 * upper half of an IEEE-754 float), kept in BF16 on the device; responses y
 * and every result written back (predictions, scores, exports, sums) are
 * FP32. Arithmetic stays FP64, so a BF16 fit equals the FP64 fit of the
 * BF16-rounded values.
 * Arithmetic: products and reductions are FP64 on the device whatever the
 * storage precision, so results agree with the reference's FP64 CPU path to
 * ~1e-10 relative. The one exception is the batched CV x permutation engine,
 * whose products with its shared n x n Gram run by default as int8 digit
 * products on the tensor cores (fastpls_b200_set_product_digits; results
 * within 1e-5 relative of FP64, ~1e-9 observed; digits = 0 restores FP64).
 */
#ifndef FASTPLS_B200_H
#define FASTPLS_B200_H
#include <stddef.h>
#if defined(__GNUC__)
#define FASTPLS_B200_API __attribute__((visibility("default")))
#else
#define FASTPLS_B200_API
#endif
#ifdef __cplusplus
extern "C" {
#endif

/* ---- reference ABI (fastPLS src/cuda_resident_api.h) ------------------- */

/* replaces src/cuda_resident_api.h:11 -- output = left (rows x inner) *
 * right (inner x columns), accumulated in FP64, returned in `precision`. */
FASTPLS_B200_API int fastpls_cuda_gemm(const void* left, const void* right, int precision,
                      int rows, int inner, int columns, void* output,
                      char* error, size_t error_capacity);

/* replaces src/cuda_resident_api.h:14 -- SIMPLS classification CV.
 * predictions: n x prefix_count labels; scores: n x classes x prefix_count;
 * status per fold: 1 fitted, 2 empty fold, 4 single active class;
 * metrics: accuracy per prefix. oversample/power/seed are accepted and
 * recorded; directions are exact (see the library documentation). */
FASTPLS_B200_API int fastpls_resident_simpls_cv_classification(
    const void* predictors, const int* labels, const int* folds,
    int precision, int n, int p, int classes, const int* prefixes,
    int prefix_count, int scaling, int lda, int oversample, int power,
    unsigned long long seed, int store_predictions, int store_scores,
    int* predictions, void* scores, int* status, double* metrics,
    char* error, size_t error_capacity);

/* replaces src/cuda_resident_api.h:20 -- SIMPLS regression CV.
 * predictions: n x q x prefix_count (double); metrics per prefix is the
 * selected metric; q2 / rmsd / observed_r2 are always filled. */
FASTPLS_B200_API int fastpls_resident_simpls_cv_regression(
    const void* predictors, const void* responses, const int* folds,
    int precision, int n, int p, int q, const int* prefixes,
    int prefix_count, int scaling, int metric, int oversample, int power,
    unsigned long long seed, int store_predictions, double* predictions,
    int* status, double* metrics, double* q2, double* rmsd,
    double* observed_r2, char* error, size_t error_capacity);

/* replaces src/cuda_resident_api.h:27 -- PLS-SVD classification CV. */
FASTPLS_B200_API int fastpls_resident_plssvd_cv_classification(
    const void* predictors, const int* labels, const int* folds,
    int precision, int n, int p, int classes, const int* prefixes,
    int prefix_count, int scaling, int lda, int oversample, int power,
    unsigned long long seed, int store_predictions, int store_scores,
    int* predictions, void* scores, int* status, double* metrics,
    char* error, size_t error_capacity);

/* replaces src/cuda_resident_api.h:33 -- PLS-SVD regression CV. */
FASTPLS_B200_API int fastpls_resident_plssvd_cv_regression(
    const void* predictors, const void* responses, const int* folds,
    int precision, int n, int p, int q, const int* prefixes,
    int prefix_count, int scaling, int metric, int oversample, int power,
    unsigned long long seed, int store_predictions, double* predictions,
    int* status, double* metrics, double* q2, double* rmsd,
    double* observed_r2, char* error, size_t error_capacity);

/* replaces src/cuda_resident_api.h:40 -- fit a resident SIMPLS model
 * (responses y n x q, or one-based labels with q classes). */
FASTPLS_B200_API void* fastpls_resident_simpls_create(
    const void* x, const void* y, const int* labels, int precision, int n,
    int p, int q, int components, int scaling, int oversample, int power,
    int retain_scores, unsigned long long seed, char* error,
    size_t error_capacity);

/* replaces src/cuda_resident_api.h:44 -- fit a resident PLS-SVD model. */
FASTPLS_B200_API void* fastpls_resident_plssvd_create(
    const void* x, const void* y, const int* labels, int precision, int n,
    int p, int q, int components, int scaling, int oversample, int power,
    int retain_scores, unsigned long long seed, char* error,
    size_t error_capacity);

/* replaces src/cuda_resident_api.h:48 -- fit a resident OPLS model. */
FASTPLS_B200_API void* fastpls_resident_opls_create(
    const void* x, const void* y, const int* labels, int precision, int n,
    int p, int q, int components, int scaling, int oversample, int power,
    int retain_scores, unsigned long long seed, int north, char* error,
    size_t error_capacity);

/* replaces src/cuda_resident_api.h:52 -- fit a resident kernel PLS model
 * (kernel 2 = RBF, 3 = polynomial). */
FASTPLS_B200_API void* fastpls_resident_kernelpls_create(
    const void* x, const void* y, const int* labels, int precision, int n,
    int p, int q, int components, int scaling, int oversample, int power,
    int retain_scores, unsigned long long seed, int kernel, double gamma,
    int degree, double coef0, char* error, size_t error_capacity);

/* replaces src/cuda_resident_api.h:57 -- predictions (rows x q per prefix,
 * concatenated) for new rows; lda = 1 returns LDA discriminant scores. */
FASTPLS_B200_API int fastpls_resident_predict_path(void* model, const void* x, int rows,
                                  const int* prefixes, int prefix_count,
                                  int lda, void* predictions, char* error,
                                  size_t error_capacity);

/* replaces src/cuda_resident_api.h:60 -- release any resident handle. */
FASTPLS_B200_API void fastpls_resident_simpls_destroy(void* model);

/* replaces src/cuda_resident_api.h:61 -- copy a model field to the host:
 * 0 R (feature_p x a), 1 Q (q x a), 2 T (n x a), 3 mX (p), 4 vX (p),
 * 5 mY (q), 6 P loadings (feature_p x a), 7 variance SS (a + 1).
 * `elements` must equal the field size exactly. */
FASTPLS_B200_API int fastpls_resident_export(void* model, int field, void* out,
                            size_t elements, char* error,
                            size_t error_capacity);

/* replaces src/cuda_resident_api.h:63 -- top-k class labels per prefix
 * (rows x top per prefix, concatenated). */
FASTPLS_B200_API int fastpls_resident_classify_path(void* model, const void* x, int rows,
                                   const int* prefixes, int prefix_count,
                                   int lda, int top, int* labels, char* error,
                                   size_t error_capacity);

/* replaces src/cuda_resident_api.h:66 -- labels plus response scores. */
FASTPLS_B200_API int fastpls_resident_classify_response_path(
    void* model, const void* x, int rows, const int* prefixes,
    int prefix_count, int lda, int top, int* labels, void* predictions,
    char* error, size_t error_capacity);

/* replaces src/cuda_resident_api.h:69 -- per response: SSE, SS about the
 * training mean, SS about the observed mean (3 x q). */
FASTPLS_B200_API int fastpls_resident_response_sums(void* model, const void* x, const void* y,
                                   const int* labels, int rows, int prefix,
                                   void* out, char* error,
                                   size_t error_capacity);

/* replaces src/cuda_resident_api.h:71 -- latent scores (rows x prefix). */
FASTPLS_B200_API int fastpls_resident_project(void* model, const void* x, int rows,
                             int prefix, void* out, char* error,
                             size_t error_capacity);

/* replaces src/cuda_resident_api.h:73 -- solver controls in effect. */
FASTPLS_B200_API int fastpls_resident_controls(void* model, int* oversample, int* power,
                              int* block, int* block_limit,
                              int* implicit_operator,
                              int* predictor_crossprod_cache, char* error,
                              size_t error_capacity);

/* replaces src/cuda_resident_api.h:76 -- release training buffers
 * (optionally preparing LDA first). */
FASTPLS_B200_API int fastpls_resident_compact(void* model, int prepare_lda, char* error,
                             size_t error_capacity);

/* ---- additions (no counterpart in the reference ABI) ------------------- */

/* Number of CUDA devices visible (0 when none); backs has_cuda()
 * (fastPLS R/native_api.R:601, src/core_cuda_backend.cu:118-121). */
FASTPLS_B200_API int fastpls_b200_device_count(void);

/* Kernels launched by this library since load (benchmark accounting). */
FASTPLS_B200_API unsigned long long fastpls_b200_launch_count(void);

/* Stream on which the batched entry points run (a cudaStream_t; NULL =
 * each call creates a private stream). Lets a caller time the work with
 * events on its own stream. Calls stay synchronous. */
FASTPLS_B200_API void fastpls_b200_set_stream(void* stream);

/* Benchmark instrumentation: bracket every FP64 GEMM launch with CUDA
 * events on its stream; read returns (and resets) the summed device time,
 * the algorithmic FLOPs (2 M N K per launch) and the launch count. */
FASTPLS_B200_API void fastpls_b200_profile_gemm(int enable);
FASTPLS_B200_API void fastpls_b200_profile_gemm_read(
    double* milliseconds, double* flops, unsigned long long* launches);

/* Measured FP64 FMA throughput of the current device in TFLOP/s (a short
 * register-resident FMA-chain kernel timed with CUDA events). */
FASTPLS_B200_API int fastpls_b200_fp64_peak(double* tflops, char* error,
                                            size_t error_capacity);

/* Products with the shared Gram in the batched CV engine (no reference
 * counterpart; the reference forms them in FP64 BLAS): digits = 0 runs them
 * as FP64 DMMA GEMMs; digits = 1..7 splits every FP64 value into that many
 * int8 digits (power-of-two row scale, base 254, round to nearest) and runs
 * the digit-pair products on the int8 tensor cores (tcgen05.mma kind::i8)
 * with exact int32 accumulation. Default 6: product error below 2^-47 of
 * max|a_i| max|b_j| k. Process-wide; read back with _product_digits. */
FASTPLS_B200_API void fastpls_b200_set_product_digits(int digits);
FASTPLS_B200_API int fastpls_b200_product_digits(void);

/* Stream lanes of the batched CV engine (no reference counterpart): the
 * instances are split into `lanes` (1..4, default 3; each lane at least 32
 * instances) that run on their own CUDA streams, enqueued component by
 * component in turn so that one lane's memory-bound score and deflation
 * kernels overlap another lane's tensor-core products. Results do not
 * depend on it. Process-wide. */
FASTPLS_B200_API void fastpls_b200_set_batch_lanes(int lanes);
FASTPLS_B200_API int fastpls_b200_batch_lanes(void);

/* Argmax guard of the batched classification engine (no reference
 * counterpart). With int8 digit products, a held-out row whose top two class
 * scores differ by no more than `margin` times their magnitude marks its
 * (fold, permutation) instance, and every marked instance is refitted with
 * FP64 products, so predicted labels equal those of the FP64 path (the
 * reference's argmax, first index on ties:
 * inst/include/fastpls/core/classification.hpp:401-425). Default 1e-5;
 * 0 disables the guard. Process-wide. fastpls_b200_guard_refits returns the
 * number of instances the last batched classification call refitted. */
FASTPLS_B200_API void fastpls_b200_set_argmax_guard(double margin);
/* Group schedule of the batched engine (no reference counterpart). Every
 * buffer of a group lives in a per-device workspace kept between calls, and
 * a group's whole component sequence (all lanes, all components) is captured
 * once as a CUDA graph and replayed by later calls of the same shape. With
 * autotuning on (default), the first group of a new (n, p, q, instances,
 * components, digits) key times every schedule -- lanes 1..4 x tile width
 * 192 / 256, which give bit-identical results -- and keeps the fastest; the
 * decisions persist in the file named by the FASTPLS_B200_TUNE_FILE
 * environment variable when it is set. 0 selects the fixed rule
 * (fastpls_b200_set_batch_lanes lanes, width from the wave count).
 * fastpls_b200_batched_stats reports the last call: groups run, groups run by
 * graph replay, graphs captured, groups tuned, and the last schedule.
 * fastpls_b200_release_workspace frees the workspaces (the next call
 * rebuilds them). Process-wide. */
/* Device time of the calling thread's last resident fit (any of the four
 * _create functions), from CUDA events on the handle's stream: the copies of
 * the inputs to the device, and the fit proper (no reference counterpart;
 * benchmark instrumentation). Milliseconds. */
FASTPLS_B200_API void fastpls_b200_last_fit_times(double* copy_ms, double* fit_ms);
/* Single-fit SIMPLS component loop (no reference counterpart): 1 (default)
 * runs every component of a fit in one cooperative persistent launch where
 * it applies (one direction per component, 1..32 responses, 1..256
 * components); 0 runs the per-kernel loop. Results agree to rounding.
 * Process-wide. */
FASTPLS_B200_API void fastpls_b200_set_persistent(int enable);
/* Tests of the bounded waits (no reference counterpart). Every wait of the
 * tensor-core product and of the persistent fit has an iteration bound after
 * which the kernel records an error, finishes its own copies and MMAs, and
 * returns, so the call fails with an error and the device stays usable.
 * fastpls_b200_int8_wait_test(1, cycles): every tile of the int8 product
 * withholds its last pipeline stage, so the MMA issuer's wait for it runs
 * out after `cycles` clocks and the product reports a timed-out wait.
 * fastpls_b200_persistent_wait_test(1, cycles): one CTA of each persistent
 * fit leaves before its first barrier, so the others' barrier waits run out.
 * (0, 0) restores normal operation. Process-wide; for tests only. */
FASTPLS_B200_API void fastpls_b200_int8_wait_test(int skip_last_stage, long long wait_cycles);
FASTPLS_B200_API void fastpls_b200_persistent_wait_test(int absent_cta, long long wait_cycles);
FASTPLS_B200_API int fastpls_b200_persistent(void);
FASTPLS_B200_API void fastpls_b200_set_autotune(int enable);
FASTPLS_B200_API int fastpls_b200_autotune(void);
FASTPLS_B200_API void fastpls_b200_batched_stats(int* groups, int* graph_replays,
                                                 int* graph_captures, int* tuned, int* lanes,
                                                 int* tile_n);
FASTPLS_B200_API void fastpls_b200_release_workspace(void);
FASTPLS_B200_API double fastpls_b200_argmax_guard(void);
FASTPLS_B200_API int fastpls_b200_guard_refits(void);

/* Benchmark instrumentation of the int8 split products, as for
 * fastpls_b200_profile_gemm; the operation count is the int8 multiply-adds
 * issued (2 M N k per digit pair, M (M + 1) k for a symmetric product). */
FASTPLS_B200_API void fastpls_b200_profile_int8(int enable);
FASTPLS_B200_API void fastpls_b200_profile_int8_read(
    double* milliseconds, double* int8_ops, unsigned long long* launches);

/* c (m x n, column-major, ldc) = a^T b by the int8 split product above, for
 * a (k x m, lda) and b (k x n, ldb) column-major FP64 host arrays. With
 * symmetric = 1 (a == b, m == n) only the lower tiles are computed and
 * mirrored. tile_n: tile width in columns of c (128, 192 or 256; 0 = chosen
 * for the shape); pair: 1 = 256-row tiles on CTA pairs (tcgen05
 * cta_group::2; widths 192, 256; slower than single-CTA tiles on B200, kept
 * selectable), 0 or -1 = single-CTA 128-row tiles. The diagonals are
 * combined in FP64 in passes of four for
 * width 128 and of two otherwise. No reference counterpart (test and
 * integration entry for the split product). */
FASTPLS_B200_API int fastpls_b200_int8_crossprod(
    const double* a, int lda, const double* b, int ldb, int m, int n, int k,
    int digits, int symmetric, int tile_n, int pair, double* c, int ldc,
    char* error, size_t error_capacity);

/* Batched SIMPLS regression CV over the observed responses and
 * `permutation_count` row permutations of them (pls.single.cv /
 * pls.double.cv with perm.test; R/main.R:9419-9450, 12048-12080), all
 * sharing one device-resident X. permutations: permutation_count x n
 * zero-based source rows (row i of instance b uses responses[perm_b[i]]);
 * folds are shared by every instance. Outputs are
 * (permutation_count + 1) x prefix_count, row-major by instance, row 0 the
 * observed responses: the selected metric, Q2, RMSD and R2; status per fold.
 */
FASTPLS_B200_API int fastpls_b200_simpls_cv_permutation(
    const void* predictors, const void* responses, const int* folds,
    const int* permutations, int permutation_count, int precision, int n,
    int p, int q, const int* prefixes, int prefix_count, int scaling,
    int metric, double* metrics, double* q2, double* rmsd,
    double* observed_r2, int* status, char* error, size_t error_capacity);

/* Classification counterpart of fastpls_b200_simpls_cv_permutation (the
 * classification perm.test of pls.single.cv, CPU-only in the reference,
 * R/main.R:9419-9450): one-based labels (n, 1..classes, classes <= 32),
 * folds and zero-based permutations as there; responses are the one-hot
 * indicators of the permuted labels, each fold fit predicts the argmax over
 * the classes present in its training rows (the reference's argmax head,
 * src/cuda_resident_api.cuh:620-745; the LDA head is in
 * fastpls_b200_simpls_cv_permutation_classification_head). accuracy
 * ((B + 1) x prefix_count, row-major, B = permutation_count, row 0 the
 * observed labels): held-out accuracy per prefix. A training fold with one
 * class predicts that class for its held-out rows (status 4, as the
 * reference's classification CV). Where n_train p classes reaches 5e8 and the
 * path has 4 or more components, an instance takes min(64, components, p,
 * classes) directions from one decomposition per block, as the reference's
 * candidate blocks (src/cuda_resident_simpls.cuh:144-153). */
FASTPLS_B200_API int fastpls_b200_simpls_cv_permutation_classification(
    const void* predictors, const int* labels, const int* folds, const int* permutations,
    int permutation_count, int precision, int n, int p, int classes, const int* prefixes,
    int prefix_count, int scaling, double* accuracy, int* status, char* error,
    size_t error_capacity);

/* As above with predictors, responses, folds and permutations already in
 * device memory (prefixes and outputs stay on the host). */
/* The same with the classification head chosen: lda = 0 is the argmax of
 * the predicted class indicators (as fastpls_b200_simpls_cv_permutation_
 * classification), lda = 1 is LDA on the latent scores as the reference's
 * classification CV offers it (inst/include/fastpls/core/cross_validation.hpp:
 * 1567-1612, lda.hpp:86-223): per instance, after its last component,
 * class means and pooled covariance of its training scores over the classes
 * present in its training rows, the ridge retry grid, and the held-out
 * argmax of the discriminants. Up to 32 components with the LDA head. */
FASTPLS_B200_API int fastpls_b200_simpls_cv_permutation_classification_head(
    const void* predictors, const int* labels, const int* folds, const int* permutations,
    int permutation_count, int precision, int n, int p, int classes, const int* prefixes,
    int prefix_count, int scaling, int lda, double* accuracy, int* status, char* error,
    size_t error_capacity);
FASTPLS_B200_API int fastpls_b200_simpls_cv_permutation_device(
    const void* predictors, const void* responses, const int* folds,
    const int* permutations, int permutation_count, int precision, int n,
    int p, int q, const int* prefixes, int prefix_count, int scaling,
    int metric, double* metrics, double* q2, double* rmsd,
    double* observed_r2, int* status, char* error, size_t error_capacity);

/* Pearson correlations (fastcor(), R/main.R:12799; src/r_api.cpp:4054-4166):
 * units are the rows of a (byrow = 1) or its columns; each unit is centred
 * and scaled to unit norm in FP64 (NaN when it holds a non-finite value or
 * has zero spread). Without b: out = units_a x units_a matrix. With b:
 * units_a x units_b, or (diag = 1, matching unit counts) the units_a paired
 * correlations. a, b, out are host memory; out is FP64. */
FASTPLS_B200_API int fastpls_b200_fastcor(const void* a, const void* b, int precision,
                                          int rows_a, int cols_a, int rows_b,
                                          int cols_b, int byrow, int diag,
                                          double* out, char* error,
                                          size_t error_capacity);

/* Truncated SVD of x (n x p) on the device with the reference's audited
 * randomized SVD policy (fastsvd(backend = "cuda"); the reference's CUDA route
 * errors, R/main.R:7932-7943; policy: inst/include/fastpls/core/
 * audited_rsvd.hpp:298-414). FP64 randomized subspace iteration (Gaussian
 * sketch from `seed`, `power` power iterations, sketch width
 * min(k + 1 + oversample, min(n, p)) of at most 120 columns, since the small
 * eigenproblem is solved in one block's shared memory) at rank k + 1; the result is returned only when certified: the
 * triplet residual is <= 1e-2 of d_1 and no direction outside the first k
 * is larger than 1.01 d_k, or two consecutive attempts agree (subspace 1e-3,
 * singular values 1e-5, residual 1e-6). Attempts escalate oversample to 32
 * and 48 and power to 3 and 4 with new seeds, then up to four recoveries with
 * wider sketches; otherwise the call fails with the reference's message.
 * min(n, p) < 6 is solved exactly. Outputs (host, FP64): u n x k (may be
 * NULL), d k, v p x k (may be NULL); singular values in decreasing order,
 * each (u, v) pair sign-normalised. */
FASTPLS_B200_API int fastpls_b200_fastsvd(const void* x, int precision, int n, int p,
                                          int k, int oversample, int power,
                                          unsigned long long seed, double* u,
                                          double* d, double* v, char* error,
                                          size_t error_capacity);

/* fastpls_b200_fastsvd with the audit record (RsvdAudit,
 * audited_rsvd.hpp:19-30) in audit[10]: certified, deterministic fallback,
 * attempts, effective oversample, effective power, effective seed, subspace
 * error, singular value error, triplet residual, omitted direction ratio. */
FASTPLS_B200_API int fastpls_b200_fastsvd_audited(const void* x, int precision, int n,
                                                  int p, int k, int oversample, int power,
                                                  unsigned long long seed, double* u,
                                                  double* d, double* v, double* audit,
                                                  char* error, size_t error_capacity);

/* Variable importance in projection of a resident model (ViP(),
 * R/main.R:12769, vip_values in src/r_api.cpp:3973-4025) computed on the
 * device from R, Q and the training scores: for response r, component prefix
 * c and feature j, sqrt(fp * sum_{c' <= c} (R_jc'^2 / ||R_c'||^2) SS_c' /
 * sum_{c' <= c} SS_c') with SS_c = Q_rc^2 ||T_c||^2 (NaN while the
 * denominator is zero). out (FP64, size = q * a * fp doubles, fp = rows of
 * export field 0) holds per response an a x fp column-major block. */
FASTPLS_B200_API int fastpls_b200_resident_vip(void* model, double* out, size_t size,
                                               char* error, size_t error_capacity);

/* Rebuild a resident SIMPLS (method 3) or OPLS (method 4) model from its
 * exported fields, so a model saved by the host survives without refitting
 * (today the reference's handle is lost on session save/load, "refit the
 * model", src/cuda_resident_r.cpp:199-201). FP64 host arrays: weights =
 * export field 0 (p x a), response_loadings = field 1 (q x a), mean_x /
 * scale_x / mean_y = fields 3 / 4 / 5; scores = field 2 (n x a) and the
 * one-based training labels are optional and enable LDA for a
 * classification model. `precision` (16, 32, 64) is that of later prediction
 * rows and results, as for the _create functions. Returns a handle released
 * with fastpls_resident_simpls_destroy; fields 6 and 7 need the training
 * predictors and are not available on an imported model. */
FASTPLS_B200_API void* fastpls_b200_model_import(
    int method, int precision, int n, int p, int q, int components, int scaling,
    int classification, const double* weights, const double* response_loadings,
    const double* scores, const double* mean_x, const double* scale_x,
    const double* mean_y, const int* labels, char* error, size_t error_capacity);

/* ---- serving loop (no counterpart in the reference) ---------------------
 * A server owns `workers` threads, each driving resident handles on its own
 * CUDA stream, and admits queued requests by their HBM footprint against
 * `budget_bytes` (oldest admissible first, so requests arriving while others
 * run start as soon as memory and a worker free up). Fit requests return a
 * ticket that is also the model id; the model stays resident (training
 * predictors released) until fastpls_b200_server_release. Predictions queued
 * against one model are merged into one projection. Inputs are copied at
 * submission. Results are deterministic: identical alone or in a mix. */
FASTPLS_B200_API void* fastpls_b200_server_create(size_t budget_bytes, int workers,
                                                  char* error, size_t error_capacity);
FASTPLS_B200_API void fastpls_b200_server_destroy(void* server);
/* method: 1 PLS-SVD, 3 SIMPLS, 4 OPLS (north), 5 kernel PLS (kernel, gamma,
 * degree, coef0); y (n x q) or one-based labels (q classes). */
FASTPLS_B200_API int fastpls_b200_server_submit_fit(
    void* server, int method, const void* x, const void* y, const int* labels,
    int precision, int n, int p, int q, int components, int scaling, int north,
    int kernel, double gamma, int degree, double coef0,
    unsigned long long* ticket, char* error, size_t error_capacity);
FASTPLS_B200_API int fastpls_b200_server_submit_predict(
    void* server, unsigned long long model, const void* x, int rows, int p,
    int precision, const int* prefixes, int prefix_count, int lda,
    unsigned long long* ticket, char* error, size_t error_capacity);
/* Blocks (at most timeout_seconds) until the request completes; predictions
 * are written to out (rows x q per prefix, request precision). queue_ms and
 * service_ms: submission-to-start and start-to-finish times. */
FASTPLS_B200_API int fastpls_b200_server_wait(
    void* server, unsigned long long ticket, double timeout_seconds, void* out,
    size_t capacity_bytes, double* queue_ms, double* service_ms, char* error,
    size_t error_capacity);
FASTPLS_B200_API int fastpls_b200_server_release(void* server, unsigned long long model,
                                                 char* error, size_t error_capacity);
FASTPLS_B200_API int fastpls_b200_server_stats(void* server, size_t* bytes_in_use,
                                               size_t* queued, size_t* resident_models);
/* Fit batching: queued SIMPLS fits of one storage precision that each run as
 * one persistent launch (one direction per component, 1..32 responses) are
 * taken together, up to 32 fits or the launch's co-resident CTAs, and run
 * their component loops in ONE cooperative launch; each fit keeps the CTA
 * count and chunking it has alone, so its result is bit-identical alone or
 * batched. launches: persistent launches that ran batches; fits: the fits
 * they carried. */
FASTPLS_B200_API int fastpls_b200_server_batch_stats(void* server, size_t* launches,
                                                     size_t* fits);
/* Borrow mode (off by default): with on != 0, requests submitted afterwards
 * read their x, y and labels in place instead of copying them at
 * submission; the caller keeps those buffers valid and unchanged until
 * fastpls_b200_server_wait has returned for the request (or the server is
 * destroyed). Saves a host copy of every input (the Python Server holds
 * references to the arrays until then). */
FASTPLS_B200_API int fastpls_b200_server_set_borrow(void* server, int on);

/* out (p x nb, FP64) = X^T V for device-resident X (n x p, leading
 * dimension ldx, FP32 or FP64 by `precision`), V (n x nb FP64, ldv) and out
 * (ldo), without any memory allocation by the library: for callers whose
 * host owns all device memory (a fixed memory plan, admission by memory
 * footprint) or that must not stall on the allocator. No counterpart in the
 * reference ABI. Partial sums live in one file-scope device array of
 * 2097152 doubles (16 MiB) that every GPU loading the library keeps until
 * exit; requests with p * nb above that size, or nb above 32, are rejected
 * with an error; any row count is accepted (rows are grouped into at most
 * 65535 chunks). The array's address is looked up on the first call made on
 * each device, so make that first call before any stream capture; the address
 * is kept for the process, so do not call again after cudaDeviceReset. All
 * calls share the array: calls that overlap on the GPU race and must be
 * serialised by the caller. Runs on `stream` (a cudaStream_t, NULL = default
 * stream) and waits for that stream before returning. */
FASTPLS_B200_API int fastpls_b200_crossprod_noalloc(
    const void* x, int precision, int n, int p, long ldx, const double* v,
    long ldv, int nb, double* out, long ldo, void* stream, char* error,
    size_t error_capacity);

#ifdef __cplusplus
}
#endif
#endif /* FASTPLS_B200_H */
