/*
 * hml_b200.h -- C ABI of the B200 (sm_100a) skinny SGEMM/SGEMV library.
 *
 * Every entry point is extern "C", takes plain pointers and sizes, and
 * returns an hml_status.  Device-pointer entry points are stream ordered
 * (the stream is passed as an opaque cudaStream_t, NULL = legacy default
 * stream) and return as soon as the work is enqueued.  Nothing here calls
 * exit(): errors come back as status codes.
 *
 * The reference's public C++ entry points (hmlSgemm, hmlSgemmBasic,
 * hmlSgemmKernelConfig, hmlSgemv, hmlSgemvBasic, hmlSgemvKernelConfig) are
 * exported too, with their original C++ linkage, from hml_sgemm.h and
 * hml_sgemv.h in this directory; they are thin shims over this ABI.
 *
 * Conventions
 *   - BLAS semantics: C = alpha * op(A) * op(B) + beta * C, op(X) = X or X^T,
 *     with column-major (HML_COL_MAJOR) or row-major (HML_ROW_MAJOR) storage
 *     and leading dimensions.  beta == 0 means C is not read (NaN in C does
 *     not propagate), unlike the reference kernels, which always read C
 *     (include/hml_sgemm_kernel_template.h:187 in the reference).
 *   - All arithmetic on the hot path is FP32 in and FP32 out.  The split-BF16
 *     algorithms use BF16 tensor-core products of FP32 operands split on the
 *     fly into 2 or 3 BF16 terms, accumulated in FP32.
 */
#ifndef HML_B200_H_INCLUDED_
#define HML_B200_H_INCLUDED_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum hml_status {
  HML_STATUS_SUCCESS = 0,
  HML_STATUS_INVALID_VALUE = 1,  /* bad size, stride, pointer or enum     */
  HML_STATUS_NOT_SUPPORTED = 2,  /* valid request this build cannot serve */
  HML_STATUS_CUDA_ERROR = 3,     /* a CUDA runtime call failed            */
  HML_STATUS_ALLOC_FAILED = 4,   /* device or pinned allocation failed    */
  HML_STATUS_CONFIG_ERROR = 5,   /* malformed or out-of-range tuning data */
  HML_STATUS_TIMEOUT = 6,        /* a bounded device-side wait expired    */
  HML_STATUS_IO_ERROR = 7        /* file could not be opened or written   */
} hml_status;

typedef enum hml_order { HML_COL_MAJOR = 0, HML_ROW_MAJOR = 1 } hml_order;
typedef enum hml_op { HML_OP_N = 0, HML_OP_T = 1 } hml_op;

/* Algorithm families of the SGEMM path. */
typedef enum hml_algo {
  HML_ALGO_AUTO = 0,   /* tuned table, then predictor, then default        */
  HML_ALGO_SIMT = 1,   /* plain FP32 FMA on CUDA cores                     */
  HML_ALGO_BF16X3 = 2, /* tcgen05: hi/lo BF16 split, 3 products (hh,hl,lh) */
  HML_ALGO_BF16X6 = 3, /* tcgen05: hi/mid/lo split, 6 products            */
  HML_ALGO_TF32X3 = 4, /* tcgen05 kind::tf32: hi/lo TF32 split, 3 products
                          (FP32-level accuracy like BF16X6; explicit
                          configurations only, 128-row tiles)           */
  HML_ALGO_FP16X3 = 5  /* tcgen05 kind::f16 with FP16 operands: each row of
                          a 32-deep block of A and each column of B scaled
                          by a power of two into FP16's range, hi/lo FP16
                          split (22 significant bits), 3 products;
                          FP32-level accuracy; 128-row tiles.  Range: the
                          running sums of a tile hold C scaled by a power
                          of two <= 1, so a result overflows only where
                          |alpha| sum_k |A(m,k)| |B(k,n)| itself exceeds
                          the FP32 range */
} hml_algo;

/* Accuracy policy of hml_sgemm_ex's automatic choice. */
typedef enum hml_math_mode {
  HML_MATH_FP32 = 0, /* default: FP32 SIMT or BF16X6 (FP32-level accuracy)   */
  HML_MATH_FAST = 1  /* BF16X3 allowed (about 2**-17 relative per product)  */
} hml_math_mode;

/* One point of the SGEMM configuration space. */
typedef struct hml_sgemm_config {
  int32_t algo;    /* hml_algo                                            */
  int32_t tile_m;  /* rows of C per CTA (the long dimension): 128 for
                      the tensor-core forms, 128 or 256 for SIMT         */
  int32_t tile_n;  /* columns of C per CTA (the skinny dimension)         */
  int32_t split_k; /* CTAs of one thread-block cluster sharing a C tile,
                      each taking a slice of K; partial tiles are summed
                      in rank order through distributed shared memory     */
  int32_t stages;  /* shared-memory pipeline depth                        */
  int32_t variant; /* per-algorithm micro-tile selector (SIMT: 0-8 the
                      tiled kernel's micro-tiles, 9-10 the stream-K
                      kernel for N <= 4 / 8 with contiguous columns of A;
                      split-BF16/TF32: the tile shape)                  */
} hml_sgemm_config;

const char *hml_status_string(hml_status status);
const char *hml_version(void);

/* ---------------------------------------------------------------- SGEMM */

/* C = alpha * op(A) * op(B) + beta * C on device pointers.  op(A) is M x K,
 * op(B) is K x N, C is M x N.  The configuration comes from the tuned table
 * (hml_tune_load / hml_autotune_sgemm; without either, the first selection
 * loads the B200 table shipped as data/tuned_b200.txt beside the library,
 * HML_TUNED=<file> names another, HML_TUNED=none disables it; an entry also
 * serves shapes within about 2x of it in every dimension), else the learned
 * predictor, else the built-in heuristic.  The predictor is the one loaded by
 * hml_predictor_load
 * or trained by hml_predictor_train; without either, the first selection
 * loads the network shipped as data/predictor_b200.txt beside the library
 * (environment: HML_PREDICTOR=<file> names another, HML_PREDICTOR=none
 * disables it).  When the chosen tensor-core configuration has split_k = 1
 * and its grid of row tiles would end in a wave that leaves at least half of
 * the SMs idle, the rows of that last wave run as a second grid with K split
 * across the idle SMs (those rows then carry split-K rounding, within the
 * same error bounds; hml_sgemm_ex_config runs a configuration exactly as
 * given).  Replaces the launch half of
 * hmlSgemm (src/hml_sgemm.cu:120-211 in the reference), generalised to
 * both storage orders, transposes and leading dimensions. */
hml_status hml_sgemm_ex(hml_order order, hml_op transA, hml_op transB, int M,
                        int N, int K, float alpha, const float *A, int lda,
                        const float *B, int ldb, float beta, float *C, int ldc,
                        void *stream);

/* Same, with an explicit configuration (algo must not be HML_ALGO_AUTO).
 * Replaces launching one chosen kernel of the reference's repository
 * (hmlSgemmKernelSelect + launch, src/hml_sgemm_kernel.cu:189-237). */
hml_status hml_sgemm_ex_config(hml_order order, hml_op transA, hml_op transB,
                               int M, int N, int K, float alpha, const float *A,
                               int lda, const float *B, int ldb, float beta,
                               float *C, int ldc,
                               const hml_sgemm_config *config, void *stream);

/* The configuration hml_sgemm_ex would use for this problem. */
hml_status hml_sgemm_select(hml_order order, hml_op transA, hml_op transB,
                            int M, int N, int K, hml_sgemm_config *config);

/* Split-BF16 SGEMM that allocates nothing.  No counterpart in the
 * reference: it exists for callers that must not allocate device memory
 * during a call -- processes that reserve their whole HBM budget up front for
 * their own pool, latency-critical paths where cudaMalloc's implicit device
 * synchronisation is not acceptable, and hosts that forbid allocation after
 * start-up.  hml_sgemm_ex_config with the same configuration computes the
 * same result, bit for bit, but keeps the BF16 planes of B in a workspace it
 * grows with cudaMalloc; this variant keeps them in a fixed 4 MiB array
 * compiled into the library (every GPU that loads the library holds it until
 * exit).
 *   - config->algo must be HML_ALGO_BF16X3 or HML_ALGO_BF16X6.
 *   - Limit: the library computes a problem whose N exceeds its M as the
 *     transposed problem (C^T = B^T A^T), so the planes are cut from the
 *     shorter of M and N.  With S = min(M, N):
 *     planes x ceil(S / tile_n) * tile_n x ceil(K / 64) * 64 x 2 bytes
 *     must not exceed 4 MiB (planes = 2 for BF16X3, 3 for BF16X6); larger
 *     problems are rejected with HML_STATUS_INVALID_VALUE and a message in
 *     hml_last_error().
 *   - The first call on a device looks up the addresses of the array and of
 *     the entry point's error word (cudaGetSymbolAddress) with that device
 *     current; make that first call before any stream capture.
 *   - Every call on a device shares the one array, which keeps the last
 *     call's contents: calls that overlap on the GPU (on different streams,
 *     or from different host threads) race and corrupt each other's planes,
 *     so serialise them (one stream, or events between streams).  Nothing
 *     in the array needs to start at zero; each call rewrites the part it
 *     uses.
 *   - A bounded wait that expires ends the kernel and records its code in an
 *     error word that is also a file-scope device variable;
 *     hml_device_error() reads and clears it (without allocating). */
hml_status hml_sgemm_ex_config_noalloc(hml_order order, hml_op transA,
                                       hml_op transB, int M, int N, int K,
                                       float alpha, const float *A, int lda,
                                       const float *B, int ldb, float beta,
                                       float *C, int ldc,
                                       const hml_sgemm_config *config,
                                       void *stream);

/* The heuristic configuration of one algorithm family for this problem
 * (HML_ALGO_AUTO: same as hml_sgemm_select).  Returns the status of
 * hml_sgemm_config_check for dense leading dimensions. */
hml_status hml_sgemm_select_algo(hml_order order, hml_op transA, hml_op transB,
                                 int M, int N, int K, int algo,
                                 hml_sgemm_config *config);

/* Whether a configuration can run this problem (status only, no launch). */
hml_status hml_sgemm_config_check(hml_order order, hml_op transA, hml_op transB,
                                  int M, int N, int K, int lda, int ldb, int ldc,
                                  const hml_sgemm_config *config);

/* Enumeration of the configuration space the autotuner searches.  Replaces
 * the reference's kernel repository tables (include/hml_sgemm_kernel.h:62-66). */
int hml_sgemm_num_configs(void);
hml_status hml_sgemm_get_config(int index, hml_sgemm_config *config);
int hml_sgemm_config_index(const hml_sgemm_config *config);

/* --------------------------------------------------------- autotuning */

/* One measured configuration. */
typedef struct hml_tune_entry {
  hml_sgemm_config config;
  float time_us;  /* median device time of one call, -1 when not timed      */
  int32_t status; /* hml_status of the trial (non-zero: refused or failed) */
} hml_tune_entry;

/* Measures every configuration of the space (restricted to the algorithm
 * families in the bitmask `families`, bit = 1 << hml_algo; 0 = all) on this
 * problem shape with leading dimensions rounded up to a multiple of 4 floats
 * (16 bytes, addressable by every kernel family) and uniform[-1,1] operands:
 * one warm-up call, then `reps` calls timed with CUDA events on the stream,
 * L2 flushed before each when the operands fit in it, median kept; each
 * configuration runs as hml_sgemm_ex would run it once selected.  A
 * configuration that cannot run or fails is recorded with its status and
 * skipped.  Writes up to max_entries results (*n_entries = count) and
 * records the fastest configuration the math mode allows in the tuned table
 * that hml_sgemm_ex consults first.  Replaces the reference's online tuner
 * (src/hml_sgemm_kernel.cu:356-555). */
hml_status hml_autotune_sgemm(hml_order order, hml_op transA, hml_op transB,
                              int M, int N, int K, uint32_t families, int reps,
                              hml_tune_entry *entries, int max_entries,
                              int *n_entries, void *stream);

/* The tuned table on disk ("#HML-B200 tuning v2"; the reference's v1
 * .cfg grammar is read by hml_cfg_v1_load), replacing the reference's
 * hmlSgemmKernelConfigPrint / ReadFile (src/hml_sgemm_kernel.cu:557-602). */
hml_status hml_tune_save(const char *path);
hml_status hml_tune_load(const char *path, int *records);
hml_status hml_tune_clear(void);
int hml_tune_size(void);

/* Selects the accuracy policy (hml_math_mode) of automatic selection. */
hml_status hml_set_math_mode(int mode);

/* ---------------------------------------------------- learned predictor */

/* A small MLP (5 -> 64 -> 64 -> one score per configuration) that predicts
 * the fastest configuration of an unseen shape from autotuner measurements,
 * replacing the reference's static per-GPU tables
 * (src/hml_sgemm_kernel.cu:189-237).  Features of the canonical (long-M)
 * problem: log2 M / 16, log2 N / 8, log2 K / 14, A K-contiguous,
 * B K-contiguous.  Scores regress y = min(log(t / t_best), target_clip) per
 * measured configuration (masked mean squared error); the prediction is the
 * lowest score among the configurations that can run the problem and that
 * the math mode allows.  Training and inference run on the GPU in this
 * library's own kernels. */
typedef struct hml_predictor_options {
  int32_t epochs;      /* passes over the training shapes                   */
  int32_t batch;       /* shapes per AdamW step                             */
  float lr;            /* peak learning rate (cosine decay to 5 %)          */
  float weight_decay;  /* AdamW decoupled weight decay                      */
  float target_clip;   /* cap on log(t / t_best)                            */
  uint64_t seed;       /* initialisation and shuffling (SplitMix64)         */
} hml_predictor_options;

/* Trains on n shapes (shapes: n x 5 int32 rows M, N, K, transA, transB in
 * `order` with 16-byte-rounded leading dimensions, the autotuner's layout)
 * and their measured times (times_us: n x n_configs, <= 0 where a
 * configuration was not measured; column j belongs to configuration j of
 * hml_sgemm_get_config, the n_configs of the space).  The
 * trained network becomes the active predictor; loss_history (may be NULL)
 * receives the mean training loss of each epoch. */
hml_status hml_predictor_train(hml_order order, const int32_t *shapes,
                               const float *times_us, int n,
                               const hml_sgemm_config *configs, int n_configs,
                               const hml_predictor_options *options,
                               float *loss_history);

/* Loss and gradient of the network with parameters `params` (layout W1[64][5]
 * b1[64] W2[64][64] b2[64] W3[C][64] b3[C]) on n rows of features (n x 5),
 * targets and weights (n x C), computed by the training kernels.  Host
 * arrays; synchronous.  loss = sum w (s - y)^2 / sum w. */
hml_status hml_predictor_loss_grad(const float *params, int n_configs,
                                   const float *features, const float *targets,
                                   const float *weights, int n, float *grad,
                                   float *loss);

/* The active predictor's choice (an index into its configuration list, -1
 * when none can run) for n shapes in one inference launch. */
hml_status hml_predictor_predict_batch(hml_order order, const int32_t *shapes,
                                       int n, int32_t *config_index);

hml_status hml_predictor_save(const char *path);
hml_status hml_predictor_load(const char *path);
hml_status hml_predictor_clear(void);
/* Number of configurations the active predictor scores (0: none loaded). */
int hml_predictor_outputs(void);
/* Copies the active predictor's parameters (count = their number). */
hml_status hml_predictor_params(float *out, size_t capacity, size_t *count);
/* The feature vector of a shape (same layout convention as training). */
hml_status hml_predictor_features(hml_order order, int transA, int transB,
                                  int M, int N, int K, float features[5]);

/* ------------------------------------------------------------- batched */

/* One problem of a batch: C = alpha * op(A) * op(B) + beta * C on device
 * pointers, stored in the batch's hml_order (same argument meaning as
 * hml_sgemm_ex).  The C matrices of one batch must not overlap. */
typedef struct hml_gemm_desc {
  int32_t transA, transB; /* hml_op */
  int32_t M, N, K;
  int32_t lda, ldb, ldc;
  float alpha, beta;
  const float *A;
  const float *B;
  float *C;
} hml_gemm_desc;

typedef struct hml_batch_plan_s *hml_batch_plan;

/* Builds a plan for a batch: validates every problem, cuts all of them into
 * tile work items ordered longest first, and uploads the items to the
 * device.  Problems with N > 8 (in the long-M form) whose A TMA can address
 * (16-byte aligned base, leading dimension a multiple of 4 floats) run as
 * split-BF16 (BF16X6) tensor-core tiles, the others as FP32 SIMT tiles.  The reference has no batched form: its callers loop over
 * hmlSgemm, one launch and one synchronisation per problem
 * (src/hml_sgemm.cu:120-211).  The descriptors are copied; the matrices they
 * point to are read when the plan runs. */
hml_status hml_batch_plan_create(hml_order order, const hml_gemm_desc *descs,
                                 int count, hml_batch_plan *plan);

/* Runs every problem of the plan: the SIMT tiles in ONE persistent kernel
 * launch whose CTAs take tiles from a device work queue, the tensor-core
 * tiles in one B-splitting launch and one persistent launch per tile width
 * (32, 64, 128 columns) whose CTAs work through host-balanced item lists.
 * Stream ordered; capturable.  One plan runs on one stream at a time. */
hml_status hml_batch_plan_run(hml_batch_plan plan, void *stream);

/* Same, through a CUDA graph holding the launch: the first call captures
 * it (not while the calling thread is capturing a stream in global mode),
 * every call launches the graph on `stream`. */
hml_status hml_batch_plan_graph_launch(hml_batch_plan plan, void *stream);

/* Work items, CTAs of the launch, useful FLOPs (2MNK summed) and
 * algorithmic bytes (A, B read once, C written once, read too when
 * beta != 0). Any output pointer may be NULL. */
hml_status hml_batch_plan_info(hml_batch_plan plan, int *tiles, int *ctas,
                               double *flops, double *bytes);
hml_status hml_batch_plan_destroy(hml_batch_plan plan);

/* One-shot batch: plan, its launches and release, all stream ordered. */
hml_status hml_sgemm_batched(hml_order order, const hml_gemm_desc *descs,
                             int count, void *stream);

/* The configuration under which a batch runs this problem (an FP32 SIMT tile
 * or BF16X6 with the tile width class); hml_sgemm_ex_config with it computes
 * the same bits.  No counterpart in the reference, which has no batches. */
hml_status hml_batch_problem_config(hml_order order, const hml_gemm_desc *desc,
                                    hml_sgemm_config *config);

/* ---------------------------------------------------------------- SGEMV */

/* y = alpha * op(A) * x + beta * y on device pointers; A is M x N in storage,
 * op(A) is A (length(y) = M) or A^T (length(y) = N).  Replaces hmlSgemv
 * (src/hml_sgemv.cu:125-213), which is the row-major, non-transposed case. */
hml_status hml_sgemv_ex(hml_order order, hml_op trans, int M, int N,
                        float alpha, const float *A, int lda, const float *x,
                        float beta, float *y, void *stream);

/* Same, forcing a kernel variant: for A with contiguous rows the number of
 * threads that share one row (4, 8, ..., 256; few long rows are also split
 * over several CTAs, as the heuristic decides); for A with contiguous
 * columns the number of CTAs that split the columns of one row tile (256
 * rows, 128 when the result has at most 128 entries), 1..256.  0 = the
 * heuristic.  Replaces launching one chosen SGEMV kernel of the reference's
 * repository (hmlSgemvKernelSelect + launch, src/hml_sgemv_kernel.cu:315-355). */
hml_status hml_sgemv_ex_variant(hml_order order, hml_op trans, int M, int N,
                                float alpha, const float *A, int lda,
                                const float *x, float beta, float *y,
                                int variant, void *stream);

/* The variant hml_sgemv_ex runs this problem with: the tuned table's
 * (*variant > 0), or 0 when the heuristic decides.  Host only, no launch. */
hml_status hml_sgemv_select(hml_order order, hml_op trans, int M, int N,
                            int lda, int *variant);

/* One measured SGEMV variant. */
typedef struct hml_sgemv_tune_entry {
  int32_t variant; /* as in hml_sgemv_ex_variant                          */
  float time_us;   /* median device time of one call, -1 when not timed   */
  int32_t status;  /* hml_status of the trial                             */
} hml_sgemv_tune_entry;

/* Measures every variant of the SGEMV kernel that serves this layout (7
 * thread-per-row widths, or 25 column splits from 1 to 256) on an M x N
 * problem with the leading dimension rounded up to a multiple of 4 floats
 * and uniform[-1,1] operands: one warm-up call, then `reps` calls timed with CUDA events on
 * the stream, L2 flushed before each when A fits in it, median kept.  Writes
 * up to max_entries results (*n_entries = count) and records the fastest
 * variant in the tuned table (saved and loaded with hml_tune_save /
 * hml_tune_load as "v" records) that hml_sgemv_ex, the SGEMM N = 1 route and
 * hmlSgemv consult first.  Replaces the reference's online SGEMV tuner
 * (hmlSgemvKernelConfigOnline, src/hml_sgemv_kernel.cu:391-633). */
hml_status hml_autotune_sgemv(hml_order order, hml_op trans, int M, int N,
                              int reps, hml_sgemv_tune_entry *entries,
                              int max_entries, int *n_entries, void *stream);

/* ------------------------------------------------- host-pointer path */

/* Row-major C = alpha*A*B + beta*C on HOST pointers (A M x K, B K x N),
 * synchronous; basic != 0 forces the heuristic configuration.  The status
 * returning form of hmlSgemm / hmlSgemmBasic (src/hml_sgemm.cu:39-211). */
hml_status hml_host_sgemm(int basic, float *C, const float *A, const float *B,
                          int M, int N, int K, float alpha, float beta);

/* Row-major y = alpha*A*x + beta*y on HOST pointers, synchronous.  The
 * status-returning form of hmlSgemv / hmlSgemvBasic (src/hml_sgemv.cu). */
hml_status hml_host_sgemv(int basic, float *y, const float *A, const float *x,
                          int M, int N, float alpha, float beta);

/* ------------------------------------------------------ tuning files */

/* kind 0 = SGEMM, 1 = SGEMV.  Reads a tuning file the way
 * hmlSgemmKernelConfig / hmlSgemvKernelConfig do (src/hml_sgemm.cu:213-226,
 * src/hml_sgemv.cu:215-228): this library's measured table, or a reference
 * v1 file.  NULL keeps the current selection. */
hml_status hml_config_file(int kind, const char *path);

/* Reads a reference v1 file (src/hml_sgemm_kernel.cu:573-602,
 * src/hml_sgemv_kernel.cu:650-679), range-checking every rule; *rules gets
 * the number of rules read.  A bad line rejects the file. */
hml_status hml_cfg_v1_load(int kind, const char *path, int *rules);

/* The v1 rule the reference would apply (its keying: K' = min(K, 96),
 * colStops = ceil(min(N, 96) / 16); SGEMV: N <= 1024 ? N : 0).
 * HML_STATUS_CONFIG_ERROR when no valid rule applies. */
hml_status hml_cfg_v1_sgemm_rule(int K, int N, int *type, int *row_stops);
hml_status hml_cfg_v1_sgemv_rule(int N, int *type, int *block_stops,
                                 int *row_stops);
void hml_cfg_v1_clear(void);

/* Writes the loaded v1 rules of `kind` back in the reference's grammar and
 * rule order (hmlSgemmKernelConfigPrint src/hml_sgemm_kernel.cu:557-568,
 * hmlSgemvKernelConfigPrint src/hml_sgemv_kernel.cu:634-645): '#' comment
 * lines, then one rule per line for every entry whose rowStops is positive.
 * HML_STATUS_CONFIG_ERROR when no v1 file of that kind is loaded. */
hml_status hml_cfg_v1_save(int kind, const char *path);

/* The configuration hmlSgemm runs a row-major M x N x K problem with when a
 * loaded v1 SGEMM rule covers it: the rule's tile (16*rowStops rows,
 * 16*colStops columns; the basic kernel's 96 x 96) mapped onto the nearest
 * tiled SIMT shape.  The reference's selection this stands in for is
 * hmlSgemmKernelSelect (src/hml_sgemm_kernel.cu:189-237).
 * HML_STATUS_CONFIG_ERROR when no rule applies (hmlSgemm then uses the
 * library's own selection). */
hml_status hml_sgemm_v1_config(int M, int N, int K, hml_sgemm_config *config);

/* --------------------------------------------------- k-means assignment */

/* assignments[p] = argmin_k sum_d (points[p][d] - centroids[k][d])^2, the
 * assignment step of HiperML's k-means (hmlKmeansAssignCtrdSmem,
 * include/hml_kmeans_kernel_template.h:19-90): device pointers, points
 * row-major [num_points][dims], centroids row-major [num_clusters][dims],
 * assignments uint32 [num_points].  Computed as ||c||^2 - 2 x.c, the dot
 * products a skinny GEMM, and made exact: every point gets the index the
 * reference kernel gives (its FP32 sums, the first k on ties).  Uses the
 * stream's second workspace.  Stream ordered. */
hml_status hml_kmeans_assign(const float *points, int num_points, int dims,
                             const float *centroids, int num_clusters,
                             uint32_t *assignments, void *stream);

/* The same with the form chosen: method 0 = the library's choice (the
 * tensor-core form where it applies, else the tiled form up to 256
 * dimensions, else the SGEMM form), 1 = the tiled form (a register-tiled FP32
 * SIMT GEMM with the argmin in its epilogue), 2 = the SGEMM form (the
 * products through HBM, num_points x num_clusters floats of workspace, then a
 * pick kernel; HML_STATUS_NOT_SUPPORTED above 51200 clusters), 3 = the
 * tensor-core form (TF32X3 products on tcgen05 into TMEM, the argmin read
 * from the accumulator; HML_STATUS_NOT_SUPPORTED unless dims is a multiple
 * of 4 in 4..64, points is 16-byte aligned and num_clusters <= 256).  When
 * exact_count (a device counter) is not NULL, the number of points whose
 * candidates had to be compared with the reference's own arithmetic is added
 * to it. */
hml_status hml_kmeans_assign_ex(const float *points, int num_points, int dims,
                                const float *centroids, int num_clusters,
                                uint32_t *assignments, int method,
                                unsigned *exact_count, void *stream);

/* ------------------------------------------------------------ utilities */

/* Text of the last CUDA error seen by this thread inside the library. */
const char *hml_last_error(void);

/* Fill n floats with the counter-based SplitMix64 generator (dist 0 =
 * uniform[-1,1), 1 = normal(0,1), 2 = log-uniform magnitude 1e-3..1e3 with
 * random sign).  Identical stream to hiperml_b200.datagen. */
hml_status hml_fill_random(float *out, size_t n, uint64_t seed,
                           uint64_t stream_id, int dist, void *stream);

/* FP64 check of an SGEMM result, on the GPU: recomputes alpha*op(A)*op(B) +
 * beta*C0 in FP64 (C0 = the C that was passed in, given here as C0) and
 * compares it with C.  err[0] = max|dC| / max|C64| (normwise),
 * err[1] = ||dC||_2 / ||C64||_2 (RMS), err[2] = max_ij |dC_ij| /
 * (|alpha| |op(A)||op(B)| + |beta||C0|)_ij (componentwise), err[3] = max|C64|.
 * FP64 is used only here and never on the hot path. */
hml_status hml_sgemm_error_fp64(hml_order order, hml_op transA, hml_op transB,
                                int M, int N, int K, float alpha,
                                const float *A, int lda, const float *B,
                                int ldb, float beta, const float *C0,
                                const float *C, int ldc, double err[4],
                                void *stream);

/* Device-side error word of bounded waits: 0 when clear.  Reading clears. */
hml_status hml_device_error(int *code);

/* Failure-path check: launches a kernel whose one waiting thread waits on a
 * barrier that nothing completes.  The bounded wait every kernel of this
 * library uses gives up after its limit (2 s), writes code 1 (a tile that
 * never landed) to the device error word and returns, so the device stays
 * usable; hml_device_error then reports the code.  No counterpart in the
 * reference, whose kernels have no waits. */
hml_status hml_check_wait_limit(void *stream);

/* Number of kernels the library has launched since it was loaded. */
uint64_t hml_launch_count(void);

/* Frees the library's cached device workspaces and staging buffers. */
hml_status hml_release_resources(void);

#ifdef __cplusplus
}
#endif

#endif /* HML_B200_H_INCLUDED_ */
