/*
 * exageostat_b200 -- C ABI of the B200 (sm_100a) exact Matern MLE library.
 *
 * Drop-in for the exact (exageostat_exact) maximum-likelihood path of
 * ExaGeoStat 1.2: the same entry points, the same MLE_data / location /
 * output structures (field for field, so drivers that poke fields keep
 * working) and the same argument meaning.  Paths in the citations are inside
 * the reference project.  Differences from the reference are listed per
 * function; the main one is that no function calls exit(): failures are
 * reported through return values, data fields and exageostat_last_error().
 * Beyond the likelihood path: kriging, the Fisher information, MLOE / MMOM,
 * the flat-file readers, great-circle distance (dm = "gc") and the
 * bivariate parsimonious Matern kernel.
 *
 * Everything runs on one CUDA device (the current device at
 * exageostat_init).  All pointers in these signatures are HOST pointers.
 *
 * Threads: one MLE_data (or batch handle) is used by one host thread at a
 * time.  Calls for different MLE_data may come from different threads; they
 * share the library's CUDA stream and so run one after the other on the
 * device.  The first exageostat_b200_batch_loglik of a batch records its
 * launch sequence into a CUDA graph on that stream: make no other library
 * call from another thread while it runs.
 */
#ifndef EXAGEOSTAT_B200_H
#define EXAGEOSTAT_B200_H

#include <stddef.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- data structures: layout-identical to misc/include/MLE_misc.h:111-328 ---- */

/* misc/include/MLE_misc.h:111-115 */
typedef struct {
    double *x; /* first coordinate (x, or latitude for dm = "gc") */
    double *y; /* second coordinate */
    double *z; /* third coordinate; NULL for 2-D locations (the only case handled here) */
} location;

/* misc/include/MLE_misc.h:130-178; the library writes final_loglik and
 * estimated_theta (when allocated) like the reference. */
typedef struct {
    int problem_size;
    char *computation;
    char *kernel;
    char *ds_type;
    char *precision;
    int z_sample;
    int dense_ts;
    int lr_ts;
    int lr_acc;
    int lr_maxrank;
    int ncores;
    int ngpus;
    int p;
    int q;
    int num_params;
    double *initial_theta;
    double *starting_theta;
    double *estimated_theta;
    double final_loglik;
    double time_per_iteration;
    double cholesky_per_iter;
    double flops_per_iteration;
    double generation_per_iter;
    double solve_per_iter;
    double total_mle_time;
    double avg_exec_time_gen_stage;
    double avg_flops_gen_stage;
    double mse_pred1;
    double mse_pred2;
    double mse_pred3;
    double mse_pred;
    double trace_pred_sum;
    double trace_pred_mean;
    double total_pred_time;
    double total_pred_flops;
    double mloe;
    double mmom;
    char *mloe_exec;
    double total_mloe_mmom_time;
    double matrix_gen_mloe_mmom_time;
    double cho_fact_mloe_mmom_time;
    double loop_mloe_mmom_time;
    double total_mloe_mmom_flops;
    double fisher_00;
    double fisher_11;
    double fisher_22;
    double fisher_time;
} output;

/* misc/include/MLE_misc.h:184-328.  Fields this library reads: computation
 * ("exact"), kernel_fun, dm ("ed" | "gc"), precision (0 FP64, 2 mixed,
 * 3 FP64 with INT8-sliced updates -- new), diag_thick (band, in tiles), l1 / lobs / lmiss, verbose, log,
 * pFileLog, recovery_file, checkpoint_file.  The desc* handles hold this
 * library's device objects (opaque). */
typedef struct {
    double variance;
    double variance1;
    double variance2;
    double variance3;
    char *computation;
    char *c_fun;
    int test;
    int async;
    int iter_count;
    location l1;
    location lmiss;
    location lobs;
    location lm;
    void *descC;
    void *descsubC11;
    void *descsubC12;
    void *descsubC21;
    void *descsubC22;
    void *descZ;
    void *descZ1;
    void *descZ2;
    void *descZ3;
    double *Adense;
    double *Adense2;
    void *descZcpy;
    void *descdet;
    void *descsum;
    void *descproduct;
    void *descproduct1;
    void *descproduct2;
    void *descproduct3;
    void *descZmiss;
    void *descC11;
    void *descC21;
    void *descC12;
    void *descC22;
    void *descZactual;
    void *descZobs;
    void *descmse;
    void *descmse1;
    void *descmse2;
    void *descmse3;
    void *descZtrace;
    void *sequence;
    void *request;
    int verbose;
    int check;
    int log;
    double avg_exec_time_per_iter;
    double total_exec_time;
    double avg_flops_per_iter;
    double avg_generation_per_iter;
    double avg_solve_per_iter;
    double avg_cholesky_per_iter;
    double avg_exec_time_gen_stage;
    double avg_flops_gen_stage;
    double final_loglik;
    char *locsFPath;
    char *timeFPath;
    char *obsFPath;
    char *obsFPath2;
    char *obsFPath3;
    char *actualZFPath;
    char *actualZFPath2;
    char *actualZFPath3;
    char *actualZLocFPath;
    char *actualTimeFPath;
    double det;
    double sum;
    double dotp;
    double dotp1;
    double dotp2;
    double dotp3;
    float sdotp;
    double mserror;
    double mserror1;
    double mserror2;
    double mserror3;
    char *dm;
    int diag_thick;
    char *nFileLog;
    FILE *pFileLog;
    int hicma_maxrank;
    int hicma_data_type;
    void *hicma_descC;
    void *hicma_descZ;
    void *hicma_descCD;
    void *hicma_descCUV;
    void *hicma_descCrk;
    void *hicma_descZcpy;
    void *hicma_descdet;
    void *hicma_descproduct;
    void *hicma_descC12D;
    void *hicma_descC12UV;
    void *hicma_descC12rk;
    void *hicma_descC22D;
    void *hicma_descC22UV;
    void *hicma_descC22rk;
    double hicma_acc;
    void *hsequence;
    void *hrequest;
    int opt_tol;
    int opt_max_iters;
    int ooc;
    char *kernel_fun;
    int precision;
    void *desctemp;
    void *desctemp22;
    void *desck_t;
    void *desck_a;
    void *desck_ttmp;
    void *desck_atmp;
    void *descK_t;
    void *descK_a;
    void *descexpr1;
    void *descexpr2;
    void *descexpr3;
    void *descexpr4;
    void *descestimatedalpha;
    void *desctruthalpha;
    void *desc_mloe_mmom;
    void *descmloe;
    void *descmmom;
    double expr1;
    double expr2;
    double expr3;
    double expr4;
    double mloe;
    double mmom;
    int mloe_mmom;
    int mloe_mmom_async;
    int mspe;
    char *recovery_file;
    char *checkpoint_file;
    int time_slots;
    int idw;
    int fisher;
    void *descr;
    void *descrcpy;
    int seed;
} MLE_data;

/* The reference's global result record (misc/include/MLE_misc.h:350, defined
 * by the driver in examples/examples.c:24).  Defined weakly here so a driver
 * that defines its own keeps working. */
extern output results;

/* ---- reference entry points ---- */

/* src/include/MLE.h:54-55 (src/compute/MLE.c:233-260).  Selects the CUDA
 * device (the current one), creates the stream and records *dts as the
 * default tile size (0 = choose automatically).  ncores and lts are
 * accepted and ignored; *gpus must be 0 or 1 (one GPU per field).  A second
 * call prints the reference's warning and keeps the first context. */
void exageostat_init(int *ncores, int *gpus, int *dts, int *lts);
void EXAGEOSTAT_init(int *ncores, int *gpus, int *dts, int *lts); /* alias */

/* src/include/MLE.h:57 (src/compute/MLE.c:263-281). */
void exageostat_finalize(void);

/* exageostat_exact/src/include/MLE_exact.h:60-62 (MLE_dexact.c:1938-2017).
 * Allocates the device covariance (lower tiles of size dts), z and the
 * solve buffers for N locations and uploads data->l1.x / l1.y (for
 * bivariate_matern_parsimonious N is twice the number of locations, as the
 * reference driver sets it, synthetic_dmle_test.c:134).  Handles are
 * stored in data->descC / descZ / descZcpy.  On failure data->descC stays
 * NULL and exageostat_last_error() says why.  MORSE_dmle_Call is the
 * MORSE-era name of the same function. */
void EXAGEOSTAT_dmle_Call(MLE_data *data, int ncores, int gpus, int dts, int p_grid, int q_grid, int N, int nZobs,
                          int nZmiss);
void MORSE_dmle_Call(MLE_data *data, int ncores, int gpus, int dts, int p_grid, int q_grid, int N, int nZobs,
                     int nZmiss);

/* src/include/MLE.h:40-42 (src/compute/MLE.c:38-92 -> MLE_dexact.c:25-148).
 * z = chol(Sigma(initial_theta)) * Nrand on the device; Nrand is n host
 * doubles.  Resets data->iter_count.  `log` writes nothing here. */
void MLE_zvg(MLE_data *data, double *Nrand, double *initial_theta, int n, int ts, int log, int p_grid, int q_grid);

/* src/include/MLE.h:48-49 (src/compute/MLE.c:138-193): NLopt objective,
 * dispatching on data->precision (0: FP64, 2: banded mixed precision, 3: FP64
 * tiles with INT8-sliced off-band updates, see exageostat_b200_set_sliced).
 * Returns the log-likelihood.  New: when grad != NULL it receives d loglik /
 * d theta (the reference ignores grad).  A non-positive-definite covariance
 * returns -INFINITY (the reference exits). */
double MLE_alg(unsigned n, const double *theta, double *grad, void *data);

/* exageostat_exact/src/include/MLE_exact.h:43-44 (MLE_dexact.c:231-489). */
double EXAGEOSTAT_dmle_Tile(unsigned n, const double *theta, double *grad, void *data);

/* The banded mixed-precision objective (EXAGEOSTAT_sdmle_Tile,
 * exageostat_exact/src/compute/MLE_sdexact.c:172-357): tiles within
 * data->diag_thick tiles of the diagonal in FP64, the others stored FP32 and
 * updated on the TF32 tensor cores (three passes by default, see
 * exageostat_b200_set_mixed).  grad must be NULL (the gradient is FP64 only). */
double EXAGEOSTAT_sdmle_Tile(unsigned n, const double *theta, double *grad, void *data);
double MORSE_dmle_Tile(unsigned n, const double *theta, double *grad, void *data);

/* src/include/MLE.h:67 (src/compute/MLE.c:420-430): copies the synthetic z
 * (n doubles) to host memory. */
void MLE_get_zobs(MLE_data *data, double *z, int n);

/* src/include/MLE.h:59-61 (src/compute/MLE.c:284-306 -> MLE_dexact.c:613-685).
 * nZmiss, nZobs count locations; the bivariate kernel doubles them into
 * matrix rows (MLE_dexact.c:640-653), and EXAGEOSTAT_dmle_Predict_Tile then
 * takes the row counts (2 nZmiss, 2 nZobs), sets data->mserror1 / mserror2
 * and results.mse_pred1 / _pred2 to the per-variable errors. */
void prediction_init(MLE_data *data, int nZmiss, int nZobs, int ts, int p_grid, int q_grid, int mse_flag);
void EXAGEOSTAT_dmle_Predict_Allocate(MLE_data *data, int nZmiss, int nZobs, int dts, int p_grid, int q_grid,
                                      int mse_flag);

/* exageostat_exact/src/include/MLE_exact.h:49-51 (MLE_dexact.c:688-874).
 * Kriging of the nZmiss locations data->lmiss from the nZobs observations
 * Zobs at data->lobs.  Writes Zmiss; returns the MSE against Zactual, or -1
 * when Zactual is NULL or nZmiss <= 0 (as the reference), -2 on a
 * non-positive-definite C22. */
double EXAGEOSTAT_dmle_Predict_Tile(MLE_data *data, double *theta, int nZmiss, int nZobs, double *Zobs,
                                    double *Zactual, double *Zmiss, int n);
double MORSE_dmle_Predict_Tile(MLE_data *data, double *theta, int nZmiss, int nZobs, double *Zobs, double *Zactual,
                               double *Zmiss, int n);

/* src/include/MLE.h:63 and :65. */
void prediction_finalize(MLE_data *data);
void MLE_Finalize(MLE_data *data);

/* ---- assessment of a fitted model ---- */

/* exageostat_exact/src/include/MLE_exact.h:78-79 (MLE_dexact.c:1777-1934).
 * Fisher information of the N locations behind data (after
 * EXAGEOSTAT_dmle_Call) for univariate_matern_stationary at initial_theta:
 * F_jk = 1/2 tr(Sigma^-1 dSigma_j Sigma^-1 dSigma_k), j, k over (sigma^2,
 * beta, nu).  Returns a malloc'd array of 10 doubles, the first 9 the
 * column-major inverse of F (the last 0), as the reference; sets
 * results.fisher_00/_11/_22 (diagonal of the inverse) and fisher_time.
 * NULL on an error (non-positive-definite Sigma or F; see exageostat_last_error). */
double *EXAGEOSTAT_Fisher_Tile(MLE_data *data, int N, double *initial_theta, int dts, int p_grid, int q_grid);

/* src/include/MLE.h:71-72 (src/compute/MLE.c:309-320 -> MLE_dexact.c:1002-1107):
 * allocates the MLOE / MMOM workspace for nZmiss missing and nZobs observed
 * locations and sets data->mloe = data->mmom = 0. */
void mloe_mmom_init(MLE_data *data, int nZmiss, int nZobs, int ts, int p_grid, int q_grid);
void EXAGEOSTAT_dmle_mloe_mmom_Allocate(MLE_data *data, int nZmiss, int nZobs, int dts, int p_grid, int q_grid);

/* exageostat_exact/src/include/MLE_exact.h:72-76 (MLE_dexact.c:1109-1434 and
 * :1437-1774).  Mean loss of efficiency and mean misspecification of the
 * mean square error of kriging the locations data->lmiss from data->lobs
 * with estimated_theta when truth_theta is the truth:
 *   MLOE = mean_m (E_t[err_a^2] / E_t[err_t^2] - 1),
 *   MMOM = mean_m (E_a[err_a^2] / E_t[err_a^2] - 1).
 * Results in data->mloe, data->mmom, results.mloe / mmom and the
 * results.*_mloe_mmom_* times.  Each call computes both afresh (the reference
 * adds to the previous values of data->mloe / mmom).  The two entry points
 * are one computation (all missing points in one batch of tile solves). */
void EXAGEOSTAT_dmle_mloe_mmom_Tile(MLE_data *data, double *truth_theta, double *estimated_theta, int nZmiss,
                                    int nZobs, int n);
void EXAGEOSTAT_dmle_mloe_mmom_Tile_Async(MLE_data *data, double *truth_theta, double *estimated_theta, int nZmiss,
                                          int nZobs, int n);

/* src/compute/MLE.c:323-337; src/include/MLE.h:74 declares it as
 * MLOE_MMOM_Finalize, which is exported too. */
void mloe_mmom_finalize(MLE_data *data);
void MLOE_MMOM_Finalize(MLE_data *data);

/* ---- host-side synthetic data helpers (misc/include/MLE_misc.h) ---- */

/* misc/compute/MLE_misc.c:763-792: srand(seed), jittered ceil(sqrt(n))^2
 * grid, Morton sort with uint16 quantisation.  Returns a malloc'd location
 * whose x / y are malloc'd n-arrays (free with free()). */
location *GenerateXYLoc(int n, int seed);
/* misc/compute/MLE_misc.c:753-761 */
double uniform_distribution(double rangeLow, double rangeHigh);
/* misc/compute/MLE_misc.c:1238-1259 */
void shuffle(double *array, location *locations, size_t n);
/* misc/compute/MLE_misc.c:453-534 */
int locations_obs_zsort_inplace(int n, location *locations, double *z);
/* misc/compute/MLE_misc.c:1700-1741: splits the synthetic z (from the
 * device) into missing / observed sets with the libc rand() stream;
 * data->lmiss.x / .y are malloc'd N-arrays and data->lobs points into them
 * at offset nZmiss, as in the reference. */
void pick_random_points(MLE_data *data, double *Zobs, double *Zactual, int nZmiss, int nZobs, int N);
/* misc/compute/MLE_misc.c:1261-1285, 1744-1810 (MLE_misc.h:442): the
 * bivariate forms.  N = 2 x locations; nZmiss, nZobs count locations; Zobs
 * and Zactual receive 2 nZobs and 2 nZmiss interleaved values. */
void shuffle2(double *array, double *array2, location *locations, size_t n);
void pick_random_points2(MLE_data *data, double *Zobs, double *Zactual, int nZmiss, int nZobs, int N);

/* ---- real-data flat files (misc/include/flat_file.h:25-31, MLE_misc.h:382) ----
 * countlines: the number of '\n' characters of the file (0 if it cannot be
 * opened).  The readers take n rows of comma-separated numbers ("x,y",
 * "x,y,z", or one value per line) into malloc'd arrays the caller frees;
 * blank lines are skipped.  They return NULL with a message on a missing
 * file, a short or malformed row, or fewer than n rows (the reference
 * writes past its arrays on a longer file and crashes on a short row). */
int countlines(char *filename);
location *readLocsFile(char *locs_file, int n);
location *readLocsFile3d(char *locs_file, int n);
double *readObsFile(char *obsfile, int n);
double *readTimeFile(char *timefile, int n);

/* ---- MLE driver ---- */

/* Bound-constrained derivative-free maximiser standing in for NLopt's
 * LN_BOBYQA, which the reference driver uses (examples/synthetic_dmle_test.c:
 * 140-142, 283-284; nlopt_set_ftol_abs / bounds in init_optimizer,
 * misc/compute/MLE_misc.c:1352-1366).  f has NLopt's objective signature, so
 * MLE_alg plugs in with data = the MLE_data pointer.  x holds the start and
 * receives the maximiser; rhobeg <= 0 picks a quarter of the smallest bound
 * range; ftol_abs > 0 stops after two accepted steps in a row that change f
 * by less;
 * maxeval <= 0 means no limit.  Returns the number of evaluations (or
 * -XG_ERR_BAD_ARGUMENT); *fmax receives the best value. */
int exageostat_b200_bobyqa(int n, double *x, const double *lb, const double *ub, double rhobeg, double rhoend,
                           double ftol_abs, int maxeval, double (*f)(unsigned, const double *, double *, void *),
                           void *data, double *fmax);

/* ---- new entry points (no counterpart in the reference) ---- */

/* Status-returning form of MLE_alg: 0 on success, else an XG_ERR_* code;
 * loglik receives the value, grad (may be NULL) the gradient. */
int exageostat_b200_loglik(MLE_data *data, const double *theta, double *loglik, double *grad);

/* Text of the last error on the calling thread ("" if none). */
const char *exageostat_last_error(void);

#define XG_OK 0
#define XG_ERR_NOT_INITIALIZED 1
#define XG_ERR_BAD_ARGUMENT 2
#define XG_ERR_CUDA 3
#define XG_ERR_NOT_SPD 4
#define XG_ERR_TIMEOUT 5
#define XG_ERR_UNSUPPORTED 6
#define XG_ERR_NO_MEMORY 7

/* Library / ABI introspection (used by the bindings' layout checks). */
int exageostat_b200_abi_version(void);
size_t exageostat_b200_sizeof_MLE_data(void);
size_t exageostat_b200_sizeof_output(void);
long exageostat_b200_offsetof_MLE_data(const char *field);

/* One-shot evaluation on host arrays (no MLE_data): uploads x, y, z (n
 * doubles each), evaluates the log-likelihood at theta (3 values, or 4 for
 * kernel 1 = Matern + nugget) with tile size ts (0 = automatic) and copies
 * the result back.  out[0..2] = loglik, logdet, z^T Sigma^-1 z. */
int exageostat_b200_dmle_host(int n, const double *x, const double *y, const double *z, const double *theta,
                              int kernel, int metric, int ts, double *out);

/* Band width (tiles kept in FP64, >= 1; also written to data->diag_thick) and
 * number of TF32 passes (1, or 3 for the hi/lo split with FP32-class
 * products) of the mixed-precision path (precision = 2). */
int exageostat_b200_set_mixed(MLE_data *data, int band, int passes);

/* One-shot mixed-precision log-likelihood on host arrays (as
 * exageostat_b200_dmle_host; ts must be a multiple of 256, 0 = 512). */
int exageostat_b200_dmle_host_mixed(int n, const double *x, const double *y, const double *z, const double *theta,
                                    int kernel, int metric, int ts, int band, int passes, double *out);

/* No counterpart in the reference (precision = 3).  Every tile stays FP64 and
 * the diagonal POTRF, the panel TRSM, the log-det and the solve run in FP64;
 * the trailing updates A_ij -= L_ik L_jk^T run on the INT8 tensor cores as
 * exact integer products of four 8-bit slices per operand with an FP64 scale
 * per row and panel (~32 significant bits relative to the row maximum, exact
 * S32 accumulation), in left-looking order.  Sets data->precision = 3; grad
 * must be NULL.  Needs 4 bytes of device memory per covariance element on
 * top of the FP64 tiles (20 GB at N = 100,000). */
int exageostat_b200_set_sliced(MLE_data *data);

/* One-shot INT8-sliced log-likelihood on host arrays (as
 * exageostat_b200_dmle_host; ts 0 = automatic, else a multiple of 128). */
int exageostat_b200_dmle_host_sliced(int n, const double *x, const double *y, const double *z, const double *theta,
                                     int kernel, int metric, int ts, double *out);

/* No counterpart in the reference.  Chooses the tile size by timing one
 * evaluation at theta for tile sizes 128, 256, 384 and 512 (multiples of 256
 * for precision 2) on temporary descriptors with the same locations
 * (data->l1) and observations, and rebuilds the descriptors with the
 * fastest (*ts).  For precision 2 it then times band widths 1, 2, 4, 8 and
 * keeps the fastest whose |dl| / |l| against one FP64 evaluation is <= tol
 * (0 = 1e-6; the most accurate band if none is), also written to
 * data->diag_thick (*band; 0 for the other precisions).  report (may be NULL)
 * receives up to 4 (tile size, seconds) pairs.  Needs the memory of two
 * descriptor sets at once. */
int exageostat_b200_autotune(MLE_data *data, const double *theta, double tol, int *ts, int *band, double *report);

/* Replaces the locations and/or observations (N host doubles each; NULL
 * keeps the current array) of an allocated MLE_data, e.g. for a new dataset
 * of the same size, without reallocating the device covariance. */
int exageostat_b200_set_data(MLE_data *data, const double *x, const double *y, const double *z);

/* Per-kernel-class CUDA-event timing of the log-likelihood evaluations of
 * one MLE_data.  set_profiling(on) resets the counters; get_profile fills
 * out[0..10] = seconds in generation, diagonal POTRF, panel TRSM, trailing
 * update (the panel overlaps the trailing update, so these may add up to
 * more than the total); trailing-update algorithmic flops; kernel launches;
 * evaluations; total seconds (generation to result); tile size; tiles per
 * side; N; and for the reduced-precision paths out[11..14] = seconds and
 * algorithmic flops of the off-band (TF32 tensor-core, precision 2; INT8
 * tensor-core, precision 3: every target) and band (FP64, precision 2)
 * trailing updates. */
int exageostat_b200_set_profiling(MLE_data *data, int on);
int exageostat_b200_get_profile(MLE_data *data, double *out, int n);

/* No counterpart in the reference.  The log-likelihood of
 * exageostat_b200_dmle_host for callers that cannot call cudaMalloc (code
 * running inside another framework's allocator or memory pool, or with the
 * device heap exhausted).  Inputs and the result are DEVICE pointers owned by
 * the caller: d_x, d_y, d_z (n doubles each) and d_out (3 doubles: loglik,
 * logdet, z^T Sigma^-1 z); theta (3 or 4 values) is a host pointer; stream is
 * a cudaStream_t (NULL = default stream); metric is 0 (Euclidean) or 1
 * (great circle), anything else is XG_ERR_BAD_ARGUMENT.  The call is
 * synchronous: it waits for its stream work and reads the status back before
 * it returns.  d_out is written only on success; when the call returns an
 * error, d_out keeps its previous contents.  The library works in one static
 * device array of about 18 MB that every GPU loading the library holds until
 * exit, so n is at most 2048 (larger n returns XG_ERR_BAD_ARGUMENT).  The
 * first call on a device checks that it is an sm_100 GPU, looks up that
 * array's device address and sets up the kernels: make it before any stream
 * capture.  The address is cached per device ordinal, so only each device's
 * primary context is supported.  All calls share the array; calls that
 * overlap on the GPU race and must be serialised by the caller. */
int exageostat_b200_dmle_device_noalloc(int n, const double *d_x, const double *d_y, const double *d_z,
                                        const double *theta, int kernel, int metric, double *d_out, void *stream);

/* Status-returning Fisher information for data's kernel (3 x 3, or 4 x 4
 * with the nugget tau^2 last): fisher and fisher_inv (either may be NULL)
 * receive the row-major matrix and its inverse. */
int exageostat_b200_fisher(MLE_data *data, const double *theta, double *fisher, double *fisher_inv);

/* One-shot forms on host arrays.  fisher_host: n locations, fisher np x np.
 * mloe_mmom_host: terms (NULL or 6 doubles per missing point) receives, per
 * point, expr1 = k_t' K_a^-1 k_a, expr2 = E_t[err_a^2], expr3 = E_t[err_t^2],
 * expr4 = E_a[err_a^2], loe, mom (the reference's descexpr1..4 after its
 * geadd steps, MLE_dexact.c:1371-1375, and the per-point terms of
 * codelet_zmloe_mmom.c:48-60); times (NULL or 4) generation, factorisation,
 * solves and total seconds. */
int exageostat_b200_fisher_host(int n, const double *x, const double *y, const double *theta, int kernel, int metric,
                                int ts, double *fisher);
int exageostat_b200_mloe_mmom_host(int nmiss, const double *xmiss, const double *ymiss, int nobs, const double *xobs,
                                   const double *yobs, const double *truth_theta, const double *estimated_theta,
                                   int kernel, int metric, int ts, double *mloe, double *mmom, double *terms,
                                   double *times);

/* ---- batches of independent fields (no counterpart in the reference) ----
 * nfields fields with n[f] locations each; x, y, z hold the fields one after
 * the other (sum n[f] doubles each).  kernel / metric as for
 * exageostat_b200_dmle_host, ts = tile size (0 = 256).  The fields share one
 * device tile store and each evaluation of all of them is one CUDA-graph
 * launch (one launch per tile step covering every field). */
int exageostat_b200_batch_create(int nfields, const int *n, const double *x, const double *y, const double *z,
                                 int kernel, int metric, int ts, void **handle);
/* theta: nfields rows of 3 (4 with the nugget) parameters; loglik receives
 * nfields values (-INFINITY for a field whose covariance is not positive
 * definite; the call then still returns 0 and exageostat_last_error() says
 * how many failed). */
int exageostat_b200_batch_loglik(void *handle, const double *theta, double *loglik);
/* The log-likelihoods and their gradients (nfields rows of 3, or 4 with the
 * nugget) of every field at theta: the batched factorisation, then the
 * adjoint of each field on its own tiles.  A field whose covariance is not
 * positive definite gets loglik -inf and NaN gradient entries. */
int exageostat_b200_batch_loglik_grad(void *handle, const double *theta, double *loglik, double *grad);
int exageostat_b200_batch_destroy(void *handle);

/* As exageostat_b200_batch_create with the tile size chosen by timing: the
 * batch is built with tile sizes 128, 256, 384 and 512 in turn and timed on
 * one evaluation at theta (nfields rows); the fastest is returned in *handle
 * and its tile size in *ts.  report (may be NULL) receives up to 4
 * (tile size, seconds) pairs. */
int exageostat_b200_batch_autotune(int nfields, const int *n, const double *x, const double *y, const double *z,
                                   int kernel, int metric, const double *theta, int *ts, double *report,
                                   void **handle);

/* The device scheduler's task list for fields of nt[f] tiles per side and
 * `workers` persistent CTAs (host only, no GPU needed): writes 4 ints per
 * task -- type | field << 2 (type 0 POTRF(k), 1 TRSM(i, k), 2 the update
 * (i, j) <- k), i, j, k -- to out when out is not NULL, and returns the
 * number of tasks.  exageostat_b200_batch_create builds its list this way;
 * exposed so the order can be checked (complete, topological). */
long long exageostat_b200_batch_plan(int nfields, const int *nt, int workers, int *out);

/* ---- diagnostics used by the parity tests (no counterpart in the reference; all run on the GPU) ---- */
/* Runs the bounded-wait path of the kernels on purpose: one thread waits on
 * a shared-memory barrier that nothing arrives on, gives up after limit_us
 * microseconds (1 to 1e6), records the timeout bit of a status word and
 * returns.  Returns XG_ERR_TIMEOUT (the expected result) and the measured
 * wait in *waited_us (may be NULL); the CUDA context stays usable. */
int exageostat_b200_diag_wait_timeout(double limit_us, double *waited_us);
int exageostat_b200_bessel_knu(int n, const double *nu, const double *x, double *out);
int exageostat_b200_matern_pairs(int n, const double *x1, const double *y1, const double *x2, const double *y2,
                                 const double *theta, int kernel, int metric, double *out);
/* Dense lower-triangular Sigma (factor = 0) or its Cholesky factor L
 * (factor = 1) of dimension n (the locations, or 2 x the locations for the
 * bivariate kernel), row-major n x n with zeros above the diagonal, computed
 * with tile size ts. */
int exageostat_b200_covariance_dense(int n, const double *x, const double *y, const double *theta, int kernel,
                                     int metric, int ts, int factor, double *out);
/* The factor L of the INT8-sliced path (all tiles FP64), row-major n x n
 * with zeros above the diagonal, for the parity tests. */
int exageostat_b200_sliced_factor_dense(int n, const double *x, const double *y, const double *theta, int kernel,
                                        int metric, int ts, double *out);

/* The mixed-precision factor L (band tiles FP64, off-band FP32 widened),
 * row-major n x n with zeros above the diagonal. */
int exageostat_b200_mixed_factor_dense(int n, const double *x, const double *y, const double *theta, int kernel,
                                       int metric, int ts, int band, int passes, double *out);

#ifdef __cplusplus
}
#endif

#endif
