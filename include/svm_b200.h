/*
 * svm_b200.h -- C-ABI of the B200 SVM engine beyond the svm.h drop-in API.
 *
 * Plain pointers and sizes only.  Every function returns 0 on success and a
 * negative value on failure; svmb_last_error() then describes the failure
 * (per calling thread).  Nothing here allocates memory the caller must free,
 * except the resident-rows handle (svmb_rows_free).
 *
 * The reference has no such layer: its svm.cpp calls the CudaSolver methods
 * (reference libsvm/cuda_solver.h:224-243: setup_solver, select_working_set,
 * compute_alpha, update_gradient, update_alpha_status, fetch_vectors) from
 * inside Solver::Solve (svm.cpp:556-776).  svmb_solve_binary_csr replaces that
 * whole seam with one call that runs an entire Solver::Solve /
 * Solver_NU::Solve on the device.
 */
#ifndef LIBSVM_B200_SVMB_H
#define LIBSVM_B200_SVMB_H

#include "svm.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Statistics of one binary solve (what the reference prints through info():
 * "#iter", "obj", "rho", "nSV", "nBSV", reference svm.cpp:821, 1739, 1763). */
typedef struct svmb_solve_stats {
    long long iters;
    double obj;          /* dual objective, after the nu-SVC 1/r^2 scaling */
    double rho;          /* after the nu-SVC 1/r scaling */
    double r;            /* nu-SVC only */
    int l;
    int nr_sv;
    int nr_bsv;
    int status;          /* 0 converged, 1 max_iter reached */
    int active_size;     /* active set size at exit (shrinking) */
    int launch;          /* index, within the call, of the persistent launch that solved it */
    double seconds;      /* device time (CUDA events) of the launch that solved it */
    /* work counters of the solve: sum over iterations of the active-set size,
     * kernel values evaluated, Q-row cache lookups and hits */
    long long sum_active;
    long long q_evals;
    long long lookups;
    long long hits;
    long long fills;            /* row-evaluation passes */
    long long prefetched;       /* rows evaluated ahead of need */
    long long prefetch_used;    /* of those, rows a later lookup hit */
    long long prof_cycles[8];   /* SM cycles per loop section (diagnostics) */
    long long fill_targets;     /* target positions of all row-evaluation passes: each pass reads
                                   every target row once, whatever the number of its source rows */
    int fill_path;              /* SVMB_FILL_*: how the solve evaluated its kernel rows */
    int reserved;
} svmb_solve_stats;

#define SVMB_FILL_DENSE          0  /* dense rows on CUDA cores, sources staged in shared memory */
#define SVMB_FILL_SPARSE_SCATTER 1  /* sparse rows; sources scattered into dense shared-memory vectors */
#define SVMB_FILL_SPARSE_TABLE   2  /* sparse rows too wide to scatter; sources in a column-keyed
                                       shared-memory table probed by each target's nonzeros */
#define SVMB_FILL_SPARSE_MERGE   3  /* sparse rows; merge walks of two index lists in global memory */
#define SVMB_FILL_TENSOR         4  /* tensor cores on the split copy of the rows */

/* Parameters of a binary solve (the subset of svm_parameter the solver reads). */
typedef struct svmb_params {
    int svm_type;        /* C_SVC, NU_SVC, ONE_CLASS, EPSILON_SVR or NU_SVR */
    int kernel_type;     /* LINEAR, POLY, RBF, SIGMOID */
    int degree;
    int shrinking;
    double gamma;
    double coef0;
    double C_pos;        /* C-SVC: C for y>0 (reference solve_c_svc Cp); epsilon-SVR / nu-SVR: C */
    double C_neg;        /* C-SVC: C for y<=0 (Cn) */
    double nu;           /* nu-SVC, one-class, nu-SVR */
    double eps;
    double cache_mb;     /* Q-row cache budget per solve, MB (svm_parameter.cache_size) */
    int form;            /* SVMB_FORM_* */
    int blocks;          /* thread blocks per solve; 0 = automatic */
    int prefetch;        /* kernel rows evaluated per cache-miss pass (1 = only the missing row); 0 = automatic */
    int gbar_mode;       /* SVMB_GBAR_*: how the gradient of the inactive variables is kept */
    double p;            /* epsilon-SVR: half-width of the insensitive tube (svm_parameter.p) */
} svmb_params;

#define SVMB_GBAR_AUTO        0  /* incremental for EXACT and FP32, recomputed for the tensor forms */
#define SVMB_GBAR_INCREMENTAL 1  /* G_bar updated on every bound change (reference svm.cpp:744-769) */
#define SVMB_GBAR_RECOMPUTE   2  /* no G_bar; reconstruction recomputes G = p + Q*alpha on the inactive
                                    variables as one block product, so no full-length rows are needed */

#define SVMB_FORM_EXACT 0   /* fp32 features, fp64 accumulation in feature order */
#define SVMB_FORM_FP32  1   /* fp32 features, fp32 accumulation (plain CUDA-core form) */
#define SVMB_FORM_BF16X3 2  /* tensor cores: features split x = hi + lo (bf16), dot = hi.hi + hi.lo + lo.hi
                               accumulated in fp32 (about 16 significant bits per product);
                               the split copy holds every row densely */
#define SVMB_FORM_FP16X3 3  /* tensor cores: each row scaled by a power of two and split x*2^e = hi + lo
                               (fp16), same three products in fp32 (about 22 significant bits) */
#define SVMB_FORM_TF32   4  /* tensor cores: features rounded to tf32, one product per pair
                               (kind::tf32, about 11 significant bits), fp32 accumulation */

const char *svmb_last_error(void);
/* Number of device kernels this library has launched in this process. */
long long svmb_kernel_launches(void);
/* Bytes this library has copied host->device and device->host in this process. */
void svmb_transfer_bytes(long long *h2d, long long *d2h);
int svmb_version(void);                         /* LIBSVM_VERSION * 100 + engine revision */
int svmb_device_available(void);                /* 1 if a CUDA device can be used */
/* A print function that discards its text: svm_set_print_string_function(
 * svmb_print_nothing) silences training output without a call back into the
 * caller (no counterpart in the reference, whose callers write their own). */
void svmb_print_nothing(const char *s);

/* Process-wide engine options used by svm_train / svm_cross_validation:
 *   "form"   SVMB_FORM_EXACT (default), SVMB_FORM_FP32, SVMB_FORM_BF16X3, SVMB_FORM_FP16X3 or SVMB_FORM_TF32
 *   "blocks" thread blocks per solve (0 = automatic)
 *   "layout" -1 automatic, 0 CSR, 1 dense device layout of the rows
 *   "prefetch" kernel rows per cache-miss pass (1 = none, 0 = automatic)
 *   "graphs" 1 (default): repeated launches replay a captured CUDA graph; 0: plain stream work
 *   "autotune" 1 (default): per workload signature (form, layout, width,
 *            instance sizes) the first calls try fill depths and block targets
 *            and later calls use the fastest; results never depend on them.
 *            0: fixed rules.  Instances with their own prefetch or blocks are
 *            never tuned.
 *   "fill_depth" 1..4 (default 2): deepest ring of column slices per warp in the
 *            CUDA-core row fills (a launch takes the deepest that keeps its
 *            instances in one launch); speed only, results never depend on it
 *   "predict_form" SVMB_FORM_EXACT (default: the reference's kernel values bit
 *            for bit) or a tensor-core form: svm_predict* and svmb_predict_batch
 *            then evaluate K(test rows, SVs) as block products on the tensor cores
 *   "blocks_per_sm" 1 (default) to 4: solver blocks one SM may hold; each gets
 *            that share of the SM's shared memory (speed only)
 *   "wait_limit_ms" bound of every wait of a solver block for the other blocks
 *            of its group (0 = the default, 30 s); a wait that runs out makes
 *            the whole group return and the call report an error
 *   "test_drop_block" 1: the next solver launch leaves out its last thread
 *            block (one shot), so that its group's waits run out; for testing
 *            the timeout path (the instance must have two or more blocks) */
int svmb_set_option(const char *name, long long value);

/* The autotuner's configuration of the last batched solve of this process:
 * rows per fill pass (0 = as deep as staging allows), positions per block
 * aimed at, and whether it was an exploring call. */
void svmb_autotune_last(int *prefetch, int *rows_per_block, int *exploring);

/* CUDA graphs of the engine's batched launches: graphs captured and graph
 * launches so far in this process.  A launch whose layout, device block and
 * host staging repeat an earlier one's replays that launch's captured stream
 * work (upload, fills, kernel, timing events, download). */
void svmb_graph_counts(long long *captured, long long *replayed);

/* Per-subproblem statistics of the last svm_train / svm_cross_validation
 * call on this process; returns the number of records (copies at most cap). */
int svmb_last_train_stats(svmb_solve_stats *out, int cap);

/* svm_cross_validation (reference svm.cpp:2407-2525) over a grid of npoints
 * (C[p], gamma[p]) values in one call: the folds are drawn once with rand(),
 * exactly as svm_cross_validation draws them, and the one-vs-one subproblems
 * of every point and fold are solved in batched launches over rows uploaded
 * once.  target[p*l + i] receives the prediction for row i of the model of
 * point p trained without i's fold (NaN where that training failed). */
int svmb_cross_validation_grid(const struct svm_problem *prob, const struct svm_parameter *param, int nr_fold,
                               int npoints, const double *C, const double *gamma, double *target);

/* Decision values of n rows in one device pass (the batched form of
 * svm_predict_values, reference svm.cpp:2569-2643).  labels[n] (one-class:
 * +1/-1; epsilon-SVR / nu-SVR: the predicted value); dec_values may be NULL
 * or [n][nr_class*(nr_class-1)/2] (one value per row for one-class and SVR). */
int svmb_predict_batch(const struct svm_model *model, const struct svm_node *const *rows, int n,
                       double *labels, double *dec_values);

/* Labels and class probabilities of n rows (the batched form of
 * svm_predict_probability, reference svm.cpp:2660-2697) of a C-SVC / nu-SVC
 * model trained with probability = 1: the pairs' decision values in one
 * device pass, then each pair's sigmoid and the pairwise coupling.
 * labels[n], prob_estimates[n][nr_class] in the model's label order. */
int svmb_predict_probability_batch(const struct svm_model *model, const struct svm_node *const *rows, int n,
                                   double *labels, double *prob_estimates);

/* One solve from host CSR rows (0-based columns, n rows, d columns) in the
 * formulation params->svm_type.  Classifiers: y[i] > 0 is the positive class;
 * one-class: y is ignored; SVR: y are the regression targets.  alpha_out[n]
 * receives the reference's decision_function.alpha: y_i*alpha_i for C-SVC
 * (nu-SVC: divided by r), alpha_i for one-class, alpha_i - alpha*_i for SVR
 * (svm.cpp:1532, :1578-1584, :1650-1655, :1691-1692); stats may be NULL.
 * Host buffers; host<->device copies are part of the call. */
int svmb_solve_binary_csr(int n, int d, const long long *rowptr, const int *col, const float *val,
                          const double *y, const svmb_params *params, double *alpha_out,
                          svmb_solve_stats *stats);

/* Many independent binary solves over subsets of one row set, in ONE
 * persistent device launch (one-vs-one pairs, CV folds, grid points).
 * Instance k uses rows inst_rows[inst_ptr[k] .. inst_ptr[k+1]) with labels
 * inst_y[same range] and params[k] (each instance has its own kernel, C,
 * eps, cache budget ...: a C x gamma grid of CV folds is one call); only the
 * arithmetic form must agree across instances.  alpha_out is laid out like
 * inst_rows. */
int svmb_solve_many_csr(int n, int d, const long long *rowptr, const int *col, const float *val,
                        int ninst, const int *inst_ptr, const int *inst_rows, const double *inst_y,
                        const svmb_params *params, double *alpha_out, svmb_solve_stats *stats);

/* One binary C-SVC solve that allocates no memory.  This entry point has no
 * counterpart in the reference.  It is for callers that cannot allocate device
 * memory once they are running (a server with a fixed device-memory pool, a
 * host application that owns every allocation): rows X [n][ld] (float32,
 * row-major, ld a multiple of 4, X 16-byte aligned), labels y[n] (y > 0 is the positive class)
 * and alpha_out[n] are DEVICE pointers the caller owns; params and stats are
 * host pointers (stats may be NULL; its nr_sv/nr_bsv/seconds are not filled).
 * All solver state lives in a fixed 8 MiB workspace compiled into the library
 * (held by every GPU that loads it, until exit), so n is limited to 16384 and
 * the Q-row cache to what remains of the workspace; larger n is rejected.
 * The first call on each device looks up the workspace address, so make it
 * before any stream capture; the address is kept for the process's lifetime,
 * so it is stale after the caller resets the device (cudaDeviceReset).  Calls
 * share the workspace: two calls whose work
 * overlaps on the GPU race on it.  `stream` is a cudaStream_t (NULL = legacy
 * default stream); the call returns after the solve has finished. */
int svmb_solve_dense_noalloc(int n, int ld, const float *X, const double *y, const svmb_params *params,
                             double *alpha_out, svmb_solve_stats *stats, void *stream);

/* Read a libsvm text file ("label idx:val ...") with the acceptance rules of
 * the reference's read_problem (svm-train/svm-train.c:288-389), parsed by all
 * host threads.  On success prob->l, prob->y, prob->x (rows terminated by
 * index -1, pointing into *x_space) and *max_index (largest feature index, 0
 * if none) are set; free them with svmb_free_problem.  Returns -1 if the file
 * cannot be read, -2 for a malformed line, whose 1-based number goes to
 * *bad_line (may be NULL), as the reference's "Wrong input format at line N". */
int svmb_read_problem(const char *path, struct svm_problem *prob, struct svm_node **x_space, int *max_index,
                      long long *bad_line);
void svmb_free_problem(struct svm_problem *prob, struct svm_node *x_space);

/* Resident rows: upload once, solve many times (the data stays in HBM). */
typedef struct svmb_rows svmb_rows;
int svmb_rows_upload_csr(int n, int d, const long long *rowptr, const int *col, const float *val,
                         int layout /* -1 auto, 0 CSR, 1 dense */, svmb_rows **out);
int svmb_rows_info(const svmb_rows *rows, int *n, int *d, int *dense, long long *bytes);
int svmb_rows_solve_many(const svmb_rows *rows, int ninst, const int *inst_ptr, const int *inst_rows,
                         const double *inst_y, const svmb_params *params, double *alpha_out,
                         svmb_solve_stats *stats);
void svmb_rows_free(svmb_rows *rows);

/* Kernel-matrix block out[i][j] = K(x_ia[i], x_ib[j]) (row-major [ma][nb],
 * float64) of resident rows, with params' kernel and form: the block form of
 * the reference's Kernel::k_function / SVC_Q::get_Q (svm.cpp:235-254,
 * :305-325, :1316-1340).  SVMB_FORM_BF16X3 and SVMB_FORM_FP16X3 run on the
 * tensor cores, the other forms on CUDA cores.  ia, ib, out are host arrays. */
int svmb_rows_kernel_block(const svmb_rows *rows, const svmb_params *params, int ma, const int *ia, int nb,
                           const int *ib, double *out);

/* ---- request loop (continuous batching of independent solves) ------------
 * No counterpart in the reference, which trains one problem per call.  A
 * scheduler thread picks a leading request (the policy), adds pending
 * requests of a similar size while their device memory (rows + solver state
 * with the Q-row cache budget) fits the server's budget and the thread blocks
 * they need fit the SMs that no running launch holds, and launches them
 * together next to the launches already running (up to max_inflight at a
 * time).  A request's result equals its solve alone. */
typedef struct svmb_server svmb_server;
typedef struct svmb_server_config {
    long long mem_bytes;     /* device memory for admitted requests; 0 = 80% of the free memory */
    int max_inflight;        /* concurrent launches; 0 = 8 */
    int max_batch;           /* requests per launch; 0 = 32 */
    int form;                /* SVMB_FORM_* of every request */
    int policy;              /* SVMB_SERVE_*: which pending request leads the next launch */
    int rows_per_block;      /* thread blocks per request = rows / rows_per_block (at least 1); 0 = 2000 */
} svmb_server_config;
#define SVMB_SERVE_SMALLEST_FIRST 0  /* the smallest pending request, unless one has waited over 2 s */
#define SVMB_SERVE_ARRIVAL_ORDER  1  /* the oldest pending request */
typedef struct svmb_server_stats {
    long long completed, failed, waves, max_concurrent_waves, peak_mem_bytes, pending;
    double p50_s, p99_s, max_s;   /* request latency: submit -> result ready */
    double solves_per_s;          /* completed / (last completion - first submit) */
} svmb_server_stats;

int svmb_server_create(const svmb_server_config *cfg, svmb_server **out);
/* One binary request from host CSR rows (copied; 0-based columns < d) and
 * labels y[n] (y > 0 positive).  Returns a ticket >= 0, or -1. */
long long svmb_server_submit(svmb_server *s, int n, int d, const long long *rowptr, const int *col, const float *val,
                             const double *y, const svmb_params *params);
int svmb_server_poll(svmb_server *s, long long ticket);       /* 1 finished, 0 running or queued, -1 unknown */
/* Wait for a ticket (collected once): alpha_out[n] receives the signed
 * coefficients as in svmb_solve_binary_csr; stats and latency_s may be NULL. */
int svmb_server_wait(svmb_server *s, long long ticket, double *alpha_out, svmb_solve_stats *stats, double *latency_s);
int svmb_server_get_stats(svmb_server *s, svmb_server_stats *out);
void svmb_server_destroy(svmb_server *s);      /* finishes the admitted and queued requests first */

#ifdef __cplusplus
}
#endif

#endif /* LIBSVM_B200_SVMB_H */
