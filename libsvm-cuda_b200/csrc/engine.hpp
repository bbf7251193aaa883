// engine.hpp -- host-side interface of the device solver (C++, internal).
#pragma once
#include <cuda_runtime.h>

#include <array>
#include <string>
#include <vector>

#include "engine.h"

struct svm_node;

namespace svmb {

void set_error(const std::string &msg);
const char *last_error();

// Feature rows resident in HBM.  Dense when the matrix is dense enough,
// otherwise CSR.  Row ids are the caller's row order.
struct DeviceRows {
    int n = 0;
    int d = 0;                  // feature columns (max index)
    int ld = 0;                 // dense row stride in floats
    bool dense = false;
    float *X = nullptr;
    long long *rowptr = nullptr;
    int *col = nullptr;
    float *val = nullptr;
    double *xsq[2] = {nullptr, nullptr};   // FORM_EXACT, FORM_FP32 (the tensor form uses the FP32 norms)
    uint16_t *Xs = nullptr;    // split rows of a tensor form (split_form), built on first use
    double *xinv = nullptr;    // FORM_FP16X3 per-row inverse scales
    int split_form = -1;
    long long nnz = 0;         // stored values (CSR)
    int nchunk = 0;
    size_t bytes = 0;          // device bytes of the layout the solver reads
    size_t h2d_bytes = 0;      // bytes copied from the host by the upload
    char *block = nullptr;     // one device block holding the rows and norms
    bool block_async = false;  // allocated stream-ordered (freed with release_async)
    bool block_pooled = false; // the process's reusable row block (returned, not freed)
    size_t block_bytes = 0;
    ~DeviceRows();
    void release_async(cudaStream_t s);
    DevX view(int form) const;
    // build Xs if the form needs it; -1 (error set) when the rows cannot take the form
    int prepare_form(int form, cudaStream_t s);
};

// Upload rows given as libsvm svm_node lists (index >= 1, terminated by -1).
// force: -1 auto, 0 CSR, 1 dense.
int upload_rows(const svm_node *const *x, int n, DeviceRows &out, int force, cudaStream_t s, int alloc = 0);
// Upload rows given as host CSR arrays (0-based columns).
// Where the device block of an upload comes from: cudaMalloc; the stream-ordered
// allocator (the call then does not wait for the upload: later work on s is
// ordered after it); or the process's reusable row block when it is free.
enum { kAllocPlain = 0, kAllocAsync = 1, kAllocPooled = 2 };
int upload_csr(const long long *rowptr, const int *col, const float *val, int n, int d, DeviceRows &out,
               int force, cudaStream_t s, int alloc = kAllocPlain);
// device bytes of one instance's solver state (gradient, status, shrink lists, Q-row cache)
size_t instance_bytes(int l, double cache_mb);

struct SolveParams;

struct SubProblem {
    std::vector<int> rows;          // row id in DeviceRows per local variable
    std::vector<signed char> y;     // +1 / -1
    std::vector<double> alpha0;     // initial alpha
    std::vector<double> p;          // linear term
    double Cp = 1, Cn = 1;
    int nu = 0;                     // Solver_NU
    const DeviceRows *rows_dev = nullptr;   // the instance's own rows (nullptr: the launch's rows)
    const SolveParams *own = nullptr;       // the instance's own parameters (nullptr: the launch's)
};

struct SolveParams {
    KernelParams kp{2, 3, 0.0, 0.0};
    double eps = 1e-3;
    int shrinking = 1;
    double cache_mb = 100;
    int form = FORM_EXACT;
    int blocks_override = 0;        // 0: heuristic
    int prefetch = 0;               // rows per fill pass; 0: automatic (as many as can be staged)
    int lazy_gbar = -1;             // -1: by form (recomputed for FORM_BF16X3), 0: incremental, 1: recomputed
};

struct SolveResult {
    int fill_path = 0;              // SVMB_FILL_*: how the solve evaluated its kernel rows
    std::vector<double> alpha;      // by local index (unsigned)
    SolveOut out{};
    double seconds = 0;
    int wave = 0;                   // index of the launch (within the call) that solved it
};

// The instances of one persistent launch ("wave"): block counts, shared
// memory, and the layout of the launch's device block and host staging.
struct Wave {
    int first = 0, count = 0, used = 0, form = 0;
    std::vector<int> nb;                      // blocks per instance
    std::vector<std::array<int, 5>> stage;    // stage_cap, stage_lds, tc_n, chunk_cap, hash_slots per instance
    std::vector<int> fill_path;               // SVMB_FILL_* per instance
    size_t dyn_smem = 0;
    struct Layout { size_t G, Gb, A, P, QD, Al, Y, S, PL, PR, Sc, Out, Sync, Part, Tag, Ep, St, Data, bytes; int sets, ways; };
    std::vector<Layout> lay;
    std::vector<size_t> loff, poff, coff, inst_off;
    size_t o_desc = 0, o_bmap = 0, o_alpha = 0, o_p = 0, o_row = 0, o_y = 0, o_out = 0, o_alocal = 0;
    size_t o_zero = 0, o_sync = 0, o_part = 0, o_ep = 0, o_st = 0, o_tag = 0;
    size_t up_bytes = 0, down_bytes = 0, zero_bytes = 0, tag_bytes = 0, dev_bytes = 0;
    char *dev = nullptr, *host = nullptr;
    cudaStream_t stream = nullptr;
    bool cooperative = true;   // false: plain launch (the caller guarantees the blocks are co-resident)
    bool use_graph = false;    // replay a captured graph of the stream work when the layout repeats
    bool drop_last_block = false;   // test hook: launch without the last block (its group's waits run out)
    bool own_events = true;    // the events belong to this wave (not to a cached graph)
    int tune_prefetch = 0;     // autotuner: rows per fill pass for every instance (0: the instances' own)
    int tune_rows_per_block = 500;   // autotuner: positions per block a solve aims at (caps its blocks)
    int tile_bufs = 2;         // transpose tiles per warp of the CUDA-core fills
    int *done_flags = nullptr; // device view of host-mapped words, one per instance (nullptr: none)
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, done = nullptr;
    float ms = 0;
};

// Plan the wave that starts at instance `first` within `capacity` co-resident
// blocks (as many instances before `limit` as fit; limit < 0: up to the end).
// Needs w.dev_bytes of device memory and w.up_bytes + w.down_bytes of
// (preferably page-locked) host staging.
int wave_plan(const DeviceRows &rows, const std::vector<SubProblem> &subs, const SolveParams &prm, int first,
              int capacity, Wave &w, int limit = -1);
// Upload, launch and queue the result download on stream s (asynchronous).
int wave_start(const DeviceRows &rows, const std::vector<SubProblem> &subs, const SolveParams &prm, Wave &w,
               char *dev, char *host, cudaStream_t s);
bool wave_ready(const Wave &w);
// Copy instance k's results (once its done flag is set) with a copy on stream s.
int wave_fetch(const Wave &w, int k, SolveResult &r, cudaStream_t s);
// Wait for the wave and unpack results[first .. first+count).
int wave_finish(Wave &w, std::vector<SolveResult> &res);

// Solve every subproblem in one persistent launch (instances get disjoint
// groups of blocks).  Returns 0 on success.
int solve_batch(const DeviceRows &rows, const std::vector<SubProblem> &subs, const SolveParams &prm,
                std::vector<SolveResult> &res, cudaStream_t s);

// Autotuner of solve_batch (on by default): for each workload signature it
// times the first calls with different fill depths and block targets, then
// keeps the fastest.  Every configuration gives the same results.
void set_autotune(int on);
// the configuration chosen for the last solve_batch call (diagnostics)
void autotune_last(int *prefetch, int *rows_per_block, int *exploring);

int device_sm_count();
void count_launch(long long n = 1);
void count_transfer(long long h2d, long long d2h);
// CUDA graphs of repeated waves in solve_batch (on by default)
void set_graphs(int on);
// bound of every cross-block wait of later launches, in ms (0: the default 30 s)
void set_wait_limit_ms(long long ms);
// Test hook, one shot: the next launch leaves out its last thread block, so
// the group of the launch's last instance never completes an exchange; its
// waits run out after the wait bound, the group returns with an error and
// the call reports it.  The instance must have two or more blocks.
void arm_drop_block();
// solver blocks placed on one SM (1 to 4, default 1): the shared memory a
// block may use is the SM's divided among them; a launch then holds up to
// that many blocks per SM where registers allow it.  Speed only.
int set_blocks_per_sm(int b);
// deepest ring of transpose tiles per warp the CUDA-core fills may use (1 to
// kMaxTileBufs, default 2: deeper rings measured no faster on B200, the rows
// being L2-resident); a launch takes the deepest that still fits its
// instances into one launch.  Results do not depend on it.
int set_fill_depth(int bufs);
int fill_depth();
void graph_counts(long long *captured, long long *replayed);
void transfer_bytes(long long *h2d, long long *d2h);
cudaError_t xfer_async(void *dst, const void *src, size_t bytes, cudaMemcpyKind kind, cudaStream_t s);
cudaError_t xfer(void *dst, const void *src, size_t bytes, cudaMemcpyKind kind);
long long launch_count();

// device-side launchers (smo_kernel.cu)
cudaError_t launch_xsq(const DevX &x, int n, double *out, int form, cudaStream_t s);
cudaError_t launch_scatter_dense(const long long *rowptr, const int *col, const float *val, int n, int ld, float *X,
                                 cudaStream_t s);
int smo_static_smem();
// kernel-matrix blocks (gram_kernel.cu)
cudaError_t launch_split(const DeviceRows &rows, int form, int nchunk, uint16_t *Xs, double *xinv, cudaStream_t s);
cudaError_t launch_kernel_block(const DeviceRows &rows, const KernelParams &kp, int form, const int *d_ia, int ma,
                                const int *d_ib, int nb, double *d_out, long long ldo, int *d_err, cudaStream_t s);
// K(A rows a0 .. a0+ma, B rows 0 .. nb) of two row sets in the same tensor
// form (equal split widths): out[i * ldo + j] = K(a_{a0+i}, b_j), or with
// `trans` out[j * ldo + i]
cudaError_t launch_kernel_block2(const DeviceRows &A, const DeviceRows &B, const KernelParams &kp, int form, int a0,
                                 int ma, int nb, double *d_out, long long ldo, int trans, int *d_err, cudaStream_t s);
cudaError_t launch_smo(int form, const InstanceDesc *d_insts, const int *d_block_inst, int nblocks,
                       size_t dyn_smem, bool cooperative, cudaStream_t s);
cudaError_t smo_max_blocks(int form, size_t dyn_smem, int *blocks_per_sm);

}  // namespace svmb
