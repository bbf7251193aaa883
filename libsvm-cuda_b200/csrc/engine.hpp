// engine.hpp -- host-side interface of the device solver (C++, internal).
#pragma once
#include <cuda_runtime.h>

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
    ~DeviceRows();
    DevX view(int form) const;
    // build Xs if the form needs it; -1 (error set) when the rows cannot take the form
    int prepare_form(int form, cudaStream_t s);
};

// Upload rows given as libsvm svm_node lists (index >= 1, terminated by -1).
// force: -1 auto, 0 CSR, 1 dense.
int upload_rows(const svm_node *const *x, int n, DeviceRows &out, int force, cudaStream_t s);
// Upload rows given as host CSR arrays (0-based columns).
int upload_csr(const long long *rowptr, const int *col, const float *val, int n, int d, DeviceRows &out,
               int force, cudaStream_t s);

struct SubProblem {
    std::vector<int> rows;          // row id in DeviceRows per local variable
    std::vector<signed char> y;     // +1 / -1
    std::vector<double> alpha0;     // initial alpha
    std::vector<double> p;          // linear term
    double Cp = 1, Cn = 1;
    int nu = 0;                     // Solver_NU
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
    std::vector<double> alpha;      // by local index (unsigned)
    SolveOut out{};
    double seconds = 0;
};

// Solve every subproblem in one persistent launch (instances get disjoint
// groups of blocks).  Returns 0 on success.
int solve_batch(const DeviceRows &rows, const std::vector<SubProblem> &subs, const SolveParams &prm,
                std::vector<SolveResult> &res, cudaStream_t s);

int device_sm_count();
void count_launch(long long n = 1);
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
cudaError_t launch_smo(int form, const InstanceDesc *d_insts, const int *d_block_inst, int nblocks,
                       size_t dyn_smem, bool cooperative, cudaStream_t s);
cudaError_t smo_max_blocks(int form, size_t dyn_smem, int *blocks_per_sm);

}  // namespace svmb
