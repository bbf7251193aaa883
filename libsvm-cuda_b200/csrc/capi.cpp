// capi.cpp -- the svmb_* C-ABI (include/svm_b200.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "engine.hpp"
#include "predict.hpp"
#include "svm_b200.h"
#include "capi_internal.hpp"
#include "formulation.hpp"

namespace svmb {
int api_set_option(const char *name, long long value);
int api_last_stats(svmb_solve_stats *out, int cap);
}

struct svmb_rows {
    svmb::DeviceRows dev;
};

namespace svmb {
namespace capi {

int check_params(const svmb_params *p)
{
    if (!p) { svmb::set_error("params is NULL"); return -1; }
    if (p->svm_type < C_SVC || p->svm_type > NU_SVR) { svmb::set_error("unknown svm_type"); return -1; }
    if (p->kernel_type < LINEAR || p->kernel_type > SIGMOID) { svmb::set_error("kernel_type must be LINEAR, POLY, RBF or SIGMOID"); return -1; }
    if (p->gamma < 0) { svmb::set_error("gamma < 0"); return -1; }
    if (p->degree < 0) { svmb::set_error("degree of polynomial kernel < 0"); return -1; }
    if (p->eps <= 0) { svmb::set_error("eps <= 0"); return -1; }
    if (p->cache_mb <= 0) { svmb::set_error("cache_size <= 0"); return -1; }
    if (p->svm_type == C_SVC && (p->C_pos <= 0 || p->C_neg <= 0)) { svmb::set_error("C <= 0"); return -1; }
    if ((p->svm_type == EPSILON_SVR || p->svm_type == NU_SVR) && p->C_pos <= 0) { svmb::set_error("C <= 0"); return -1; }
    if ((p->svm_type == NU_SVC || p->svm_type == ONE_CLASS || p->svm_type == NU_SVR) && (p->nu <= 0 || p->nu > 1)) {
        svmb::set_error("nu <= 0 or nu > 1");
        return -1;
    }
    if (p->svm_type == EPSILON_SVR && p->p < 0) { svmb::set_error("p < 0"); return -1; }
    if (p->form < SVMB_FORM_EXACT || p->form > SVMB_FORM_TF32) { svmb::set_error("unknown form"); return -1; }
    if (p->gbar_mode < SVMB_GBAR_AUTO || p->gbar_mode > SVMB_GBAR_RECOMPUTE) { svmb::set_error("unknown gbar_mode"); return -1; }
    return 0;
}

SolveParams to_solve_params(const svmb_params &p)
{
    SolveParams prm;
    prm.kp.type = p.kernel_type;
    prm.kp.degree = p.degree;
    prm.kp.gamma = p.gamma;
    prm.kp.coef0 = p.coef0;
    prm.eps = p.eps;
    prm.shrinking = p.shrinking;
    prm.cache_mb = p.cache_mb;
    prm.form = p.form;
    prm.blocks_override = p.blocks;
    prm.prefetch = p.prefetch;
    prm.lazy_gbar = p.gbar_mode == SVMB_GBAR_INCREMENTAL ? 0 : p.gbar_mode == SVMB_GBAR_RECOMPUTE ? 1 : -1;
    return prm;
}

// the input checks of one instance (sets the error message; no side effects
// otherwise, so instances can be built in parallel once all have passed)
int check_subproblem(const svmb_params &p, int l, const int *rows, const double *y, int nrows)
{
    if (l < 0) { set_error("inst_ptr must be non-decreasing"); return -1; }
    for (int i = 0; i < l; i++)
        if (rows[i] < 0 || rows[i] >= nrows) { set_error("row id out of range"); return -1; }
    if (p.svm_type == NU_SVC) {
        // the feasibility test of svm_check_parameter (svm.cpp:3164-3213)
        int npos = 0, nneg = 0;
        for (int i = 0; i < l; i++) (y[i] > 0 ? npos : nneg)++;
        if (p.nu * l / 2 > std::min(npos, nneg)) { set_error("specified nu is infeasible"); return -1; }
    }
    return 0;
}

// one problem in the reference's formulation of params.svm_type
// (svm.cpp:1500-1699), over the rows with ids rows[0..l)
int make_subproblem(const svmb_params &p, int l, const int *rows, const double *y, int nrows, SubProblem &sp)
{
    if (check_subproblem(p, l, rows, y, nrows) != 0) return -1;
    return formulate(p.svm_type, rows, y, l, p.C_pos, p.C_neg, p.C_pos, p.nu, p.p, sp);
}

// coefficients per point (svm_train_one's decision function: y_i alpha_i,
// nu-SVC / r, SVR alpha_i - alpha*_i) and the statistics of one solve
void finish_instance(const svmb_params &p, const SubProblem &sp, const SolveResult &R, const double *y, int l,
                     double *alpha_out, svmb_solve_stats *stats)
{
    Decision f;
    decide(p.svm_type, sp, R, y, l, f);
    for (int i = 0; i < l; i++) alpha_out[i] = f.coef[i];
    if (!stats) return;
    svmb_solve_stats &st = *stats;
    memset(&st, 0, sizeof st);
    st.iters = R.out.iters;
    st.obj = f.obj;
    st.rho = f.rho;
    st.r = R.out.r;
    st.l = l;
    st.nr_sv = f.nSV;
    st.nr_bsv = f.nBSV;
    st.status = R.out.status;
    st.active_size = R.out.active_size;
    st.seconds = R.seconds;
    st.launch = R.wave;
    st.sum_active = R.out.sum_active;
    st.q_evals = R.out.q_evals;
    st.lookups = R.out.lookups;
    st.hits = R.out.hits;
    st.fills = R.out.fills;
    st.prefetched = R.out.prefetched;
    st.prefetch_used = R.out.prefetch_used;
    for (int q = 0; q < 8; q++) st.prof_cycles[q] = R.out.prof[q];
    st.fill_path = R.fill_path;
    st.fill_targets = R.out.fill_targets;
}

int solve_many(const DeviceRows &rows, int ninst, const int *inst_ptr, const int *inst_rows, const double *inst_y,
               const svmb_params *params, double *alpha_out, svmb_solve_stats *stats)
{
    if (ninst <= 0) return 0;
    for (int k = 0; k < ninst; k++) {
        if (check_params(&params[k])) return -1;
        if (params[k].form != params[0].form) {
            set_error("instances of one launch must share the arithmetic form");
            return -1;
        }
    }
    // every instance carries its own parameters (kernel, C, eps, cache, ...);
    // only the arithmetic form is common to a launch
    for (int k = 0; k < ninst; k++)
        if (check_subproblem(params[k], inst_ptr[k + 1] - inst_ptr[k], inst_rows + inst_ptr[k], inst_y + inst_ptr[k],
                             rows.n) != 0)
            return -1;
    // the instances are independent: built, and their results decoded, on all
    // host threads (formulate fails only for an svm_type that check_params
    // already rejected)
    std::vector<SolveParams> own(ninst);
    std::vector<SubProblem> subs(ninst);
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(| : bad) if (ninst > 1)
    for (int k = 0; k < ninst; k++) {
        const int a = inst_ptr[k], b = inst_ptr[k + 1];
        bad |= formulate(params[k].svm_type, inst_rows + a, inst_y + a, b - a, params[k].C_pos, params[k].C_neg,
                         params[k].C_pos, params[k].nu, params[k].p, subs[k]) != 0;
        own[k] = to_solve_params(params[k]);
        subs[k].own = &own[k];
    }
    if (bad) { set_error("unknown svm_type"); return -1; }
    std::vector<SolveResult> res;
    if (solve_batch(rows, subs, own[0], res, 0) != 0) return -1;
#pragma omp parallel for schedule(dynamic, 1) if (ninst > 1)
    for (int k = 0; k < ninst; k++)
        finish_instance(params[k], subs[k], res[k], inst_y + inst_ptr[k], inst_ptr[k + 1] - inst_ptr[k],
                        alpha_out + inst_ptr[k], stats ? &stats[k] : nullptr);
    return 0;
}

}  // namespace capi
}  // namespace svmb

using svmb::capi::check_params;
using svmb::capi::solve_many;

extern "C" {

const char *svmb_last_error(void) { return svmb::last_error(); }
long long svmb_kernel_launches(void) { return svmb::launch_count(); }
void svmb_transfer_bytes(long long *h2d, long long *d2h) { svmb::transfer_bytes(h2d, d2h); }
int svmb_version(void) { return LIBSVM_VERSION * 100 + 1; }

int svmb_device_available(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n > 0 ? 1 : 0;
}

int svmb_set_option(const char *name, long long value)
{
    if (!name || svmb::api_set_option(name, value) != 0) {
        svmb::set_error("unknown option or value");
        return -1;
    }
    return 0;
}

int svmb_last_train_stats(svmb_solve_stats *out, int cap) { return svmb::api_last_stats(out, cap); }

int svmb_predict_batch(const struct svm_model *model, const struct svm_node *const *rows, int n, double *labels,
                       double *dec_values)
{
    if (!model || (n > 0 && (!rows || !labels))) {
        svmb::set_error("NULL argument");
        return -1;
    }
    return svmb::predict_batch(model, rows, n, labels, dec_values);
}

int svmb_rows_upload_csr(int n, int d, const long long *rowptr, const int *col, const float *val, int layout,
                         svmb_rows **out)
{
    if (!out || n < 0 || d < 0 || (n > 0 && !rowptr)) {
        svmb::set_error("invalid rows");
        return -1;
    }
    for (int r = 0; r < n; r++)
        if (rowptr[r + 1] < rowptr[r]) { svmb::set_error("rowptr must be non-decreasing"); return -1; }
    for (long long e = 0; e < (n ? rowptr[n] : 0); e++)
        if (col[e] < 0 || col[e] >= d) { svmb::set_error("column index out of range"); return -1; }
    std::unique_ptr<svmb_rows> h(new svmb_rows());
    if (svmb::upload_csr(rowptr, col, val, n, d, h->dev, layout, 0) != 0) return -1;
    *out = h.release();
    return 0;
}

int svmb_rows_info(const svmb_rows *rows, int *n, int *d, int *dense, long long *bytes)
{
    if (!rows) { svmb::set_error("NULL rows"); return -1; }
    if (n) *n = rows->dev.n;
    if (d) *d = rows->dev.d;
    if (dense) *dense = rows->dev.dense ? 1 : 0;
    if (bytes) *bytes = (long long)rows->dev.bytes;
    return 0;
}

int svmb_rows_solve_many(const svmb_rows *rows, int ninst, const int *inst_ptr, const int *inst_rows, const double *inst_y,
                         const svmb_params *params, double *alpha_out, svmb_solve_stats *stats)
{
    if (!rows) { svmb::set_error("NULL rows"); return -1; }
    return solve_many(rows->dev, ninst, inst_ptr, inst_rows, inst_y, params, alpha_out, stats);
}

void svmb_rows_free(svmb_rows *rows) { delete rows; }

void svmb_autotune_last(int *prefetch, int *rows_per_block, int *exploring)
{
    svmb::autotune_last(prefetch, rows_per_block, exploring);
}

void svmb_graph_counts(long long *captured, long long *replayed) { svmb::graph_counts(captured, replayed); }

int svmb_rows_kernel_block(const svmb_rows *rows, const svmb_params *params, int ma, const int *ia, int nb,
                           const int *ib, double *out)
{
    if (!rows || !params || ma < 0 || nb < 0 || (ma && (!ia || !out)) || (nb && !ib)) {
        svmb::set_error("invalid arguments");
        return -1;
    }
    if (params->kernel_type < LINEAR || params->kernel_type > SIGMOID) { svmb::set_error("kernel_type must be LINEAR, POLY, RBF or SIGMOID"); return -1; }
    if (params->form < SVMB_FORM_EXACT || params->form > SVMB_FORM_TF32) { svmb::set_error("unknown form"); return -1; }
    const int n = rows->dev.n;
    for (int i = 0; i < ma; i++)
        if (ia[i] < 0 || ia[i] >= n) { svmb::set_error("row index out of range"); return -1; }
    for (int j = 0; j < nb; j++)
        if (ib[j] < 0 || ib[j] >= n) { svmb::set_error("row index out of range"); return -1; }
    if (ma == 0 || nb == 0) return 0;
    svmb::DeviceRows &dev = const_cast<svmb::DeviceRows &>(rows->dev);
    if (dev.prepare_form(params->form, 0) != 0) return -1;
    svmb::KernelParams kp{params->kernel_type, params->degree, params->gamma, params->coef0};
    int *d_ia = nullptr, *d_ib = nullptr, *d_err = nullptr;
    double *d_out = nullptr;
    int herr = 0;
    cudaError_t e = cudaMalloc(&d_ia, sizeof(int) * (size_t)ma);
    if (e == cudaSuccess) e = cudaMalloc(&d_ib, sizeof(int) * (size_t)nb);
    if (e == cudaSuccess) e = cudaMalloc(&d_err, sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&d_out, sizeof(double) * (size_t)ma * nb);
    if (e == cudaSuccess) e = svmb::xfer(d_ia, ia, sizeof(int) * (size_t)ma, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = svmb::xfer(d_ib, ib, sizeof(int) * (size_t)nb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(d_err, 0, sizeof(int));
    if (e == cudaSuccess) e = svmb::launch_kernel_block(dev, kp, params->form, d_ia, ma, d_ib, nb, d_out, nb, d_err, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = svmb::xfer(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = svmb::xfer(out, d_out, sizeof(double) * (size_t)ma * nb, cudaMemcpyDeviceToHost);
    cudaFree(d_ia); cudaFree(d_ib); cudaFree(d_err); cudaFree(d_out);
    if (e != cudaSuccess) {
        svmb::set_error(std::string("kernel block: ") + cudaGetErrorString(e));
        return -1;
    }
    if (herr) {
        svmb::set_error("kernel block: a tensor-core wait timed out");
        return -1;
    }
    return 0;
}

int svmb_solve_many_csr(int n, int d, const long long *rowptr, const int *col, const float *val, int ninst,
                        const int *inst_ptr, const int *inst_rows, const double *inst_y, const svmb_params *params,
                        double *alpha_out, svmb_solve_stats *stats)
{
    svmb_rows *rows = nullptr;
    if (svmb_rows_upload_csr(n, d, rowptr, col, val, -1, &rows) != 0) return -1;
    const int rc = solve_many(rows->dev, ninst, inst_ptr, inst_rows, inst_y, params, alpha_out, stats);
    svmb_rows_free(rows);
    return rc;
}

int svmb_solve_binary_csr(int n, int d, const long long *rowptr, const int *col, const float *val, const double *y,
                          const svmb_params *params, double *alpha_out, svmb_solve_stats *stats)
{
    std::vector<int> ptr = {0, n};
    std::vector<int> idx(n);
    for (int i = 0; i < n; i++) idx[i] = i;
    return svmb_solve_many_csr(n, d, rowptr, col, val, 1, ptr.data(), idx.data(), y, params, alpha_out, stats);
}

}  // extern "C"
