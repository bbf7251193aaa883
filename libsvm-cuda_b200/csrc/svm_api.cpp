// svm_api.cpp -- the drop-in svm.h API (include/svm.h) on top of the device engine.
//
// Behaviour follows the reference's libsvm/svm.cpp interface functions
// (svm_train :2159-2404, svm_cross_validation :2407-2525, svm_predict* :2569-2697,
// model I/O :2699-3044, svm_check_parameter :3097-3216).  Differences:
//   * every binary subproblem of one svm_train call (all one-vs-one pairs)
//     is solved in ONE persistent device launch instead of one after another;
//   * decision values are computed on the device (predict_kernel.cu);
//   * errors never exit() the process: svm_train returns NULL and the reason is
//     available from svmb_last_error() and through the print hook.
// Only C-SVC and nu-SVC are trained on the device; the other svm_types are
// rejected with an error (svm_train returns NULL).
#include <algorithm>
#include <clocale>
#include <cmath>
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "engine.hpp"
#include "predict.hpp"
#include "svm.h"
#include "svm_b200.h"

extern "C" {
int libsvm_version = LIBSVM_VERSION;
}

namespace svmb {
int api_force_layout();
}

namespace {

void print_string_stdout(const char *s)
{
    fputs(s, stdout);
    fflush(stdout);
}
void (*svm_print_string)(const char *) = &print_string_stdout;

void info(const char *fmt, ...)
{
    char buf[8192];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    (*svm_print_string)(buf);
}

// the text of one info() call kept as one entry of `out` (printed later, in
// order, one print-hook call per entry as the reference makes them)
void info_to(std::vector<std::string> &out, const char *fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    out.emplace_back(buf);
}

// engine options settable through svmb_set_option (process wide)
struct Options {
    int form = svmb::FORM_EXACT;
    int blocks = 0;
    int force_layout = -1;
    int prefetch = 0;
} g_opt;

// statistics of the last svm_train call (svmb_last_train_stats)
std::vector<svmb_solve_stats> g_last_stats;
std::mutex g_stats_mu;

// Labels in first-occurrence order; -1/+1 with -1 first are swapped so that
// +1 is class 0 (reference svm.cpp:2081-2154).
void group_classes(const svm_problem *prob, int *nr_class_ret, std::vector<int> &label, std::vector<int> &start,
                   std::vector<int> &count, std::vector<int> &perm)
{
    const int l = prob->l;
    label.clear();
    count.clear();
    std::vector<int> data_label(l);
    for (int i = 0; i < l; i++) {
        const int this_label = (int)prob->y[i];
        int j;
        for (j = 0; j < (int)label.size(); j++)
            if (this_label == label[j]) {
                ++count[j];
                break;
            }
        data_label[i] = j;
        if (j == (int)label.size()) {
            label.push_back(this_label);
            count.push_back(1);
        }
    }
    const int nr_class = (int)label.size();
    if (nr_class == 2 && label[0] == -1 && label[1] == 1) {
        std::swap(label[0], label[1]);
        std::swap(count[0], count[1]);
        for (int i = 0; i < l; i++) data_label[i] = data_label[i] == 0 ? 1 : 0;
    }
    start.assign(nr_class, 0);
    for (int i = 1; i < nr_class; i++) start[i] = start[i - 1] + count[i - 1];
    perm.assign(l, 0);
    std::vector<int> fill = start;
    for (int i = 0; i < l; i++) perm[fill[data_label[i]]++] = i;
    *nr_class_ret = nr_class;
}

// One binary subproblem in the form the formulations build it
// (solve_c_svc svm.cpp:1500-1533, solve_nu_svc :1535-1588).
svmb::SubProblem make_sub(const std::vector<int> &rows, const std::vector<signed char> &y, const svm_parameter *param,
                          double Cp, double Cn)
{
    svmb::SubProblem sp;
    const int l = (int)rows.size();
    sp.rows = rows;
    sp.y = y;
    sp.alpha0.assign(l, 0.0);
    sp.p.assign(l, 0.0);
    if (param->svm_type == NU_SVC) {
        const double nu = param->nu;
        double sum_pos = nu * l / 2, sum_neg = nu * l / 2;
        for (int i = 0; i < l; i++) {
            if (y[i] == +1) {
                sp.alpha0[i] = std::min(1.0, sum_pos);
                sum_pos -= sp.alpha0[i];
            } else {
                sp.alpha0[i] = std::min(1.0, sum_neg);
                sum_neg -= sp.alpha0[i];
            }
        }
        sp.nu = 1;
        sp.Cp = 1.0;
        sp.Cn = 1.0;
    } else {
        for (int i = 0; i < l; i++) sp.p[i] = -1;
        sp.nu = 0;
        sp.Cp = Cp;
        sp.Cn = Cn;
    }
    return sp;
}

svmb::SolveParams make_solve_params(const svm_parameter *param)
{
    svmb::SolveParams prm;
    prm.kp.type = param->kernel_type;
    prm.kp.degree = param->degree;
    prm.kp.gamma = param->gamma;
    prm.kp.coef0 = param->coef0;
    prm.eps = param->eps;
    prm.shrinking = param->shrinking;
    prm.cache_mb = param->cache_size;
    prm.form = g_opt.form;
    prm.blocks_override = g_opt.blocks;
    prm.prefetch = g_opt.prefetch;
    return prm;
}

struct DecisionFunction {
    std::vector<double> alpha;   // signed coefficients
    double rho = 0;
};

// Post-processing of one solve (svm.cpp:1517-1532, :1572-1587 and svm_train_one :1739-1766).
// One subproblem's decision function and statistics; its messages go to
// `log` (the caller prints the logs of all pairs in pair order).
DecisionFunction finish_solve(const svmb::SubProblem &sp, const svmb::SolveResult &R, const svm_parameter *param,
                              const double *yvals, std::vector<std::string> &log, svmb_solve_stats &st)
{
    DecisionFunction f;
    const int l = (int)sp.rows.size();
    f.alpha = R.alpha;
    double rho = R.out.rho, obj = R.out.obj;
    double upper_p, upper_n;
    info_to(log, "\noptimization finished, #iter = %lld\n", R.out.iters);
    // (the max_iter warning goes to stderr from the caller, in pair order)
    if (sp.nu) {
        const double r = R.out.r;
        info_to(log, "C = %f\n", 1 / r);
        for (int i = 0; i < l; i++) f.alpha[i] *= sp.y[i] / r;
        rho /= r;
        obj /= (r * r);
        upper_p = upper_n = 1 / r;
    } else {
        double sum_alpha = 0;
        for (int i = 0; i < l; i++) sum_alpha += f.alpha[i];
        if (sp.Cp == sp.Cn) info_to(log, "nu = %f\n", sum_alpha / (sp.Cp * l));
        for (int i = 0; i < l; i++) f.alpha[i] *= sp.y[i];
        upper_p = sp.Cp;
        upper_n = sp.Cn;
    }
    f.rho = rho;
    info_to(log, "obj = %f, rho = %f\n", obj, rho);
    int nSV = 0, nBSV = 0;
    for (int i = 0; i < l; i++) {
        if (fabs(f.alpha[i]) > 0) {
            ++nSV;
            if (yvals[i] > 0) {
                if (fabs(f.alpha[i]) >= upper_p) ++nBSV;
            } else {
                if (fabs(f.alpha[i]) >= upper_n) ++nBSV;
            }
        }
    }
    info_to(log, "nSV = %d, nBSV = %d\n", nSV, nBSV);
    memset(&st, 0, sizeof st);
    st.iters = R.out.iters;
    st.obj = obj;
    st.rho = rho;
    st.r = R.out.r;
    st.l = l;
    st.nr_sv = nSV;
    st.nr_bsv = nBSV;
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
    return f;
}

bool svm_type_supported(int t) { return t == C_SVC || t == NU_SVC; }

bool train_supported(const svm_parameter *param)
{
    if (!svm_type_supported(param->svm_type) || param->kernel_type == PRECOMPUTED) {
        svmb::set_error("only C_SVC and NU_SVC with linear/poly/rbf/sigmoid kernels are trained on the GPU");
        info("ERROR: %s\n", svmb::last_error());
        return false;
    }
    return true;
}

// One svm_train call (reference svm.cpp:2159-2404) split into its one-vs-one
// subproblems -- which address the rows of an uploaded row set by id -- and
// the model assembly from their solutions, so that the subproblems of many
// trainings (CV folds, grid points) can share one batched solve.
struct TrainJob {
    const svm_problem *prob = nullptr;
    svm_parameter param{};
    int l = 0, nr_class = 0;
    std::vector<int> label, start, count, perm;
    std::vector<svm_node *> x;                 // rows in grouped order
    std::vector<svmb::SubProblem> subs;
    std::vector<std::vector<double>> subys;
    svmb::SolveParams own;                     // solve parameters of this training
};

// row_id[i]: id of prob row i in the uploaded row set (nullptr: rows uploaded in grouped order)
void setup_train(const svm_problem *prob, const svm_parameter *param, const int *row_id, TrainJob &tj)
{
    tj.prob = prob;
    tj.param = *param;
    tj.l = prob->l;
    group_classes(prob, &tj.nr_class, tj.label, tj.start, tj.count, tj.perm);
    const int nr_class = tj.nr_class;
    if (nr_class == 1) info("WARNING: training data in only one class. See README for details.\n");
    tj.x.resize(tj.l);
    for (int i = 0; i < tj.l; i++) tj.x[i] = prob->x[tj.perm[i]];
    std::vector<double> weighted_C(nr_class, param->C);
    for (int i = 0; i < param->nr_weight; i++) {
        int j;
        for (j = 0; j < nr_class; j++)
            if (param->weight_label[i] == tj.label[j]) break;
        if (j == nr_class)
            fprintf(stderr, "WARNING: class label %d specified in weight is not found\n", param->weight_label[i]);
        else
            weighted_C[j] *= param->weight[i];
    }
    auto id = [&](int g) { return row_id ? row_id[tj.perm[g]] : g; };   // grouped index -> uploaded row id
    // the one-vs-one subproblems in pair order (class i rows +1, then class j
    // rows -1), built in parallel: they are independent
    std::vector<std::pair<int, int>> pairs;
    for (int i = 0; i < nr_class; i++)
        for (int j = i + 1; j < nr_class; j++) pairs.emplace_back(i, j);
    const size_t first = tj.subs.size();
    tj.subs.resize(first + pairs.size());
    tj.subys.resize(first + pairs.size());
#pragma omp parallel for schedule(dynamic, 1)
    for (int q = 0; q < (int)pairs.size(); q++) {
        const int i = pairs[q].first, j = pairs[q].second;
        const int n = tj.count[i] + tj.count[j];
        std::vector<int> r(n);
        std::vector<signed char> y(n);
        std::vector<double> yv(n);
        for (int k = 0; k < tj.count[i]; k++) { r[k] = id(tj.start[i] + k); y[k] = +1; yv[k] = +1; }
        for (int k = 0; k < tj.count[j]; k++) {
            r[tj.count[i] + k] = id(tj.start[j] + k);
            y[tj.count[i] + k] = -1;
            yv[tj.count[i] + k] = -1;
        }
        tj.subs[first + q] = make_sub(r, y, param, weighted_C[i], weighted_C[j]);
        tj.subys[first + q] = std::move(yv);
    }
    tj.own = make_solve_params(param);
}

// model assembly (reference svm.cpp:2297-2386) from the solutions res[first ..]
svm_model *assemble_model(const TrainJob &tj, const std::vector<svmb::SolveResult> &res, size_t first)
{
    const svm_parameter *param = &tj.param;
    const int l = tj.l, nr_class = tj.nr_class;
    const std::vector<int> &start = tj.start, &count = tj.count;
    std::vector<DecisionFunction> f(tj.subs.size());
    // the pairs' decision functions in parallel; their messages, warnings and
    // statistics then in pair order
    std::vector<std::vector<std::string>> logs(tj.subs.size());
    std::vector<svmb_solve_stats> sts(tj.subs.size());
#pragma omp parallel for schedule(dynamic, 1)
    for (int p = 0; p < (int)tj.subs.size(); p++)
        f[p] = finish_solve(tj.subs[p], res[first + p], param, tj.subys[p].data(), logs[p], sts[p]);
    for (size_t p = 0; p < tj.subs.size(); p++) {
        // the solver's max_iter warning precedes its "optimization finished" line (svm.cpp:779-787)
        if (res[first + p].out.status == 1) fprintf(stderr, "\nWARNING: reaching max number of iterations\n");
        for (const std::string &line : logs[p]) (*svm_print_string)(line.c_str());
        std::lock_guard<std::mutex> g(g_stats_mu);
        g_last_stats.push_back(sts[p]);
    }
    svm_model *model = (svm_model *)malloc(sizeof(svm_model));
    model->param = *param;
    model->free_sv = 0;
    model->nr_class = nr_class;
    model->label = (int *)malloc(sizeof(int) * std::max(nr_class, 1));
    for (int i = 0; i < nr_class; i++) model->label[i] = tj.label[i];
    const int npair = nr_class * (nr_class - 1) / 2;
    model->rho = (double *)malloc(sizeof(double) * std::max(npair, 1));
    for (int i = 0; i < npair; i++) model->rho[i] = f[i].rho;
    model->probA = NULL;
    model->probB = NULL;
    std::vector<char> nonzero(l, 0);
    {
        int p = 0;
        for (int i = 0; i < nr_class; i++)
            for (int j = i + 1; j < nr_class; j++) {
                for (int k = 0; k < count[i]; k++)
                    if (fabs(f[p].alpha[k]) > 0) nonzero[start[i] + k] = 1;
                for (int k = 0; k < count[j]; k++)
                    if (fabs(f[p].alpha[count[i] + k]) > 0) nonzero[start[j] + k] = 1;
                ++p;
            }
    }
    int total_sv = 0;
    std::vector<int> nz_count(nr_class);
    model->nSV = (int *)malloc(sizeof(int) * std::max(nr_class, 1));
    for (int i = 0; i < nr_class; i++) {
        int nSV = 0;
        for (int j = 0; j < count[i]; j++)
            if (nonzero[start[i] + j]) { ++nSV; ++total_sv; }
        model->nSV[i] = nSV;
        nz_count[i] = nSV;
    }
    info("Total nSV = %d\n", total_sv);
    model->l = total_sv;
    model->SV = (svm_node **)malloc(sizeof(svm_node *) * std::max(total_sv, 1));
    model->sv_indices = (int *)malloc(sizeof(int) * std::max(total_sv, 1));
    {
        int p = 0;
        for (int i = 0; i < l; i++)
            if (nonzero[i]) {
                model->SV[p] = tj.x[i];
                model->sv_indices[p++] = tj.perm[i] + 1;
            }
    }
    std::vector<int> nz_start(nr_class, 0);
    for (int i = 1; i < nr_class; i++) nz_start[i] = nz_start[i - 1] + nz_count[i - 1];
    model->sv_coef = (double **)malloc(sizeof(double *) * std::max(nr_class - 1, 1));
    for (int i = 0; i < nr_class - 1; i++) model->sv_coef[i] = (double *)malloc(sizeof(double) * std::max(total_sv, 1));
    {
        int p = 0;
        for (int i = 0; i < nr_class; i++)
            for (int j = i + 1; j < nr_class; j++) {
                int q = nz_start[i];
                for (int k = 0; k < count[i]; k++)
                    if (nonzero[start[i] + k]) model->sv_coef[j - 1][q++] = f[p].alpha[k];
                q = nz_start[j];
                for (int k = 0; k < count[j]; k++)
                    if (nonzero[start[j] + k]) model->sv_coef[i][q++] = f[p].alpha[count[i] + k];
                ++p;
            }
    }
    return model;
}

// Stratified k-fold cross-validation (reference svm.cpp:2407-2525) over a grid
// of (C, gamma) points: one fold assignment with the C library rand(), as the
// reference draws it, then every point's and fold's one-vs-one subproblems are
// solved in batched launches over the rows uploaded once.  target[p*l + i] is
// the prediction of row i by the model of point p trained without i's fold.
int cross_validation_grid(const svm_problem *prob, const svm_parameter *param, int nr_fold, int npoints,
                          const double *Cs, const double *gammas, double *target)
{
    {
        std::lock_guard<std::mutex> g(g_stats_mu);
        g_last_stats.clear();
    }
    const int l = prob->l;
    std::vector<int> perm(l);
    if (nr_fold > l) {
        nr_fold = l;
        fprintf(stderr, "WARNING: # folds > # data. Will use # folds = # data instead (i.e., leave-one-out cross validation)\n");
    }
    std::vector<int> fold_start(nr_fold + 1);
    if ((param->svm_type == C_SVC || param->svm_type == NU_SVC) && nr_fold < l) {
        int nr_class;
        std::vector<int> label, start, count;
        group_classes(prob, &nr_class, label, start, count, perm);
        std::vector<int> fold_count(nr_fold), index(perm);
        // stratified shuffle with the C library rand(), as the reference (svm.cpp:2436-2442)
        for (int c = 0; c < nr_class; c++)
            for (int i = 0; i < count[c]; i++) {
                const int j = i + rand() % (count[c] - i);
                std::swap(index[start[c] + j], index[start[c] + i]);
            }
        for (int i = 0; i < nr_fold; i++) {
            fold_count[i] = 0;
            for (int c = 0; c < nr_class; c++) fold_count[i] += (i + 1) * count[c] / nr_fold - i * count[c] / nr_fold;
        }
        fold_start[0] = 0;
        for (int i = 1; i <= nr_fold; i++) fold_start[i] = fold_start[i - 1] + fold_count[i - 1];
        for (int c = 0; c < nr_class; c++)
            for (int i = 0; i < nr_fold; i++) {
                const int begin = start[c] + i * count[c] / nr_fold;
                const int end = start[c] + (i + 1) * count[c] / nr_fold;
                for (int j = begin; j < end; j++) perm[fold_start[i]++] = index[j];
            }
        fold_start[0] = 0;
        for (int i = 1; i <= nr_fold; i++) fold_start[i] = fold_start[i - 1] + fold_count[i - 1];
    } else {
        for (int i = 0; i < l; i++) perm[i] = i;
        for (int i = 0; i < l; i++) {
            const int j = i + rand() % (l - i);
            std::swap(perm[i], perm[j]);
        }
        for (int i = 0; i <= nr_fold; i++) fold_start[i] = i * l / nr_fold;
    }
    for (long long k = 0; k < (long long)npoints * l; k++) target[k] = NAN;
    if (!train_supported(param)) return -1;
    const bool trace = getenv("SVMB_TRACE") && *getenv("SVMB_TRACE") == '1';
    const auto c0 = std::chrono::steady_clock::now();
    auto since = [&](std::chrono::steady_clock::time_point a) {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - a).count();
    };
    // all rows once, in the problem's order (row id = index in prob)
    svmb::DeviceRows rows;
    if (l > 0 && svmb::upload_rows(prob->x, l, rows, svmb::api_force_layout(), 0, svmb::kAllocPooled) != 0) {
        info("ERROR: %s\n", svmb::last_error());
        return -1;
    }
    // the training set of every fold, its row ids, and one training per (point, fold)
    std::vector<svm_problem> fold_prob(nr_fold);
    std::vector<std::vector<svm_node *>> fold_x(nr_fold);
    std::vector<std::vector<double>> fold_y(nr_fold);
    std::vector<std::vector<int>> fold_id(nr_fold);
    for (int i = 0; i < nr_fold; i++) {
        const int begin = fold_start[i], end = fold_start[i + 1];
        for (int j = 0; j < l; j++) {
            if (j >= begin && j < end) continue;
            fold_x[i].push_back(prob->x[perm[j]]);
            fold_y[i].push_back(prob->y[perm[j]]);
            fold_id[i].push_back(perm[j]);
        }
        fold_prob[i].l = (int)fold_x[i].size();
        fold_prob[i].x = fold_x[i].data();
        fold_prob[i].y = fold_y[i].data();
    }
    std::vector<svm_parameter> pparam(npoints, *param);
    std::vector<TrainJob> jobs((size_t)npoints * nr_fold);
    std::vector<svmb::SubProblem> all;
    std::vector<size_t> first(jobs.size());
    for (int q = 0; q < npoints; q++) {
        pparam[q].C = Cs[q];
        pparam[q].gamma = gammas[q];
        for (int i = 0; i < nr_fold; i++) {
            TrainJob &tj = jobs[(size_t)q * nr_fold + i];
            setup_train(&fold_prob[i], &pparam[q], fold_id[i].data(), tj);
        }
    }
    for (size_t k = 0; k < jobs.size(); k++) {
        first[k] = all.size();
        for (svmb::SubProblem &sp : jobs[k].subs) {
            sp.own = &jobs[k].own;
            all.push_back(sp);
        }
    }
    std::vector<svmb::SolveResult> res;
    {
        std::lock_guard<std::mutex> g(g_stats_mu);
        g_last_stats.clear();
    }
    const double t_setup = since(c0);
    const auto c1 = std::chrono::steady_clock::now();
    if (!all.empty() && svmb::solve_batch(rows, all, jobs[0].own, res, 0) != 0) {
        info("ERROR: %s\n", svmb::last_error());
        return -1;
    }
    const double t_solve = since(c1);
    const auto c2 = std::chrono::steady_clock::now();
    for (int q = 0; q < npoints; q++)
        for (int i = 0; i < nr_fold; i++) {
            const size_t k = (size_t)q * nr_fold + i;
            svm_model *m = assemble_model(jobs[k], res, first[k]);
            const int begin = fold_start[i], end = fold_start[i + 1];
            std::vector<const svm_node *> held;
            for (int j = begin; j < end; j++) held.push_back(prob->x[perm[j]]);
            std::vector<double> lab(held.size());
            if (held.empty() || svmb::predict_batch(m, held.data(), (int)held.size(), lab.data(), nullptr) == 0)
                for (int j = begin; j < end; j++) target[(size_t)q * l + perm[j]] = lab[j - begin];
            svm_free_and_destroy_model(&m);
        }
    if (trace)
        fprintf(stderr, "[svmb] cv_grid points=%d folds=%d subproblems=%zu setup=%.2fms solve=%.2fms predict=%.2fms\n", npoints,
                nr_fold, all.size(), t_setup, t_solve, since(c2));
    return 0;
}


}  // namespace

namespace svmb {
int api_set_option(const char *name, long long value)
{
    if (!strcmp(name, "form")) {
        if (value != FORM_EXACT && value != FORM_FP32 && value != FORM_BF16X3 && value != FORM_FP16X3) return -1;
        g_opt.form = (int)value;
    } else if (!strcmp(name, "blocks")) {
        g_opt.blocks = (int)value;
    } else if (!strcmp(name, "layout")) {
        g_opt.force_layout = (int)value;
    } else if (!strcmp(name, "graphs")) {
        set_graphs((int)value);
    } else if (!strcmp(name, "autotune")) {
        set_autotune((int)value);
    } else if (!strcmp(name, "fill_depth")) {
        if (set_fill_depth((int)value) != 0) return -1;
    } else if (!strcmp(name, "predict_form")) {
        if (predict_set_form((int)value) != 0) return -1;
    } else if (!strcmp(name, "prefetch")) {
        if (value < 0 || value > kPrefetchMax) return -1;
        g_opt.prefetch = (int)value;
    } else {
        return -1;
    }
    return 0;
}
int api_last_stats(svmb_solve_stats *out, int cap)
{
    std::lock_guard<std::mutex> g(g_stats_mu);
    const int n = (int)g_last_stats.size();
    for (int k = 0; k < n && k < cap; k++) out[k] = g_last_stats[k];
    return n;
}
void api_print(const char *s) { (*svm_print_string)(s); }
int api_force_layout() { return g_opt.force_layout; }
}  // namespace svmb

extern "C" {

struct svm_model *svm_train(const struct svm_problem *prob, const struct svm_parameter *param)
{
    {
        std::lock_guard<std::mutex> g(g_stats_mu);
        g_last_stats.clear();
    }
    if (!train_supported(param)) return NULL;
    const auto t0 = std::chrono::steady_clock::now();
    TrainJob tj;
    setup_train(prob, param, nullptr, tj);
    const auto t1 = std::chrono::steady_clock::now();
    // rows are uploaded once, in grouped order; every pair addresses them by id
    svmb::DeviceRows rows;
    if (tj.l > 0 && svmb::upload_rows(tj.x.data(), tj.l, rows, svmb::api_force_layout(), 0, svmb::kAllocPooled) != 0) {
        info("ERROR: %s\n", svmb::last_error());
        return NULL;
    }
    const auto t2 = std::chrono::steady_clock::now();
    std::vector<svmb::SolveResult> res;
    if (!tj.subs.empty() && svmb::solve_batch(rows, tj.subs, make_solve_params(param), res, 0) != 0) {
        info("ERROR: %s\n", svmb::last_error());
        return NULL;
    }
    const auto t3 = std::chrono::steady_clock::now();
    svm_model *model = assemble_model(tj, res, 0);
    if (getenv("SVMB_TRACE") && *getenv("SVMB_TRACE") == '1') {
        const auto t4 = std::chrono::steady_clock::now();
        auto ms = [](std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
            return std::chrono::duration<double, std::milli>(b - a).count();
        };
        fprintf(stderr, "[svmb] svm_train setup=%.2fms upload=%.2fms solve=%.2fms assemble=%.2fms\n", ms(t0, t1), ms(t1, t2),
                ms(t2, t3), ms(t3, t4));
    }
    return model;
}

void svm_cross_validation(const struct svm_problem *prob, const struct svm_parameter *param, int nr_fold, double *target)
{
    const double C1[1] = {param->C}, G1[1] = {param->gamma};
    cross_validation_grid(prob, param, nr_fold, 1, C1, G1, target);
}

int svmb_cross_validation_grid(const struct svm_problem *prob, const struct svm_parameter *param, int nr_fold,
                               int npoints, const double *C, const double *gamma, double *target)
{
    if (!prob || !param || !C || !gamma || !target || npoints <= 0 || nr_fold < 2) {
        svmb::set_error("invalid arguments");
        return -1;
    }
    return cross_validation_grid(prob, param, nr_fold, npoints, C, gamma, target);
}

int svm_get_svm_type(const svm_model *model) { return model->param.svm_type; }
int svm_get_nr_class(const svm_model *model) { return model->nr_class; }

void svm_get_labels(const svm_model *model, int *label)
{
    if (model->label != NULL)
        for (int i = 0; i < model->nr_class; i++) label[i] = model->label[i];
}

void svm_get_sv_indices(const svm_model *model, int *indices)
{
    if (model->sv_indices != NULL)
        for (int i = 0; i < model->l; i++) indices[i] = model->sv_indices[i];
}

int svm_get_nr_sv(const svm_model *model) { return model->l; }

double svm_get_svr_probability(const svm_model *model)
{
    if ((model->param.svm_type == EPSILON_SVR || model->param.svm_type == NU_SVR) && model->probA != NULL)
        return model->probA[0];
    fprintf(stderr, "Model doesn't contain information for SVR probability inference\n");
    return 0;
}

double svm_predict_values(const svm_model *model, const svm_node *x, double *dec_values)
{
    double lab = 0;
    if (svmb::predict_batch(model, &x, 1, &lab, dec_values) != 0) {
        info("ERROR: %s\n", svmb::last_error());
        return NAN;
    }
    return lab;
}

double svm_predict(const svm_model *model, const svm_node *x)
{
    const int k = model->nr_class;
    std::vector<double> dec(std::max(k * (k - 1) / 2, 1));
    return svm_predict_values(model, x, dec.data());
}

// Probability outputs need probA/probB, which this engine does not train
// (svm_parameter.probability is accepted and ignored); as in the reference
// (svm.cpp:2660-2697) such a model falls back to svm_predict.
double svm_predict_probability(const svm_model *model, const svm_node *x, double *prob_estimates)
{
    (void)prob_estimates;
    return svm_predict(model, x);
}

static const char *svm_type_table[] = {"c_svc", "nu_svc", "one_class", "epsilon_svr", "nu_svr", NULL};
static const char *kernel_type_table[] = {"linear", "polynomial", "rbf", "sigmoid", "precomputed", NULL};

// Model file format of the reference (svm.cpp:2709-2801): same keys, same
// number formats (%g header values, %.16g coefficients, %.8g feature values).
int svm_save_model(const char *model_file_name, const svm_model *model)
{
    FILE *fp = fopen(model_file_name, "w");
    if (fp == NULL) return -1;
    char *old_locale = strdup(setlocale(LC_ALL, NULL));
    setlocale(LC_ALL, "C");
    const svm_parameter &param = model->param;
    fprintf(fp, "svm_type %s\n", svm_type_table[param.svm_type]);
    fprintf(fp, "kernel_type %s\n", kernel_type_table[param.kernel_type]);
    if (param.kernel_type == POLY) fprintf(fp, "degree %d\n", param.degree);
    if (param.kernel_type == POLY || param.kernel_type == RBF || param.kernel_type == SIGMOID)
        fprintf(fp, "gamma %g\n", param.gamma);
    if (param.kernel_type == POLY || param.kernel_type == SIGMOID) fprintf(fp, "coef0 %g\n", param.coef0);
    const int nr_class = model->nr_class;
    const int l = model->l;
    const int npair = nr_class * (nr_class - 1) / 2;
    fprintf(fp, "nr_class %d\n", nr_class);
    fprintf(fp, "total_sv %d\n", l);
    fprintf(fp, "rho");
    for (int i = 0; i < npair; i++) fprintf(fp, " %g", model->rho[i]);
    fprintf(fp, "\n");
    if (model->label) {
        fprintf(fp, "label");
        for (int i = 0; i < nr_class; i++) fprintf(fp, " %d", model->label[i]);
        fprintf(fp, "\n");
    }
    if (model->probA) {
        fprintf(fp, "probA");
        for (int i = 0; i < npair; i++) fprintf(fp, " %g", model->probA[i]);
        fprintf(fp, "\n");
    }
    if (model->probB) {
        fprintf(fp, "probB");
        for (int i = 0; i < npair; i++) fprintf(fp, " %g", model->probB[i]);
        fprintf(fp, "\n");
    }
    if (model->nSV) {
        fprintf(fp, "nr_sv");
        for (int i = 0; i < nr_class; i++) fprintf(fp, " %d", model->nSV[i]);
        fprintf(fp, "\n");
    }
    fprintf(fp, "SV\n");
    for (int i = 0; i < l; i++) {
        for (int j = 0; j < nr_class - 1; j++) fprintf(fp, "%.16g ", model->sv_coef[j][i]);
        const svm_node *p = model->SV[i];
        if (param.kernel_type == PRECOMPUTED)
            fprintf(fp, "0:%d ", (int)(p->value));
        else
            for (; p->index != -1; ++p) fprintf(fp, "%d:%.8g ", p->index, p->value);
        fprintf(fp, "\n");
    }
    setlocale(LC_ALL, old_locale);
    free(old_locale);
    if (ferror(fp) != 0 || fclose(fp) != 0) return -1;
    return 0;
}

static bool read_model_header(FILE *fp, svm_model *model)
{
    svm_parameter &param = model->param;
    char cmd[81];
    while (true) {
        if (fscanf(fp, "%80s", cmd) != 1) return false;
        if (!strcmp(cmd, "svm_type")) {
            if (fscanf(fp, "%80s", cmd) != 1) return false;
            int i;
            for (i = 0; svm_type_table[i]; i++)
                if (!strcmp(svm_type_table[i], cmd)) { param.svm_type = i; break; }
            if (!svm_type_table[i]) { fprintf(stderr, "unknown svm type.\n"); return false; }
        } else if (!strcmp(cmd, "kernel_type")) {
            if (fscanf(fp, "%80s", cmd) != 1) return false;
            int i;
            for (i = 0; kernel_type_table[i]; i++)
                if (!strcmp(kernel_type_table[i], cmd)) { param.kernel_type = i; break; }
            if (!kernel_type_table[i]) { fprintf(stderr, "unknown kernel function.\n"); return false; }
        } else if (!strcmp(cmd, "degree")) {
            if (fscanf(fp, "%d", &param.degree) != 1) return false;
        } else if (!strcmp(cmd, "gamma")) {
            if (fscanf(fp, "%lf", &param.gamma) != 1) return false;
        } else if (!strcmp(cmd, "coef0")) {
            if (fscanf(fp, "%lf", &param.coef0) != 1) return false;
        } else if (!strcmp(cmd, "nr_class")) {
            if (fscanf(fp, "%d", &model->nr_class) != 1) return false;
        } else if (!strcmp(cmd, "total_sv")) {
            if (fscanf(fp, "%d", &model->l) != 1) return false;
        } else if (!strcmp(cmd, "rho") || !strcmp(cmd, "probA") || !strcmp(cmd, "probB")) {
            const int n = model->nr_class * (model->nr_class - 1) / 2;
            double *v = (double *)malloc(sizeof(double) * std::max(n, 1));
            if (!strcmp(cmd, "rho")) model->rho = v;
            else if (!strcmp(cmd, "probA")) model->probA = v;
            else model->probB = v;
            for (int i = 0; i < n; i++)
                if (fscanf(fp, "%lf", &v[i]) != 1) return false;
        } else if (!strcmp(cmd, "label") || !strcmp(cmd, "nr_sv")) {
            const int n = model->nr_class;
            int *v = (int *)malloc(sizeof(int) * std::max(n, 1));
            if (!strcmp(cmd, "label")) model->label = v;
            else model->nSV = v;
            for (int i = 0; i < n; i++)
                if (fscanf(fp, "%d", &v[i]) != 1) return false;
        } else if (!strcmp(cmd, "SV")) {
            while (true) {
                const int c = getc(fp);
                if (c == EOF || c == '\n') break;
            }
            break;
        } else {
            fprintf(stderr, "unknown text in model file: [%s]\n", cmd);
            return false;
        }
    }
    return true;
}

static char *read_line(FILE *fp, char **buf, size_t *cap)
{
    size_t len = 0;
    if (!fgets(*buf, (int)*cap, fp)) return NULL;
    while (!strchr(*buf + len, '\n')) {
        len = strlen(*buf);
        *cap *= 2;
        *buf = (char *)realloc(*buf, *cap);
        if (!fgets(*buf + len, (int)(*cap - len), fp)) break;
    }
    return *buf;
}

// Reader for the format above (reference svm.cpp:2941-3044).
svm_model *svm_load_model(const char *model_file_name)
{
    FILE *fp = fopen(model_file_name, "rb");
    if (fp == NULL) return NULL;
    char *old_locale = strdup(setlocale(LC_ALL, NULL));
    setlocale(LC_ALL, "C");
    svm_model *model = (svm_model *)calloc(1, sizeof(svm_model));
    if (!read_model_header(fp, model)) {
        fprintf(stderr, "ERROR: fscanf failed to read model\n");
        setlocale(LC_ALL, old_locale);
        free(old_locale);
        free(model->rho);
        free(model->label);
        free(model->nSV);
        free(model->probA);
        free(model->probB);
        free(model);
        fclose(fp);
        return NULL;
    }
    long elements = 0;
    const long pos = ftell(fp);
    size_t cap = 1024;
    char *line = (char *)malloc(cap);
    while (read_line(fp, &line, &cap)) {
        char *save = NULL;
        char *p = strtok_r(line, ":", &save);
        (void)p;
        while (strtok_r(NULL, ":", &save)) ++elements;
    }
    elements += model->l;
    fseek(fp, pos, SEEK_SET);
    const int m = model->nr_class - 1;
    const int l = model->l;
    model->sv_coef = (double **)malloc(sizeof(double *) * std::max(m, 1));
    for (int i = 0; i < m; i++) model->sv_coef[i] = (double *)malloc(sizeof(double) * std::max(l, 1));
    model->SV = (svm_node **)malloc(sizeof(svm_node *) * std::max(l, 1));
    svm_node *x_space = l > 0 ? (svm_node *)malloc(sizeof(svm_node) * elements) : NULL;
    long j = 0;
    for (int i = 0; i < l; i++) {
        read_line(fp, &line, &cap);
        model->SV[i] = &x_space[j];
        char *save = NULL;
        char *p = strtok_r(line, " \t", &save);
        model->sv_coef[0][i] = strtod(p, NULL);
        for (int k = 1; k < m; k++) {
            p = strtok_r(NULL, " \t", &save);
            model->sv_coef[k][i] = strtod(p, NULL);
        }
        while (true) {
            char *idx = strtok_r(NULL, ":", &save);
            char *val = strtok_r(NULL, " \t", &save);
            if (val == NULL) break;
            x_space[j].index = (int)strtol(idx, NULL, 10);
            x_space[j].value = strtod(val, NULL);
            ++j;
        }
        x_space[j++].index = -1;
    }
    free(line);
    setlocale(LC_ALL, old_locale);
    free(old_locale);
    if (ferror(fp) != 0 || fclose(fp) != 0) return NULL;
    model->free_sv = 1;
    return model;
}

void svm_free_model_content(svm_model *model_ptr)
{
    svmb::predict_forget(model_ptr);
    if (model_ptr->free_sv && model_ptr->l > 0 && model_ptr->SV != NULL) free((void *)(model_ptr->SV[0]));
    if (model_ptr->sv_coef)
        for (int i = 0; i < model_ptr->nr_class - 1; i++) free(model_ptr->sv_coef[i]);
    free(model_ptr->SV);
    model_ptr->SV = NULL;
    free(model_ptr->sv_coef);
    model_ptr->sv_coef = NULL;
    free(model_ptr->rho);
    model_ptr->rho = NULL;
    free(model_ptr->label);
    model_ptr->label = NULL;
    free(model_ptr->probA);
    model_ptr->probA = NULL;
    free(model_ptr->probB);
    model_ptr->probB = NULL;
    free(model_ptr->sv_indices);
    model_ptr->sv_indices = NULL;
    free(model_ptr->nSV);
    model_ptr->nSV = NULL;
}

void svm_free_and_destroy_model(svm_model **model_ptr_ptr)
{
    if (model_ptr_ptr != NULL && *model_ptr_ptr != NULL) {
        svm_free_model_content(*model_ptr_ptr);
        free(*model_ptr_ptr);
        *model_ptr_ptr = NULL;
    }
}

void svm_destroy_param(svm_parameter *param)
{
    free(param->weight_label);
    free(param->weight);
}

// Same checks and messages as the reference (svm.cpp:3097-3216).
const char *svm_check_parameter(const svm_problem *prob, const svm_parameter *param)
{
    const int svm_type = param->svm_type;
    if (svm_type != C_SVC && svm_type != NU_SVC && svm_type != ONE_CLASS && svm_type != EPSILON_SVR && svm_type != NU_SVR)
        return "unknown svm type";
    const int kernel_type = param->kernel_type;
    if (kernel_type != LINEAR && kernel_type != POLY && kernel_type != RBF && kernel_type != SIGMOID &&
        kernel_type != PRECOMPUTED)
        return "unknown kernel type";
    if (param->gamma < 0) return "gamma < 0";
    if (param->degree < 0) return "degree of polynomial kernel < 0";
    if (param->cache_size <= 0) return "cache_size <= 0";
    if (param->eps <= 0) return "eps <= 0";
    if (svm_type == C_SVC || svm_type == EPSILON_SVR || svm_type == NU_SVR)
        if (param->C <= 0) return "C <= 0";
    if (svm_type == NU_SVC || svm_type == ONE_CLASS || svm_type == NU_SVR)
        if (param->nu <= 0 || param->nu > 1) return "nu <= 0 or nu > 1";
    if (svm_type == EPSILON_SVR)
        if (param->p < 0) return "p < 0";
    if (param->shrinking != 0 && param->shrinking != 1) return "shrinking != 0 and shrinking != 1";
    if (param->probability != 0 && param->probability != 1) return "probability != 0 and probability != 1";
    if (param->probability == 1 && svm_type == ONE_CLASS) return "one-class SVM probability output not supported yet";
    if (svm_type == NU_SVC) {
        std::vector<int> label, count;
        for (int i = 0; i < prob->l; i++) {
            const int this_label = (int)prob->y[i];
            size_t j;
            for (j = 0; j < label.size(); j++)
                if (this_label == label[j]) { ++count[j]; break; }
            if (j == label.size()) { label.push_back(this_label); count.push_back(1); }
        }
        for (size_t i = 0; i < label.size(); i++)
            for (size_t j = i + 1; j < label.size(); j++) {
                const int n1 = count[i], n2 = count[j];
                if (param->nu * (n1 + n2) / 2 > std::min(n1, n2)) return "specified nu is infeasible";
            }
    }
    return NULL;
}

int svm_check_probability_model(const svm_model *model)
{
    return ((model->param.svm_type == C_SVC || model->param.svm_type == NU_SVC) && model->probA != NULL &&
            model->probB != NULL) ||
           ((model->param.svm_type == EPSILON_SVR || model->param.svm_type == NU_SVR) && model->probA != NULL);
}

void svm_set_print_string_function(void (*print_func)(const char *))
{
    svm_print_string = print_func == NULL ? &print_string_stdout : print_func;
}

void svmb_print_nothing(const char *) {}

}  // extern "C"
