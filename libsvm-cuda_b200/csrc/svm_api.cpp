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
#include "training.hpp"
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


bool train_supported(const svm_parameter *param)
{
    if (param->kernel_type == PRECOMPUTED) {
        svmb::set_error("precomputed kernels are not trained on the GPU");
        info("ERROR: %s\n", svmb::last_error());
        return false;
    }
    if (param->svm_type < C_SVC || param->svm_type > NU_SVR) {
        svmb::set_error("unknown svm type");
        info("ERROR: %s\n", svmb::last_error());
        return false;
    }
    return true;
}

void record_stats(const std::vector<svmb_solve_stats> &st)
{
    std::lock_guard<std::mutex> g(g_stats_mu);
    g_last_stats.insert(g_last_stats.end(), st.begin(), st.end());
}

// Stratified k-fold cross-validation (reference svm.cpp:2407-2525) over a grid
// of (C, gamma) points: one fold assignment with the C library rand(), as the
// reference draws it, then every point's and fold's training (with its
// probability cross-validations, if asked for) is planned, all their binary
// subproblems are solved in batched launches over the rows uploaded once, and
// the models are assembled and evaluated point by point, fold by fold.
// target[p*l + i] is the prediction of row i by the model of point p trained
// without i's fold.
int cross_validation_grid(const svm_problem *prob, const svm_parameter *param, int nr_fold, int npoints,
                          const double *Cs, const double *gammas, double *target)
{
    {
        std::lock_guard<std::mutex> g(g_stats_mu);
        g_last_stats.clear();
    }
    const int l = prob->l;
    std::vector<int> perm, fold_start;
    svmb::cv_folds(prob, param, nr_fold, perm, fold_start);
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
    // the training set of every fold and one training per (point, fold)
    std::vector<svm_problem> fold_prob(nr_fold);
    std::vector<std::vector<svm_node *>> fold_x(nr_fold);
    std::vector<std::vector<double>> fold_y(nr_fold);
    std::vector<std::vector<int>> fold_id(nr_fold);
    for (int i = 0; i < nr_fold; i++) {
        for (int j = 0; j < l; j++) {
            if (j >= fold_start[i] && j < fold_start[i + 1]) continue;
            fold_x[i].push_back(prob->x[perm[j]]);
            fold_y[i].push_back(prob->y[perm[j]]);
            fold_id[i].push_back(perm[j]);
        }
        fold_prob[i].l = (int)fold_x[i].size();
        fold_prob[i].x = fold_x[i].data();
        fold_prob[i].y = fold_y[i].data();
    }
    std::vector<svm_parameter> pparam(npoints, *param);
    std::vector<svmb::Training> jobs((size_t)npoints * nr_fold);
    std::vector<svmb::SubProblem> all;
    for (int q = 0; q < npoints; q++) {
        pparam[q].C = Cs[q];
        pparam[q].gamma = gammas[q];
        for (int i = 0; i < nr_fold; i++)
            svmb::plan_training(&fold_prob[i], &pparam[q], fold_id[i].data(), make_solve_params(&pparam[q]),
                                jobs[(size_t)q * nr_fold + i]);
    }
    for (svmb::Training &t : jobs) svmb::collect(t, all);
    std::vector<svmb::SolveResult> res;
    const double t_setup = since(c0);
    const auto c1 = std::chrono::steady_clock::now();
    if (!all.empty() && svmb::solve_batch(rows, all, jobs[0].solve, res, 0) != 0) {
        info("ERROR: %s\n", svmb::last_error());
        return -1;
    }
    const double t_solve = since(c1);
    const auto c2 = std::chrono::steady_clock::now();
    const bool with_prob = param->probability && (param->svm_type == C_SVC || param->svm_type == NU_SVC);
    for (int q = 0; q < npoints; q++)
        for (int i = 0; i < nr_fold; i++) {
            std::vector<svmb_solve_stats> st;
            svm_model *m = svmb::assemble(jobs[(size_t)q * nr_fold + i], res, st);
            record_stats(st);
            if (!m) continue;
            const int begin = fold_start[i], end = fold_start[i + 1];
            std::vector<const svm_node *> held;
            for (int j = begin; j < end; j++) held.push_back(prob->x[perm[j]]);
            std::vector<double> lab(std::max<size_t>(held.size(), 1));
            int rc = 0;
            if (held.empty()) rc = 0;
            else if (with_prob) {
                // svm_predict_probability's label (svm.cpp:2500-2506)
                std::vector<double> pe(held.size() * (size_t)std::max(m->nr_class, 1));
                rc = svmb::predict_probability_batch(m, held.data(), (int)held.size(), lab.data(), pe.data());
            } else {
                rc = svmb::predict_batch(m, held.data(), (int)held.size(), lab.data(), nullptr);
            }
            if (rc == 0)
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
        if (value < FORM_EXACT || value > FORM_TF32) return -1;
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
    } else if (!strcmp(name, "blocks_per_sm")) {
        if (set_blocks_per_sm((int)value) != 0) return -1;
    } else if (!strcmp(name, "wait_limit_ms")) {
        if (value < 0) return -1;
        set_wait_limit_ms(value);
    } else if (!strcmp(name, "test_drop_block")) {
        if (value != 1) return -1;
        arm_drop_block();
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
    svmb::Training t;
    svmb::plan_training(prob, param, nullptr, make_solve_params(param), t);
    std::vector<svmb::SubProblem> all;
    svmb::collect(t, all);
    const auto t1 = std::chrono::steady_clock::now();
    // rows are uploaded once, in the plan's order (grouped by class for the
    // classifiers); every subproblem addresses them by id
    svmb::DeviceRows rows;
    if (prob->l > 0 &&
        svmb::upload_rows(t.x.data(), prob->l, rows, svmb::api_force_layout(), 0, svmb::kAllocPooled) != 0) {
        info("ERROR: %s\n", svmb::last_error());
        return NULL;
    }
    const auto t2 = std::chrono::steady_clock::now();
    std::vector<svmb::SolveResult> res;
    if (!all.empty() && svmb::solve_batch(rows, all, t.solve, res, 0) != 0) {
        info("ERROR: %s\n", svmb::last_error());
        return NULL;
    }
    const auto t3 = std::chrono::steady_clock::now();
    std::vector<svmb_solve_stats> st;
    svm_model *model = svmb::assemble(t, res, st);
    record_stats(st);
    if (!model) info("ERROR: %s\n", svmb::last_error());
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

// Class probabilities by pairwise coupling of the pairs' sigmoid estimates
// (reference svm.cpp:2660-2697); models without probA/probB fall back to
// svm_predict, as there.
double svm_predict_probability(const svm_model *model, const svm_node *x, double *prob_estimates)
{
    if ((model->param.svm_type == C_SVC || model->param.svm_type == NU_SVC) && model->probA != NULL &&
        model->probB != NULL) {
        double lab = 0;
        if (svmb::predict_probability_batch(model, &x, 1, &lab, prob_estimates) != 0) {
            info("ERROR: %s\n", svmb::last_error());
            return NAN;
        }
        return lab;
    }
    return svm_predict(model, x);
}

int svmb_predict_probability_batch(const struct svm_model *model, const struct svm_node *const *rows, int n,
                                   double *labels, double *prob_estimates)
{
    if (!model || (n > 0 && (!rows || !labels || !prob_estimates)) || n < 0) {
        svmb::set_error("invalid arguments");
        return -1;
    }
    if (!svm_check_probability_model(model) || model->param.svm_type == EPSILON_SVR ||
        model->param.svm_type == NU_SVR) {
        svmb::set_error("the model has no class probability information (train with probability = 1)");
        return -1;
    }
    return svmb::predict_probability_batch(model, rows, n, labels, prob_estimates);
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
