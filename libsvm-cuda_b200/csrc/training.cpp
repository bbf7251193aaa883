// training.cpp -- see training.hpp.
#include "training.hpp"

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "predict.hpp"

namespace svmb {

void api_print(const char *s);

void print_line(const char *s) { api_print(s); }

namespace {

void say(const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    api_print(buf);
}

// Classes in first-occurrence order; a -1/+1 problem whose first label is -1
// is flipped so that +1 is class 0 (svm.cpp:2081-2154).  perm lists the rows
// class by class, each class in input order.
void group_classes(const svm_problem *prob, int &nr_class, std::vector<int> &label, std::vector<int> &start,
                   std::vector<int> &count, std::vector<int> &perm)
{
    const int l = prob->l;
    label.clear();
    count.clear();
    std::vector<int> cls(l);
    for (int i = 0; i < l; i++) {
        const int v = (int)prob->y[i];
        const auto it = std::find(label.begin(), label.end(), v);
        const int c = (int)(it - label.begin());
        if (it == label.end()) {
            label.push_back(v);
            count.push_back(0);
        }
        ++count[c];
        cls[i] = c;
    }
    nr_class = (int)label.size();
    if (nr_class == 2 && label[0] == -1 && label[1] == 1) {
        std::swap(label[0], label[1]);
        std::swap(count[0], count[1]);
        for (int &c : cls) c = 1 - c;
    }
    start.assign(nr_class, 0);
    for (int c = 1; c < nr_class; c++) start[c] = start[c - 1] + count[c - 1];
    perm.assign(l, 0);
    std::vector<int> next = start;
    for (int i = 0; i < l; i++) perm[next[cls[i]]++] = i;
}

// j = i + rand() % (n - i), swapped, for i = 0..n-1: the reference's shuffle
// (svm.cpp:1969-1974, :2470-2474)
void shuffle(std::vector<int> &v)
{
    const int n = (int)v.size();
    for (int i = 0; i < n; i++) std::swap(v[i], v[i + rand() % (n - i)]);
}

// The points of an internal cross-validation fold: everything outside
// [begin, end) of the shuffled order.
void fold_points(const Training::Estimate &e, Training::Fold &f)
{
    const int n = (int)e.perm.size();
    for (int j = 0; j < n; j++) {
        if (j >= f.begin && j < f.end) continue;
        f.x.push_back(e.x[e.perm[j]]);
        f.y.push_back(e.y[e.perm[j]]);
        f.ids.push_back(e.ids[e.perm[j]]);
    }
}

void plan_nested(Training::Fold &f, const svm_parameter &param, const SolveParams &solve)
{
    svm_problem sub;
    sub.l = (int)f.x.size();
    sub.x = f.x.data();
    sub.y = f.y.data();
    f.model.reset(new Training());
    plan_training(&sub, &param, f.ids.data(), solve, *f.model);
}

// Platt's sigmoid fit of the decision values (svm.cpp:1772-1883: Newton steps
// with a backtracking line search on the regularised targets; every sum is
// accumulated in point order, as there, so the fit is bit-identical).
void sigmoid_train(int l, const double *dec, const double *labels, double &A, double &B)
{
    double n_pos = 0, n_neg = 0;
    for (int i = 0; i < l; i++) (labels[i] > 0 ? n_pos : n_neg) += 1;
    const int max_iter = 100;
    const double min_step = 1e-10, sigma = 1e-12, eps = 1e-5;
    const double hi = (n_pos + 1.0) / (n_pos + 2.0), lo = 1 / (n_neg + 2.0);
    std::vector<double> t(l);
    for (int i = 0; i < l; i++) t[i] = labels[i] > 0 ? hi : lo;
    // negative log-likelihood at (a, b), written to avoid exp overflow
    auto objective = [&](double a, double b) {
        double f = 0.0;
        for (int i = 0; i < l; i++) {
            const double z = dec[i] * a + b;
            if (z >= 0)
                f += t[i] * z + log(1 + exp(-z));
            else
                f += (t[i] - 1) * z + log(1 + exp(z));
        }
        return f;
    };
    A = 0.0;
    B = log((n_neg + 1.0) / (n_pos + 1.0));
    double fval = objective(A, B);
    int iter;
    for (iter = 0; iter < max_iter; iter++) {
        double h11 = sigma, h22 = sigma, h21 = 0.0, g1 = 0.0, g2 = 0.0;
        for (int i = 0; i < l; i++) {
            const double z = dec[i] * A + B;
            double p, q;
            if (z >= 0) {
                p = exp(-z) / (1.0 + exp(-z));
                q = 1.0 / (1.0 + exp(-z));
            } else {
                p = 1.0 / (1.0 + exp(z));
                q = exp(z) / (1.0 + exp(z));
            }
            const double d2 = p * q;
            h11 += dec[i] * dec[i] * d2;
            h22 += d2;
            h21 += dec[i] * d2;
            const double d1 = t[i] - p;
            g1 += dec[i] * d1;
            g2 += d1;
        }
        if (fabs(g1) < eps && fabs(g2) < eps) break;
        const double det = h11 * h22 - h21 * h21;
        const double dA = -(h22 * g1 - h21 * g2) / det;
        const double dB = -(-h21 * g1 + h11 * g2) / det;
        const double gd = g1 * dA + g2 * dB;
        double step = 1;
        while (step >= min_step) {
            const double nA = A + step * dA, nB = B + step * dB;
            const double nf = objective(nA, nB);
            if (nf < fval + 0.0001 * step * gd) {
                A = nA;
                B = nB;
                fval = nf;
                break;
            }
            step = step / 2.0;
        }
        if (step < min_step) {
            say("Line search fails in two-class probability estimates\n");
            break;
        }
    }
    if (iter >= max_iter) say("Reaching maximal iterations in two-class probability estimates\n");
}

double sigmoid_predict(double dec, double A, double B)
{
    const double z = dec * A + B;
    return z >= 0 ? exp(-z) / (1.0 + exp(-z)) : 1.0 / (1 + exp(z));
}

// Pairwise coupling of the pairs' probabilities into class probabilities
// (Wu, Lin and Weng 2004, method 2; svm.cpp:1896-1958): fixed-point updates
// of p on the quadratic form Q built from the pairwise estimates r.
void couple(int k, const std::vector<double> &r, double *p)
{
    auto R = [&](int i, int j) { return r[(size_t)i * k + j]; };
    std::vector<double> Q((size_t)k * k), Qp(k);
    const int max_iter = std::max(100, k);
    const double eps = 0.005 / k;
    for (int t = 0; t < k; t++) {
        p[t] = 1.0 / k;
        double &qtt = Q[(size_t)t * k + t];
        qtt = 0;
        for (int j = 0; j < t; j++) {
            qtt += R(j, t) * R(j, t);
            Q[(size_t)t * k + j] = Q[(size_t)j * k + t];
        }
        for (int j = t + 1; j < k; j++) {
            qtt += R(j, t) * R(j, t);
            Q[(size_t)t * k + j] = -R(j, t) * R(t, j);
        }
    }
    int iter;
    for (iter = 0; iter < max_iter; iter++) {
        double pQp = 0;
        for (int t = 0; t < k; t++) {
            Qp[t] = 0;
            for (int j = 0; j < k; j++) Qp[t] += Q[(size_t)t * k + j] * p[j];
            pQp += p[t] * Qp[t];
        }
        double worst = 0;
        for (int t = 0; t < k; t++) worst = std::max(worst, fabs(Qp[t] - pQp));
        if (worst < eps) break;
        for (int t = 0; t < k; t++) {
            const double qtt = Q[(size_t)t * k + t];
            const double diff = (-Qp[t] + pQp) / qtt;
            p[t] += diff;
            pQp = (pQp + diff * (diff * qtt + 2 * Qp[t])) / (1 + diff) / (1 + diff);
            for (int j = 0; j < k; j++) {
                Qp[j] = (Qp[j] + diff * Q[(size_t)t * k + j]) / (1 + diff);
                p[j] /= (1 + diff);
            }
        }
    }
    if (iter >= max_iter) say("Exceeds max_iter in multiclass_prob\n");
}

void fill_stats(const Decision &f, const SolveResult &R, int l, svmb_solve_stats &st)
{
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

// the solver's messages of one subproblem: the max_iter warning first
// (svm.cpp:779-787), then one print-hook call per info() of the reference
void emit(const Decision &f, const SolveResult &R)
{
    if (R.out.status == 1) fprintf(stderr, "\nWARNING: reaching max number of iterations\n");
    for (const std::string &line : f.log) api_print(line.c_str());
}

// Decision values of held-out points by a fold's model (or its fixed value).
// Returns -1 if the fold's model could not be built or evaluated.
int fold_values(Training::Fold &f, const Training::Estimate &e, const std::vector<SolveResult> &res,
                std::vector<svmb_solve_stats> &stats, bool want_label, double *out)
{
    const int n = f.end - f.begin;
    if (!f.model) {
        for (int j = f.begin; j < f.end; j++) out[e.perm[j]] = f.fixed;
        return 0;
    }
    svm_model *m = assemble(*f.model, res, stats);
    if (!m) return -1;
    std::vector<const svm_node *> held(n);
    for (int j = 0; j < n; j++) held[j] = e.x[e.perm[f.begin + j]];
    std::vector<double> lab(std::max(n, 1)), dec(std::max(n, 1));
    int rc = n ? predict_batch(m, held.data(), n, lab.data(), dec.data()) : 0;
    if (rc == 0)
        for (int j = 0; j < n; j++)
            // the classifier's value is taken in +1/-1 order (svm.cpp:2027-2033)
            out[e.perm[f.begin + j]] = want_label ? lab[j] : dec[j] * m->label[0];
    svm_free_and_destroy_model(&m);
    return rc;
}

}  // namespace

void cv_folds(const svm_problem *prob, const svm_parameter *param, int &nr_fold, std::vector<int> &perm,
              std::vector<int> &fold_start)
{
    const int l = prob->l;
    perm.assign(l, 0);
    if (nr_fold > l) {
        nr_fold = l;
        fprintf(stderr, "WARNING: # folds > # data. Will use # folds = # data instead (i.e., leave-one-out cross validation)\n");
    }
    fold_start.assign(nr_fold + 1, 0);
    if ((param->svm_type == C_SVC || param->svm_type == NU_SVC) && nr_fold < l) {
        // stratified: each class shuffled with rand() and dealt to the folds in
        // contiguous runs (svm.cpp:2420-2467)
        int nr_class;
        std::vector<int> label, start, count;
        group_classes(prob, nr_class, label, start, count, perm);
        std::vector<int> index(perm);
        for (int c = 0; c < nr_class; c++)
            for (int i = 0; i < count[c]; i++) {
                const int j = i + rand() % (count[c] - i);
                std::swap(index[start[c] + j], index[start[c] + i]);
            }
        std::vector<int> fold_count(nr_fold, 0);
        for (int i = 0; i < nr_fold; i++)
            for (int c = 0; c < nr_class; c++) fold_count[i] += (i + 1) * count[c] / nr_fold - i * count[c] / nr_fold;
        std::vector<int> next(nr_fold, 0);
        for (int i = 1; i < nr_fold; i++) next[i] = next[i - 1] + fold_count[i - 1];
        for (int c = 0; c < nr_class; c++)
            for (int i = 0; i < nr_fold; i++)
                for (int j = start[c] + i * count[c] / nr_fold; j < start[c] + (i + 1) * count[c] / nr_fold; j++)
                    perm[next[i]++] = index[j];
        for (int i = 1; i <= nr_fold; i++) fold_start[i] = fold_start[i - 1] + fold_count[i - 1];
    } else {
        for (int i = 0; i < l; i++) perm[i] = i;
        shuffle(perm);
        for (int i = 0; i <= nr_fold; i++) fold_start[i] = i * l / nr_fold;
    }
}

void plan_training(const svm_problem *prob, const svm_parameter *param, const int *row_id, const SolveParams &solve,
                   Training &t)
{
    t.prob = *prob;
    t.param = *param;
    t.solve = solve;
    const int l = prob->l;
    t.classify = param->svm_type == C_SVC || param->svm_type == NU_SVC;
    if (!t.classify) {
        // one-class / eps-SVR / nu-SVR: one problem over the rows in input order
        t.x.assign(prob->x, prob->x + l);
        t.ids.resize(l);
        for (int i = 0; i < l; i++) t.ids[i] = row_id ? row_id[i] : i;
        if (param->probability && (param->svm_type == EPSILON_SVR || param->svm_type == NU_SVR)) {
            // svm_svr_probability: a 5-fold cross-validation of the same
            // training without probability outputs (svm.cpp:2047-2078)
            svm_parameter inner = *param;
            inner.probability = 0;
            int nr_fold = 5;
            std::vector<int> perm, fold_start;
            cv_folds(prob, &inner, nr_fold, perm, fold_start);
            t.est.resize(1);
            Training::Estimate &e = t.est[0];
            e.x = t.x;
            e.y.assign(prob->y, prob->y + l);
            e.ids = t.ids;
            e.perm = perm;
            e.folds.resize(nr_fold);
            for (int f = 0; f < nr_fold; f++) {
                Training::Fold &fd = e.folds[f];
                fd.begin = fold_start[f];
                fd.end = fold_start[f + 1];
                fold_points(e, fd);
                plan_nested(fd, inner, solve);
            }
        }
        t.subs.resize(1);
        t.sub_y.assign(1, std::vector<double>(prob->y, prob->y + l));
        formulate(param->svm_type, t.ids.data(), prob->y, l, 0, 0, param->C, param->nu, param->p, t.subs[0]);
        return;
    }
    group_classes(prob, t.nr_class, t.label, t.start, t.count, t.perm);
    const int nr_class = t.nr_class;
    if (nr_class == 1) say("WARNING: training data in only one class. See README for details.\n");
    t.x.resize(l);
    t.ids.resize(l);
    for (int g = 0; g < l; g++) {
        t.x[g] = prob->x[t.perm[g]];
        t.ids[g] = row_id ? row_id[t.perm[g]] : g;
    }
    t.weighted_C.assign(nr_class, param->C);
    for (int w = 0; w < param->nr_weight; w++) {
        const auto it = std::find(t.label.begin(), t.label.end(), param->weight_label[w]);
        if (it == t.label.end())
            fprintf(stderr, "WARNING: class label %d specified in weight is not found\n", param->weight_label[w]);
        else
            t.weighted_C[it - t.label.begin()] *= param->weight[w];
    }
    const int npair = nr_class * (nr_class - 1) / 2;
    t.subs.resize(npair);
    t.sub_y.resize(npair);
    if (param->probability) t.est.resize(npair);
    std::vector<int> pair_i(npair), pair_j(npair);
    for (int i = 0, p = 0; i < nr_class; i++)
        for (int j = i + 1; j < nr_class; j++, p++) pair_i[p] = i, pair_j[p] = j;
    // the pairs are independent, so they are built on all host threads --
    // except with probability estimates, whose shuffles draw rand() in pair order
#pragma omp parallel for schedule(dynamic, 1) if (npair > 1 && !param->probability)
    for (int p = 0; p < npair; p++) {
        {
            const int i = pair_i[p], j = pair_j[p];
            // class i's rows as +1, then class j's as -1
            const int ci = t.count[i], cj = t.count[j], n = ci + cj;
            std::vector<int> rows(n);
            std::vector<double> &yv = t.sub_y[p];
            yv.assign(n, -1.0);
            for (int k = 0; k < ci; k++) rows[k] = t.ids[t.start[i] + k], yv[k] = +1;
            for (int k = 0; k < cj; k++) rows[ci + k] = t.ids[t.start[j] + k];
            if (param->probability) {
                // svm_binary_svc_probability (svm.cpp:1960-2045): shuffle the
                // pair's points, 5 folds; each fold trains with C = 1 and the
                // pair's bounds as class weights, unless one class is missing
                Training::Estimate &e = t.est[p];
                e.x.resize(n);
                for (int k = 0; k < ci; k++) e.x[k] = t.x[t.start[i] + k];
                for (int k = 0; k < cj; k++) e.x[ci + k] = t.x[t.start[j] + k];
                e.y = yv;
                e.ids = rows;
                e.perm.resize(n);
                for (int k = 0; k < n; k++) e.perm[k] = k;
                shuffle(e.perm);
                const int nr_fold = 5;
                e.folds.resize(nr_fold);
                for (int f = 0; f < nr_fold; f++) {
                    Training::Fold &fd = e.folds[f];
                    fd.begin = f * n / nr_fold;
                    fd.end = (f + 1) * n / nr_fold;
                    fold_points(e, fd);
                    int npos = 0, nneg = 0;
                    for (double v : fd.y) (v > 0 ? npos : nneg)++;
                    if (npos == 0 || nneg == 0) {
                        fd.fixed = npos > 0 ? 1 : nneg > 0 ? -1 : 0;
                        continue;
                    }
                    svm_parameter inner = *param;
                    inner.probability = 0;
                    inner.C = 1.0;
                    fd.wlabel = {+1, -1};
                    fd.wvalue = {t.weighted_C[i], t.weighted_C[j]};
                    inner.nr_weight = 2;
                    inner.weight_label = fd.wlabel.data();
                    inner.weight = fd.wvalue.data();
                    plan_nested(fd, inner, solve);
                }
            }
            formulate(param->svm_type, rows.data(), yv.data(), n, t.weighted_C[i], t.weighted_C[j], param->C,
                      param->nu, param->p, t.subs[p]);
        }
    }
}

void collect(Training &t, std::vector<SubProblem> &all)
{
    for (Training::Estimate &e : t.est)
        for (Training::Fold &f : e.folds)
            if (f.model) collect(*f.model, all);
    t.first = all.size();
    const int nsub = (int)t.subs.size();
    all.resize(t.first + nsub);
    // copies of independent subproblems (hundreds of thousands of positions)
#pragma omp parallel for schedule(dynamic, 1) if (nsub > 1)
    for (int p = 0; p < nsub; p++) {
        t.subs[p].own = &t.solve;
        all[t.first + p] = t.subs[p];
    }
}

svm_model *assemble(Training &t, const std::vector<SolveResult> &res, std::vector<svmb_solve_stats> &stats)
{
    const svm_parameter &param = t.param;
    const int l = t.prob.l;
    const int nsub = (int)t.subs.size();
    // the decision functions (independent, so in parallel); the messages,
    // probability fits and statistics follow in the reference's order
    std::vector<Decision> f(nsub);
#pragma omp parallel for schedule(dynamic, 1) if (nsub > 1)
    for (int p = 0; p < nsub; p++)
        decide(param.svm_type, t.subs[p], res[t.first + p], t.sub_y[p].data(), (int)t.sub_y[p].size(), f[p]);
    svm_model *model = (svm_model *)calloc(1, sizeof(svm_model));
    model->param = param;
    model->free_sv = 0;
    if (!t.classify) {
        if (!t.est.empty()) {
            // Laplace scale of the cross-validation residuals, leaving out those
            // beyond 5 standard deviations (svm.cpp:2055-2075)
            Training::Estimate &e = t.est[0];
            std::vector<double> pred(std::max(l, 1));
            for (Training::Fold &fd : e.folds)
                if (fold_values(fd, e, res, stats, true, pred.data()) != 0) {
                    svm_free_and_destroy_model(&model);
                    return nullptr;
                }
            double mae = 0;
            for (int i = 0; i < l; i++) {
                pred[i] = t.prob.y[i] - pred[i];
                mae += fabs(pred[i]);
            }
            mae /= l;
            const double sd = sqrt(2 * mae * mae);
            int outliers = 0;
            mae = 0;
            for (int i = 0; i < l; i++) {
                if (fabs(pred[i]) > 5 * sd)
                    outliers = outliers + 1;
                else
                    mae += fabs(pred[i]);
            }
            mae /= (l - outliers);
            say("Prob. model for test data: target value = predicted value + z,\nz: Laplace distribution "
                "e^(-|z|/sigma)/(2sigma),sigma= %g\n", mae);
            model->probA = (double *)malloc(sizeof(double));
            model->probA[0] = mae;
        }
        emit(f[0], res[t.first]);
        stats.emplace_back();
        fill_stats(f[0], res[t.first], (int)t.subs[0].rows.size(), stats.back());
        // the support vectors in input order (svm.cpp:2192-2208)
        model->nr_class = 2;
        model->rho = (double *)malloc(sizeof(double));
        model->rho[0] = f[0].rho;
        int nsv = 0;
        for (int i = 0; i < l; i++)
            if (fabs(f[0].coef[i]) > 0) ++nsv;
        model->l = nsv;
        model->SV = (svm_node **)malloc(sizeof(svm_node *) * std::max(nsv, 1));
        model->sv_coef = (double **)malloc(sizeof(double *));
        model->sv_coef[0] = (double *)malloc(sizeof(double) * std::max(nsv, 1));
        model->sv_indices = (int *)malloc(sizeof(int) * std::max(nsv, 1));
        for (int i = 0, q = 0; i < l; i++)
            if (fabs(f[0].coef[i]) > 0) {
                model->SV[q] = t.x[i];
                model->sv_coef[0][q] = f[0].coef[i];
                model->sv_indices[q++] = i + 1;
            }
        return model;
    }

    const int nr_class = t.nr_class;
    const int npair = nsub;
    std::vector<double> probA, probB;
    if (param.probability) {
        probA.assign(npair, 0.0);
        probB.assign(npair, 0.0);
    }
    for (int p = 0; p < npair; p++) {
        if (param.probability) {
            Training::Estimate &e = t.est[p];
            const int n = (int)e.perm.size();
            std::vector<double> dec(std::max(n, 1));
            for (Training::Fold &fd : e.folds)
                if (fold_values(fd, e, res, stats, false, dec.data()) != 0) {
                    svm_free_and_destroy_model(&model);
                    return nullptr;
                }
            sigmoid_train(n, dec.data(), e.y.data(), probA[p], probB[p]);
        }
        emit(f[p], res[t.first + p]);
        stats.emplace_back();
        fill_stats(f[p], res[t.first + p], (int)t.subs[p].rows.size(), stats.back());
    }
    // the model (svm.cpp:2297-2386): SVs are the points with a nonzero
    // coefficient in any pair, class by class; sv_coef[j-1] holds class i's
    // coefficients against j and sv_coef[i] class j's against i
    model->nr_class = nr_class;
    model->label = (int *)malloc(sizeof(int) * std::max(nr_class, 1));
    for (int i = 0; i < nr_class; i++) model->label[i] = t.label[i];
    model->rho = (double *)malloc(sizeof(double) * std::max(npair, 1));
    for (int p = 0; p < npair; p++) model->rho[p] = f[p].rho;
    if (param.probability) {
        model->probA = (double *)malloc(sizeof(double) * std::max(npair, 1));
        model->probB = (double *)malloc(sizeof(double) * std::max(npair, 1));
        for (int p = 0; p < npair; p++) model->probA[p] = probA[p], model->probB[p] = probB[p];
    }
    std::vector<char> nonzero(l, 0);
    for (int i = 0, p = 0; i < nr_class; i++)
        for (int j = i + 1; j < nr_class; j++, p++) {
            for (int k = 0; k < t.count[i]; k++)
                if (fabs(f[p].coef[k]) > 0) nonzero[t.start[i] + k] = 1;
            for (int k = 0; k < t.count[j]; k++)
                if (fabs(f[p].coef[t.count[i] + k]) > 0) nonzero[t.start[j] + k] = 1;
        }
    int total_sv = 0;
    model->nSV = (int *)malloc(sizeof(int) * std::max(nr_class, 1));
    std::vector<int> nz_start(nr_class, 0);
    for (int i = 0; i < nr_class; i++) {
        int c = 0;
        for (int j = 0; j < t.count[i]; j++) c += nonzero[t.start[i] + j];
        model->nSV[i] = c;
        if (i > 0) nz_start[i] = nz_start[i - 1] + model->nSV[i - 1];
        total_sv += c;
    }
    say("Total nSV = %d\n", total_sv);
    model->l = total_sv;
    model->SV = (svm_node **)malloc(sizeof(svm_node *) * std::max(total_sv, 1));
    model->sv_indices = (int *)malloc(sizeof(int) * std::max(total_sv, 1));
    for (int g = 0, q = 0; g < l; g++)
        if (nonzero[g]) {
            model->SV[q] = t.x[g];
            model->sv_indices[q++] = t.perm[g] + 1;
        }
    model->sv_coef = (double **)malloc(sizeof(double *) * std::max(nr_class - 1, 1));
    for (int i = 0; i < nr_class - 1; i++) model->sv_coef[i] = (double *)malloc(sizeof(double) * std::max(total_sv, 1));
    for (int i = 0, p = 0; i < nr_class; i++)
        for (int j = i + 1; j < nr_class; j++, p++) {
            int q = nz_start[i];
            for (int k = 0; k < t.count[i]; k++)
                if (nonzero[t.start[i] + k]) model->sv_coef[j - 1][q++] = f[p].coef[k];
            q = nz_start[j];
            for (int k = 0; k < t.count[j]; k++)
                if (nonzero[t.start[j] + k]) model->sv_coef[i][q++] = f[p].coef[t.count[i] + k];
        }
    return model;
}

int predict_probability_batch(const svm_model *model, const svm_node *const *rows, int n, double *labels,
                              double *prob)
{
    const int k = model->nr_class, npair = k * (k - 1) / 2;
    std::vector<double> dec((size_t)std::max(n, 1) * std::max(npair, 1));
    if (predict_batch(model, rows, n, labels, dec.data()) != 0) return -1;
    const double min_prob = 1e-7;
    std::vector<double> r((size_t)k * k);
    for (int t = 0; t < n; t++) {
        const double *d = dec.data() + (size_t)t * npair;
        for (int i = 0, p = 0; i < k; i++)
            for (int j = i + 1; j < k; j++, p++) {
                const double v = std::min(std::max(sigmoid_predict(d[p], model->probA[p], model->probB[p]), min_prob),
                                          1 - min_prob);
                r[(size_t)i * k + j] = v;
                r[(size_t)j * k + i] = 1 - v;
            }
        double *pt = prob + (size_t)t * k;
        couple(k, r, pt);
        int best = 0;
        for (int i = 1; i < k; i++)
            if (pt[i] > pt[best]) best = i;
        labels[t] = model->label[best];
    }
    return 0;
}

}  // namespace svmb
