// training.hpp -- svm_train / svm_cross_validation as plans of batched solves
// (internal).
//
// One svm_train call (reference svm.cpp:2159-2404) is planned as the binary
// subproblems it solves -- every one-vs-one pair, or the one regression /
// one-class problem -- plus, with probability outputs, the trainings of the
// internal 5-fold cross-validations (svm_binary_svc_probability :1960-2045,
// svm_svr_probability :2047-2078) as nested plans.  The subproblems of a plan
// and of all its nested plans (and of many plans: CV folds, grid points) are
// solved together in batched device launches; the models are then assembled
// in the reference's order, so its messages, its rand() draws and its results
// come out the same.
#pragma once
#include <memory>
#include <vector>

#include "engine.hpp"
#include "formulation.hpp"
#include "svm.h"
#include "svm_b200.h"

namespace svmb {

struct Training {
    svm_problem prob{};                 // the caller's rows and targets
    svm_parameter param{};
    bool classify = true;               // C_SVC / NU_SVC
    // classification: classes in first-occurrence order (svm_group_classes, svm.cpp:2081-2154)
    int nr_class = 0;
    std::vector<int> label, start, count, perm;
    std::vector<svm_node *> x;          // rows in the order they are addressed (grouped for classification)
    std::vector<int> ids;               // device row id of x[i]
    std::vector<double> weighted_C;
    // the binary problems: classification pairs in pair order, or the one problem
    std::vector<SubProblem> subs;
    std::vector<std::vector<double>> sub_y;   // targets of each problem's points
    // probability estimation: one internal cross-validation per pair (or for the SVR problem)
    struct Fold {
        int begin = 0, end = 0;
        double fixed = 0;               // decision value of the held-out points when no model is trained
        std::vector<svm_node *> x;
        std::vector<double> y;
        std::vector<int> ids;
        std::vector<int> wlabel;
        std::vector<double> wvalue;
        std::unique_ptr<Training> model;
    };
    struct Estimate {
        std::vector<svm_node *> x;      // the points of the estimate's problem
        std::vector<double> y;
        std::vector<int> ids;
        std::vector<int> perm;          // rand() shuffle of those points
        std::vector<Fold> folds;
    };
    std::vector<Estimate> est;
    SolveParams solve;
    size_t first = 0;                   // index of subs[0] in the collected batch
};

// Plan one svm_train.  row_id[i]: device row id of prob->x[i]; nullptr: the
// rows are uploaded in the order of t.x (grouped by class for classification).
// Draws the C library rand() exactly where the reference does.
void plan_training(const svm_problem *prob, const svm_parameter *param, const int *row_id, const SolveParams &solve,
                   Training &t);
// Append the subproblems of t and of its nested plans to `all` (each keeps its
// own solve parameters).
void collect(Training &t, std::vector<SubProblem> &all);
// Decision functions, messages (through the print hook), probability fits and
// the model.  stats receives one record per solve, in message order.
svm_model *assemble(Training &t, const std::vector<SolveResult> &res, std::vector<svmb_solve_stats> &stats);

// Fold assignment of svm_cross_validation (svm.cpp:2407-2475): perm[] lists the
// rows fold by fold, fold_start[nr_fold+1]; nr_fold is clamped to l.
void cv_folds(const svm_problem *prob, const svm_parameter *param, int &nr_fold, std::vector<int> &perm,
              std::vector<int> &fold_start);

// Labels and probability estimates (svm_predict_probability, svm.cpp:2660-2697)
// of n rows of a C-SVC / nu-SVC model with probA/probB; prob [n][nr_class].
int predict_probability_batch(const svm_model *model, const svm_node *const *rows, int n, double *labels,
                              double *prob);

void print_line(const char *s);

}  // namespace svmb
