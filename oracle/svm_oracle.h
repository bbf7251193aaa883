/*
 * svm_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's CPU training and prediction path
 * (libsvm 3.18 as carried by climber544/libsvm-cuda, reference libsvm/svm.cpp).
 * It is the checker for the GPU engine: only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline leg may load it.  The product library never
 * links or calls it.
 *
 * Parity pin: tests/test_oracle_pin.py runs this restatement (oracle_dump)
 * and the reference itself (oracle/_ref/ref_dump, compiled from the reference
 * sources) on the committed fixtures under tests/golden/ and requires
 * identical output (alpha, rho, #iter, decision values, CV targets).
 *
 * Q storage precision: built with -DORACLE_QDOUBLE the cached kernel rows are
 * double (the "FP64 oracle"); otherwise float exactly like the reference
 * (`typedef float Qfloat`, reference svm.cpp:16).
 */
#ifndef SVM_ORACLE_H
#define SVM_ORACLE_H

#include "svm.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Per binary subproblem record of the last oracle_svm_train / cross validation
 * call, in solve order (what the reference prints through info()). */
typedef struct {
    long long iters;
    double obj;
    double rho;
    double r;           /* nu-SVC only (Solver_NU si->r) */
    int l;
    int nr_free;        /* #alpha strictly inside (0, C) */
    int nr_sv;
} oracle_solve_info;

struct svm_model *oracle_svm_train(const struct svm_problem *prob, const struct svm_parameter *param);
void oracle_cross_validation(const struct svm_problem *prob, const struct svm_parameter *param, int nr_fold, double *target);
double oracle_predict_values(const struct svm_model *model, const struct svm_node *x, double *dec_values);
double oracle_predict(const struct svm_model *model, const struct svm_node *x);
double oracle_k_function(const struct svm_node *x, const struct svm_node *y, const struct svm_parameter *param);
void oracle_free_model(struct svm_model *model);

/* Binary solve of one C-SVC (svm_type C_SVC, labels >0 -> +1) or nu-SVC
 * problem; alpha_out[l] receives the signed coefficients y_i*alpha_i
 * (divided by r for nu-SVC), like decision_function.alpha in the reference. */
int oracle_solve_binary(const struct svm_problem *prob, const struct svm_parameter *param,
                        double Cp, double Cn, double *alpha_out, oracle_solve_info *info);

int oracle_solve_count(void);
int oracle_solve_get(int k, oracle_solve_info *out);
int oracle_q_is_double(void);
void oracle_srand(unsigned seed);

#ifdef __cplusplus
}
#endif

#endif
