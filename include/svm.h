/*
 * svm.h -- drop-in C API of the B200 SVM engine.
 *
 * This header declares the same structures and functions as the libsvm-cuda
 * API (reference libsvm/svm.h:23-118, libsvm 3.18 with a leading `cuda_flag`
 * member in svm_parameter).  Structure layouts are byte-identical so that a
 * program written against the reference (e.g. svm-train/svm-train.c) compiles
 * and links against libsvm_b200.so unchanged.  The layouts have to be alike:
 * they are the ABI.
 *
 * Behavioural differences from the reference:
 *   - training always runs on the GPU (cuda_flag is accepted and ignored;
 *     there is no CPU fallback: a missing/unusable GPU makes svm_train
 *     return NULL and report the reason through the print hook and
 *     svmb_last_error());
 *   - shrinking is honoured on the GPU (the reference's GPU path forces it off,
 *     reference svm-train/svm-train.c:260-262);
 *   - nothing ever calls exit() or cudaDeviceReset() on the caller's behalf.
 */
#ifndef LIBSVM_B200_SVM_H
#define LIBSVM_B200_SVM_H

#define LIBSVM_VERSION 318

#ifdef __cplusplus
extern "C" {
#endif

/* reference libsvm/svm.h:29, svm.cpp:15 */
extern int libsvm_version;

/* One (index, value) feature; a row ends with index == -1.  reference svm.h:31-35 */
struct svm_node {
    int index;
    double value;
};

/* reference svm.h:37-42 */
struct svm_problem {
    int l;
    double *y;
    struct svm_node **x;
};

/* reference svm.h:44-45 */
enum { C_SVC, NU_SVC, ONE_CLASS, EPSILON_SVR, NU_SVR };     /* svm_type */
enum { LINEAR, POLY, RBF, SIGMOID, PRECOMPUTED };           /* kernel_type */

/* reference svm.h:47-67 (note the leading cuda_flag, reference svm.h:49) */
struct svm_parameter {
    int cuda_flag;
    int svm_type;
    int kernel_type;
    int degree;
    double gamma;
    double coef0;

    double cache_size;      /* MB */
    double eps;
    double C;
    int nr_weight;
    int *weight_label;
    double *weight;
    double nu;
    double p;
    int shrinking;
    int probability;
};

/* reference svm.h:72-92 */
struct svm_model {
    struct svm_parameter param;
    int nr_class;
    int l;
    struct svm_node **SV;
    double **sv_coef;
    double *rho;
    double *probA;
    double *probB;
    int *sv_indices;
    int *label;
    int *nSV;
    int free_sv;
};

/* reference svm.h:94-118 */
struct svm_model *svm_train(const struct svm_problem *prob, const struct svm_parameter *param);
void svm_cross_validation(const struct svm_problem *prob, const struct svm_parameter *param, int nr_fold, double *target);

int svm_save_model(const char *model_file_name, const struct svm_model *model);
struct svm_model *svm_load_model(const char *model_file_name);

int svm_get_svm_type(const struct svm_model *model);
int svm_get_nr_class(const struct svm_model *model);
void svm_get_labels(const struct svm_model *model, int *label);
void svm_get_sv_indices(const struct svm_model *model, int *sv_indices);
int svm_get_nr_sv(const struct svm_model *model);
double svm_get_svr_probability(const struct svm_model *model);

double svm_predict_values(const struct svm_model *model, const struct svm_node *x, double *dec_values);
double svm_predict(const struct svm_model *model, const struct svm_node *x);
double svm_predict_probability(const struct svm_model *model, const struct svm_node *x, double *prob_estimates);

void svm_free_model_content(struct svm_model *model_ptr);
void svm_free_and_destroy_model(struct svm_model **model_ptr_ptr);
void svm_destroy_param(struct svm_parameter *param);

const char *svm_check_parameter(const struct svm_problem *prob, const struct svm_parameter *param);
int svm_check_probability_model(const struct svm_model *model);

void svm_set_print_string_function(void (*print_func)(const char *));

#ifdef __cplusplus
}
#endif

#endif /* LIBSVM_B200_SVM_H */
