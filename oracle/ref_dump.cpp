// Test infrastructure only: runs the reference's own libsvm CPU solver
// (reference libsvm/svm.cpp, built from the reference's sources by
// oracle/Makefile into oracle/_ref/) on one libsvm text file and dumps
// everything the parity tests compare: the model (rho, sv_coef, sv_indices,
// nSV, labels), the solver's #iter/obj per binary subproblem, decision values
// and labels for an optional test file (and class probabilities of a model
// trained with -b 1), or cross-validation targets.
//
// usage: ref_dump [svm-train options] train_file [test_file]
//        ref_dump -v nfold [options] train_file      (cross validation)
#include "svm.h"
#include "dump_common.h"

int main(int argc, char **argv)
{
    struct svm_parameter param;
    int nr_fold = 0, first = 0;
    if (dump_parse_options(argc, argv, &param, &nr_fold, &first) != 0 || first >= argc) {
        fprintf(stderr, "usage: ref_dump [options] train_file [test_file]\n");
        return 1;
    }
    dump_problem tr;
    if (dump_read_problem(argv[first], &tr) != 0) { fprintf(stderr, "cannot read %s\n", argv[first]); return 1; }
    if (param.gamma == 0 && tr.max_index > 0) param.gamma = 1.0 / tr.max_index;
    struct svm_problem prob;
    prob.l = tr.l; prob.y = tr.y; prob.x = tr.x;
    const char *err = svm_check_parameter(&prob, &param);
    if (err) { printf("error %s\n", err); return 2; }
    svm_set_print_string_function(dump_capture);
    if (nr_fold > 0) {
        double *target = (double *)malloc(sizeof(double) * (tr.l ? tr.l : 1));
        svm_cross_validation(&prob, &param, nr_fold, target);
        for (int i = 0; i < tr.l; i++) printf("cv %d %.17g\n", i, target[i]);
        dump_solver_log(stdout);
        return 0;
    }
    struct svm_model *model = svm_train(&prob, &param);
    dump_model(stdout, model);
    dump_solver_log(stdout);
    if (first + 1 < argc) {
        dump_problem te;
        if (dump_read_problem(argv[first + 1], &te) != 0) { fprintf(stderr, "cannot read %s\n", argv[first + 1]); return 1; }
        int k = model->nr_class;
        int npair = k * (k - 1) / 2;
        double *dec = (double *)malloc(sizeof(double) * (npair > 0 ? npair : 1));
        for (int i = 0; i < te.l; i++) {
            double lab = svm_predict_values(model, te.x[i], dec);
            printf("dec %d %.17g", i, lab);
            for (int p = 0; p < npair; p++) printf(" %.17g", dec[p]);
            printf("\n");
        }
        free(dec);
        /* class probabilities (svm_predict_probability) of a model trained with -b 1 */
        if (svm_check_probability_model(model) &&
            (svm_get_svm_type(model) == C_SVC || svm_get_svm_type(model) == NU_SVC)) {
            double *pe = (double *)malloc(sizeof(double) * (k > 0 ? k : 1));
            for (int i = 0; i < te.l; i++) {
                double lab = svm_predict_probability(model, te.x[i], pe);
                printf("prob %d %.17g", i, lab);
                for (int c = 0; c < k; c++) printf(" %.17g", pe[c]);
                printf("\n");
            }
            free(pe);
        }
    }
    svm_free_and_destroy_model(&model);
    return 0;
}
