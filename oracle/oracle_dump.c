#define _POSIX_C_SOURCE 200809L
/* Test infrastructure only: the restatement's twin of ref_dump.cpp.  Same
 * options, same output records, so that the two can be compared line by line.
 * The objective is printed after a round trip through "%f" because that is the
 * precision the reference reports it with (svm.cpp:1739). */
#include "svm_oracle.h"
#include "dump_common.h"

int main(int argc, char **argv)
{
    struct svm_parameter param;
    int nr_fold = 0, first = 0;
    if (dump_parse_options(argc, argv, &param, &nr_fold, &first) != 0 || first >= argc) {
        fprintf(stderr, "usage: oracle_dump [options] train_file [test_file]\n");
        return 1;
    }
    dump_problem tr;
    if (dump_read_problem(argv[first], &tr) != 0) { fprintf(stderr, "cannot read %s\n", argv[first]); return 1; }
    if (param.gamma == 0 && tr.max_index > 0) param.gamma = 1.0 / tr.max_index;
    struct svm_problem prob;
    prob.l = tr.l; prob.y = tr.y; prob.x = tr.x;
    if (nr_fold > 0) {
        double *target = (double *)malloc(sizeof(double) * (tr.l ? tr.l : 1));
        oracle_cross_validation(&prob, &param, nr_fold, target);
        for (int i = 0; i < tr.l; i++) printf("cv %d %.17g\n", i, target[i]);
    } else {
        struct svm_model *model = oracle_svm_train(&prob, &param);
        dump_model(stdout, model);
        if (first + 1 < argc) {
            /* decision values are printed after the solver log, below */
        }
        int n = oracle_solve_count();
        for (int k = 0; k < n; k++) { oracle_solve_info s; oracle_solve_get(k, &s); printf("iter %d %lld\n", k, s.iters); }
        for (int k = 0; k < n; k++) {
            oracle_solve_info s; oracle_solve_get(k, &s);
            char buf[64]; snprintf(buf, sizeof buf, "%f", s.obj);
            printf("obj %d %.17g\n", k, strtod(buf, NULL));
        }
        if (first + 1 < argc) {
            dump_problem te;
            if (dump_read_problem(argv[first + 1], &te) != 0) { fprintf(stderr, "cannot read %s\n", argv[first + 1]); return 1; }
            int k = model->nr_class, npair = k * (k - 1) / 2;
            double *dec = (double *)malloc(sizeof(double) * (npair > 0 ? npair : 1));
            for (int i = 0; i < te.l; i++) {
                double lab = oracle_predict_values(model, te.x[i], dec);
                printf("dec %d %.17g", i, lab);
                for (int p = 0; p < npair; p++) printf(" %.17g", dec[p]);
                printf("\n");
            }
            free(dec);
        }
        oracle_free_model(model);
        return 0;
    }
    int n = oracle_solve_count();
    for (int k = 0; k < n; k++) { oracle_solve_info s; oracle_solve_get(k, &s); printf("iter %d %lld\n", k, s.iters); }
    for (int k = 0; k < n; k++) {
        oracle_solve_info s; oracle_solve_get(k, &s);
        char buf[64]; snprintf(buf, sizeof buf, "%f", s.obj);
        printf("obj %d %.17g\n", k, strtod(buf, NULL));
    }
    return 0;
}
