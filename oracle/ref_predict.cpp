// Test infrastructure only: prediction from a model file by the reference's
// own svm.cpp (built from the reference sources into oracle/_ref/), one row at
// a time through svm_predict / svm_predict_probability (reference
// libsvm/svm.cpp:2569-2697), writing the output format of the engine's
// svm-predict command so the two files can be compared byte for byte:
//   one line per test row: the label or value (%.17g); with -b 1 on a
//   classifier a first line "labels <l1> ... <lk>" and then the label and the
//   k class probabilities.
//
// usage: ref_predict [-b 0|1] test_file model_file output_file
#include "svm.h"
#include "dump_common.h"

int main(int argc, char **argv)
{
    int probability = 0, i = 1;
    if (argc > 2 && !strcmp(argv[1], "-b")) {
        probability = atoi(argv[2]);
        i = 3;
    }
    if (argc - i != 3) {
        fprintf(stderr, "usage: ref_predict [-b 0|1] test_file model_file output_file\n");
        return 1;
    }
    struct svm_model *model = svm_load_model(argv[i + 1]);
    if (!model) { fprintf(stderr, "can't open model file %s\n", argv[i + 1]); return 1; }
    dump_problem te;
    if (dump_read_problem(argv[i], &te) != 0) { fprintf(stderr, "cannot read %s\n", argv[i]); return 1; }
    FILE *out = fopen(argv[i + 2], "w");
    if (!out) return 1;
    int type = svm_get_svm_type(model), k = svm_get_nr_class(model);
    int classifier = type == C_SVC || type == NU_SVC;
    double *pe = (double *)malloc(sizeof(double) * (k > 0 ? k : 1));
    if (probability && classifier) {
        int *labels = (int *)malloc(sizeof(int) * (k > 0 ? k : 1));
        svm_get_labels(model, labels);
        fprintf(out, "labels");
        for (int c = 0; c < k; c++) fprintf(out, " %d", labels[c]);
        fprintf(out, "\n");
        free(labels);
    }
    for (int t = 0; t < te.l; t++) {
        if (probability && classifier) {
            double lab = svm_predict_probability(model, te.x[t], pe);
            fprintf(out, "%.17g", lab);
            for (int c = 0; c < k; c++) fprintf(out, " %.17g", pe[c]);
            fprintf(out, "\n");
        } else {
            fprintf(out, "%.17g\n", svm_predict(model, te.x[t]));
        }
    }
    fclose(out);
    free(pe);
    svm_free_and_destroy_model(&model);
    return 0;
}
