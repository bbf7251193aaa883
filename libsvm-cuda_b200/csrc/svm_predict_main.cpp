// svm-predict -- prediction from a model file for a whole test file in one
// batched device pass (the reference ships no prediction command; this one
// follows libsvm's usual conventions).
//
//   svm-predict [-b 0|1] [-q] test_file model_file output_file
//
// The model is read with svm_load_model (the reference's model format,
// svm.cpp:2941-3044), the test file with svmb_read_problem (the training
// file's rules), and all rows are predicted with one svmb_predict_batch /
// svmb_predict_probability_batch call (decision values of the reference's
// svm_predict_values / svm_predict_probability, svm.cpp:2569-2697).
// Output, one line per test row: the predicted label or value (%.17g); with
// -b 1 on a classifier, a first line "labels <l1> ... <lk>" and then the
// label followed by the k class probabilities.  The summary (accuracy, or
// mean squared error and squared correlation for regression) goes to stdout
// unless -q.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "svm.h"
#include "svm_b200.h"

namespace {

[[noreturn]] void usage()
{
    printf("Usage: svm-predict [options] test_file model_file output_file\n"
           "options:\n"
           "-b probability_estimates: whether to predict probability estimates, 0 or 1 (default 0)\n"
           "-q : quiet mode (no outputs)\n");
    exit(1);
}

}  // namespace

int main(int argc, char **argv)
{
    int probability = 0;
    bool quiet = false;
    int i = 1;
    for (; i < argc && argv[i][0] == '-'; i++) {
        if (argv[i][1] == 'q') {
            quiet = true;
            continue;
        }
        if (argv[i][1] != 'b' || i + 1 >= argc) {
            if (argv[i][1] != 'b') fprintf(stderr, "Unknown option: -%c\n", argv[i][1]);
            usage();
        }
        probability = atoi(argv[++i]);
    }
    if (argc - i != 3) usage();
    const char *test_path = argv[i], *model_path = argv[i + 1], *out_path = argv[i + 2];
    auto say = [&](const char *s) {
        if (!quiet) fputs(s, stdout);
    };
    svm_model *model = svm_load_model(model_path);
    if (!model) {
        fprintf(stderr, "can't open model file %s\n", model_path);
        exit(1);
    }
    const int type = svm_get_svm_type(model);
    const bool classifier = type == C_SVC || type == NU_SVC;
    const bool regression = type == EPSILON_SVR || type == NU_SVR;
    if (probability) {
        if (!svm_check_probability_model(model)) {
            fprintf(stderr, "Model does not support probabiliy estimates\n");
            exit(1);
        }
    } else if (svm_check_probability_model(model)) {
        say("Model supports probability estimates, but disabled in prediction.\n");
    }
    svm_problem test{};
    svm_node *space = nullptr;
    long long bad = 0;
    const int rc = svmb_read_problem(test_path, &test, &space, nullptr, &bad);
    if (rc == -2) {
        fprintf(stderr, "Wrong input format at line %lld\n", bad);
        exit(1);
    }
    if (rc != 0) {
        fprintf(stderr, "can't open input file %s\n", test_path);
        exit(1);
    }
    FILE *out = fopen(out_path, "w");
    if (!out) {
        fprintf(stderr, "can't open output file %s\n", out_path);
        exit(1);
    }
    const int n = test.l, k = svm_get_nr_class(model);
    std::vector<double> label(n > 0 ? n : 1);
    std::vector<double> prob;
    int ok;
    if (probability && classifier) {
        prob.resize((size_t)(n > 0 ? n : 1) * k);
        ok = svmb_predict_probability_batch(model, test.x, n, label.data(), prob.data());
    } else {
        ok = svmb_predict_batch(model, test.x, n, label.data(), nullptr);
    }
    if (ok != 0) {
        fprintf(stderr, "ERROR: %s\n", svmb_last_error());
        exit(1);
    }
    if (probability && regression) {
        char buf[256];
        snprintf(buf, sizeof buf,
                 "Prob. model for test data: target value = predicted value + z,\nz: Laplace distribution "
                 "e^(-|z|/sigma)/(2sigma),sigma=%g\n", svm_get_svr_probability(model));
        say(buf);
    }
    if (probability && classifier) {
        std::vector<int> labels(k);
        svm_get_labels(model, labels.data());
        fprintf(out, "labels");
        for (int c = 0; c < k; c++) fprintf(out, " %d", labels[c]);
        fprintf(out, "\n");
    }
    int correct = 0;
    double se = 0, sv = 0, sy = 0, svv = 0, syy = 0, svy = 0;
    for (int t = 0; t < n; t++) {
        fprintf(out, "%.17g", label[t]);
        if (probability && classifier)
            for (int c = 0; c < k; c++) fprintf(out, " %.17g", prob[(size_t)t * k + c]);
        fprintf(out, "\n");
        const double v = label[t], y = test.y[t];
        correct += v == y;
        se += (v - y) * (v - y);
        sv += v;
        sy += y;
        svv += v * v;
        syy += y * y;
        svy += v * y;
    }
    fclose(out);
    char buf[256];
    if (regression) {
        snprintf(buf, sizeof buf, "Mean squared error = %g (regression)\n", n ? se / n : 0.0);
        say(buf);
        snprintf(buf, sizeof buf, "Squared correlation coefficient = %g (regression)\n",
                 ((n * svy - sv * sy) * (n * svy - sv * sy)) / ((n * svv - sv * sv) * (n * syy - sy * sy)));
        say(buf);
    } else {
        snprintf(buf, sizeof buf, "Accuracy = %g%% (%d/%d) (classification)\n", n ? 100.0 * correct / n : 0.0,
                 correct, n);
        say(buf);
    }
    svm_free_and_destroy_model(&model);
    svmb_free_problem(&test, space);
    return 0;
}
