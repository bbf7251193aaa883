// svm-train -- the reference's training command line (svm-train/svm-train.c)
// on the GPU engine: same options, defaults, files and messages; input parsed
// by all host threads (svmb_read_problem), training through svm.h.
//
// What is kept identical because it is interface: the usage text, the option
// letters and their argument rules (an option's second character selects it;
// every option but -C takes the next argument, -q needs one more argument to
// follow it; -wN weight), the default model file name (<input basename>.model),
// the messages and exit codes, and the cross-validation report lines.
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "svm.h"
#include "svm_b200.h"

namespace {

const char kUsage[] =
    "Usage: svm-train [options] training_set_file [model_file]\n"
    "options:\n"
    "-C cuda integration (exerimental)\n"
    "-s svm_type : set type of SVM (default 0)\n"
    "\t0 -- C-SVC\t\t(multi-class classification)\n"
    "\t1 -- nu-SVC\t\t(multi-class classification)\n"
    "\t2 -- one-class SVM\n"
    "\t3 -- epsilon-SVR\t(regression)\n"
    "\t4 -- nu-SVR\t\t(regression)\n"
    "-t kernel_type : set type of kernel function (default 2)\n"
    "\t0 -- linear: u'*v\n"
    "\t1 -- polynomial: (gamma*u'*v + coef0)^degree\n"
    "\t2 -- radial basis function: exp(-gamma*|u-v|^2)\n"
    "\t3 -- sigmoid: tanh(gamma*u'*v + coef0)\n"
    "\t4 -- precomputed kernel (kernel values in training_set_file)\n"
    "-d degree : set degree in kernel function (default 3)\n"
    "-g gamma : set gamma in kernel function (default 1/num_features)\n"
    "-r coef0 : set coef0 in kernel function (default 0)\n"
    "-c cost : set the parameter C of C-SVC, epsilon-SVR, and nu-SVR (default 1)\n"
    "-n nu : set the parameter nu of nu-SVC, one-class SVM, and nu-SVR (default 0.5)\n"
    "-p epsilon : set the epsilon in loss function of epsilon-SVR (default 0.1)\n"
    "-m cachesize : set cache memory size in MB (default 100)\n"
    "-e epsilon : set tolerance of termination criterion (default 0.001)\n"
    "-h shrinking : whether to use the shrinking heuristics, 0 or 1 (default 1)\n"
    "-b probability_estimates : whether to train a SVC or SVR model for probability estimates, 0 or 1 (default 0)\n"
    "-wi weight : set the parameter C of class i to weight*C, for C-SVC (default 1)\n"
    "-v n: n-fold cross validation mode\n"
    "-q : quiet mode (no outputs)\n";

[[noreturn]] void usage()
{
    fputs(kUsage, stdout);
    exit(1);
}

struct Job {
    svm_parameter param{};
    std::vector<int> wlabel;
    std::vector<double> wvalue;
    int nr_fold = 0;             // > 0: cross-validation
    bool quiet = false;
    std::string input, model;
};

void defaults(svm_parameter &p)
{
    memset(&p, 0, sizeof p);
    p.svm_type = C_SVC;
    p.kernel_type = RBF;
    p.degree = 3;
    p.gamma = 0;                 // 1/num_features once the data is read
    p.nu = 0.5;
    p.cache_size = 100;
    p.C = 1;
    p.eps = 1e-3;
    p.p = 0.1;
    p.shrinking = 1;
}

Job parse_args(int argc, char **argv)
{
    Job job;
    svm_parameter &p = job.param;
    defaults(p);
    int i = 1;
    for (; i < argc && argv[i][0] == '-'; i++) {
        const char opt = argv[i][1];
        if (opt == 'C') {        // the reference's GPU switch (no argument)
            p.cuda_flag = 1;
            continue;
        }
        if (i + 1 >= argc) usage();
        if (opt == 'q') {        // no argument of its own, but one must follow
            job.quiet = true;
            continue;
        }
        const char *v = argv[++i];
        switch (opt) {
        case 's': p.svm_type = atoi(v); break;
        case 't': p.kernel_type = atoi(v); break;
        case 'd': p.degree = atoi(v); break;
        case 'g': p.gamma = atof(v); break;
        case 'r': p.coef0 = atof(v); break;
        case 'n': p.nu = atof(v); break;
        case 'm': p.cache_size = atof(v); break;
        case 'c': p.C = atof(v); break;
        case 'e': p.eps = atof(v); break;
        case 'p': p.p = atof(v); break;
        case 'h': p.shrinking = atoi(v); break;
        case 'b': p.probability = atoi(v); break;
        case 'v':
            job.nr_fold = atoi(v);
            if (job.nr_fold < 2) {
                fprintf(stderr, "n-fold cross validation: n must >= 2\n");
                usage();
            }
            break;
        case 'w':
            job.wlabel.push_back(atoi(argv[i - 1] + 2));
            job.wvalue.push_back(atof(v));
            break;
        default:
            fprintf(stderr, "Unknown option: -%c\n", opt);
            usage();
        }
    }
    // the reference's GPU solver runs without shrinking
    if (p.cuda_flag == 1) p.shrinking = 0;
    if (i >= argc) usage();
    job.input = argv[i];
    if (i + 1 < argc) {
        job.model = argv[i + 1];
    } else {
        const char *slash = strrchr(argv[i], '/');
        job.model = std::string(slash ? slash + 1 : argv[i]) + ".model";
    }
    p.nr_weight = (int)job.wlabel.size();
    p.weight_label = job.wlabel.empty() ? nullptr : job.wlabel.data();
    p.weight = job.wvalue.empty() ? nullptr : job.wvalue.data();
    return job;
}

void report_cross_validation(const svm_problem &prob, const svm_parameter &p, const std::vector<double> &target)
{
    const int l = prob.l;
    if (p.svm_type == EPSILON_SVR || p.svm_type == NU_SVR) {
        // mean squared error and squared correlation of predictions and targets
        double se = 0, sv = 0, sy = 0, svv = 0, syy = 0, svy = 0;
        for (int i = 0; i < l; i++) {
            const double y = prob.y[i], v = target[i];
            se += (v - y) * (v - y);
            sv += v;
            sy += y;
            svv += v * v;
            syy += y * y;
            svy += v * y;
        }
        printf("Cross Validation Mean squared error = %g\n", se / l);
        printf("Cross Validation Squared correlation coefficient = %g\n",
               ((l * svy - sv * sy) * (l * svy - sv * sy)) / ((l * svv - sv * sv) * (l * syy - sy * sy)));
        return;
    }
    int correct = 0;
    for (int i = 0; i < l; i++) correct += target[i] == prob.y[i];
    printf("Cross Validation Accuracy = %g%%\n", 100.0 * correct / l);
}

}  // namespace

int main(int argc, char **argv)
{
    Job job = parse_args(argc, argv);
    svm_set_print_string_function(job.quiet ? svmb_print_nothing : nullptr);
    svm_problem prob{};
    svm_node *space = nullptr;
    int max_index = 0;
    long long bad = 0;
    const int rc = svmb_read_problem(job.input.c_str(), &prob, &space, &max_index, &bad);
    if (rc == -2) {
        fprintf(stderr, "Wrong input format at line %lld\n", bad);
        exit(1);
    }
    if (rc != 0) {
        fprintf(stderr, "can't open input file %s\n", job.input.c_str());
        exit(1);
    }
    svm_parameter &p = job.param;
    if (p.gamma == 0 && max_index > 0) p.gamma = 1.0 / max_index;
    if (p.kernel_type == PRECOMPUTED)
        for (int i = 0; i < prob.l; i++) {
            if (prob.x[i][0].index != 0) {
                fprintf(stderr, "Wrong input format: first column must be 0:sample_serial_number\n");
                exit(1);
            }
            if ((int)prob.x[i][0].value <= 0 || (int)prob.x[i][0].value > max_index) {
                fprintf(stderr, "Wrong input format: sample_serial_number out of range\n");
                exit(1);
            }
        }
    if (const char *msg = svm_check_parameter(&prob, &p)) {
        fprintf(stderr, "ERROR: %s\n", msg);
        exit(1);
    }
    if (job.nr_fold > 0) {
        std::vector<double> target(prob.l > 0 ? prob.l : 1);
        svm_cross_validation(&prob, &p, job.nr_fold, target.data());
        report_cross_validation(prob, p, target);
    } else {
        svm_model *model = svm_train(&prob, &p);
        if (!model) {
            fprintf(stderr, "ERROR: %s\n", svmb_last_error());
            exit(1);
        }
        if (svm_save_model(job.model.c_str(), model)) {
            fprintf(stderr, "can't save model to file %s\n", job.model.c_str());
            exit(1);
        }
        svm_free_and_destroy_model(&model);
    }
    svmb_free_problem(&prob, space);
    return 0;
}
