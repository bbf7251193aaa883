/* svm-train -- command line front end of the B200 engine.
 *
 * Same options, input format, defaults and outputs as the reference CLI
 * (reference svm-train/svm-train.c:10-389): libsvm sparse text in, model file
 * out (or "-v n" cross-validation accuracy).  -C is accepted for
 * compatibility; training always runs on the GPU and, unlike the reference
 * (svm-train.c:260-262), -C does not switch shrinking off.
 */
#define _POSIX_C_SOURCE 200809L
#include <ctype.h>
#include <errno.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "svm.h"

static void print_null(const char *s) { (void)s; }

static void exit_with_help(void)
{
    printf(
        "Usage: svm-train [options] training_set_file [model_file]\n"
        "options:\n"
        "-C : accepted for compatibility (training always runs on the GPU)\n"
        "-s svm_type : set type of SVM (default 0)\n"
        "	0 -- C-SVC		(multi-class classification)\n"
        "	1 -- nu-SVC		(multi-class classification)\n"
        "-t kernel_type : set type of kernel function (default 2)\n"
        "	0 -- linear: u'*v\n"
        "	1 -- polynomial: (gamma*u'*v + coef0)^degree\n"
        "	2 -- radial basis function: exp(-gamma*|u-v|^2)\n"
        "	3 -- sigmoid: tanh(gamma*u'*v + coef0)\n"
        "-d degree : set degree in kernel function (default 3)\n"
        "-g gamma : set gamma in kernel function (default 1/num_features)\n"
        "-r coef0 : set coef0 in kernel function (default 0)\n"
        "-c cost : set the parameter C of C-SVC (default 1)\n"
        "-n nu : set the parameter nu of nu-SVC (default 0.5)\n"
        "-m cachesize : set cache memory size in MB (default 100)\n"
        "-e epsilon : set tolerance of termination criterion (default 0.001)\n"
        "-h shrinking : whether to use the shrinking heuristics, 0 or 1 (default 1)\n"
        "-b probability_estimates : accepted, not trained (default 0)\n"
        "-wi weight : set the parameter C of class i to weight*C, for C-SVC (default 1)\n"
        "-v n: n-fold cross validation mode\n"
        "-q : quiet mode (no outputs)\n");
    exit(1);
}

static void exit_input_error(int line_num)
{
    fprintf(stderr, "Wrong input format at line %d\n", line_num);
    exit(1);
}

static struct svm_parameter param;
static struct svm_problem prob;
static struct svm_node *x_space;
static int cross_validation, nr_fold;

static char *line;
static size_t max_line_len;

static char *readline(FILE *input)
{
    if (fgets(line, (int)max_line_len, input) == NULL) return NULL;
    while (strrchr(line, '\n') == NULL) {
        max_line_len *= 2;
        line = (char *)realloc(line, max_line_len);
        size_t len = strlen(line);
        if (fgets(line + len, (int)(max_line_len - len), input) == NULL) break;
    }
    return line;
}

static void parse_command_line(int argc, char **argv, char *input_file_name, char *model_file_name)
{
    void (*print_func)(const char *) = NULL;
    memset(&param, 0, sizeof param);
    param.cuda_flag = 0;
    param.svm_type = C_SVC;
    param.kernel_type = RBF;
    param.degree = 3;
    param.gamma = 0;
    param.coef0 = 0;
    param.nu = 0.5;
    param.cache_size = 100;
    param.C = 1;
    param.eps = 1e-3;
    param.p = 0.1;
    param.shrinking = 1;
    param.probability = 0;
    param.nr_weight = 0;
    param.weight_label = NULL;
    param.weight = NULL;
    cross_validation = 0;
    int i;
    for (i = 1; i < argc; i++) {
        if (argv[i][0] != '-') break;
        if (argv[i][1] == 'C') { param.cuda_flag = 1; continue; }
        if (argv[i][1] == 'q') { print_func = &print_null; continue; }
        if (++i >= argc) exit_with_help();
        switch (argv[i - 1][1]) {
        case 's': param.svm_type = atoi(argv[i]); break;
        case 't': param.kernel_type = atoi(argv[i]); break;
        case 'd': param.degree = atoi(argv[i]); break;
        case 'g': param.gamma = atof(argv[i]); break;
        case 'r': param.coef0 = atof(argv[i]); break;
        case 'n': param.nu = atof(argv[i]); break;
        case 'm': param.cache_size = atof(argv[i]); break;
        case 'c': param.C = atof(argv[i]); break;
        case 'e': param.eps = atof(argv[i]); break;
        case 'p': param.p = atof(argv[i]); break;
        case 'h': param.shrinking = atoi(argv[i]); break;
        case 'b': param.probability = atoi(argv[i]); break;
        case 'v':
            cross_validation = 1;
            nr_fold = atoi(argv[i]);
            if (nr_fold < 2) {
                fprintf(stderr, "n-fold cross validation: n must >= 2\n");
                exit_with_help();
            }
            break;
        case 'w':
            ++param.nr_weight;
            param.weight_label = (int *)realloc(param.weight_label, sizeof(int) * param.nr_weight);
            param.weight = (double *)realloc(param.weight, sizeof(double) * param.nr_weight);
            param.weight_label[param.nr_weight - 1] = atoi(&argv[i - 1][2]);
            param.weight[param.nr_weight - 1] = atof(argv[i]);
            break;
        default:
            fprintf(stderr, "Unknown option: -%c\n", argv[i - 1][1]);
            exit_with_help();
        }
    }
    svm_set_print_string_function(print_func);
    if (i >= argc) exit_with_help();
    strcpy(input_file_name, argv[i]);
    if (i < argc - 1) {
        strcpy(model_file_name, argv[i + 1]);
    } else {
        char *p = strrchr(argv[i], '/');
        p = p == NULL ? argv[i] : p + 1;
        sprintf(model_file_name, "%s.model", p);
    }
}

/* libsvm sparse text, same acceptance rules as the reference (svm-train.c:288-389) */
static void read_problem(const char *filename)
{
    FILE *fp = fopen(filename, "r");
    if (fp == NULL) {
        fprintf(stderr, "can't open input file %s\n", filename);
        exit(1);
    }
    long elements = 0;
    prob.l = 0;
    max_line_len = 1024;
    line = (char *)malloc(max_line_len);
    while (readline(fp) != NULL) {
        char *save = NULL;
        char *p = strtok_r(line, " \t", &save);
        (void)p;
        while (1) {
            p = strtok_r(NULL, " \t", &save);
            if (p == NULL || *p == '\n') break;
            ++elements;
        }
        ++elements;
        ++prob.l;
    }
    rewind(fp);
    prob.y = (double *)malloc(sizeof(double) * (prob.l ? prob.l : 1));
    prob.x = (struct svm_node **)malloc(sizeof(struct svm_node *) * (prob.l ? prob.l : 1));
    x_space = (struct svm_node *)malloc(sizeof(struct svm_node) * (elements ? elements : 1));
    int max_index = 0;
    long j = 0;
    for (int i = 0; i < prob.l; i++) {
        int inst_max_index = -1;
        char *endptr, *save = NULL;
        readline(fp);
        prob.x[i] = &x_space[j];
        char *label = strtok_r(line, " \t\n", &save);
        if (label == NULL) exit_input_error(i + 1);
        prob.y[i] = strtod(label, &endptr);
        if (endptr == label || *endptr != '\0') exit_input_error(i + 1);
        while (1) {
            char *idx = strtok_r(NULL, ":", &save);
            char *val = strtok_r(NULL, " \t", &save);
            if (val == NULL) break;
            errno = 0;
            x_space[j].index = (int)strtol(idx, &endptr, 10);
            if (endptr == idx || errno != 0 || *endptr != '\0' || x_space[j].index <= inst_max_index)
                exit_input_error(i + 1);
            inst_max_index = x_space[j].index;
            errno = 0;
            x_space[j].value = strtod(val, &endptr);
            if (endptr == val || errno != 0 || (*endptr != '\0' && !isspace((unsigned char)*endptr)))
                exit_input_error(i + 1);
            ++j;
        }
        if (inst_max_index > max_index) max_index = inst_max_index;
        x_space[j++].index = -1;
    }
    if (param.gamma == 0 && max_index > 0) param.gamma = 1.0 / max_index;
    fclose(fp);
}

static void do_cross_validation(void)
{
    int total_correct = 0;
    double *target = (double *)malloc(sizeof(double) * (prob.l ? prob.l : 1));
    svm_cross_validation(&prob, &param, nr_fold, target);
    for (int i = 0; i < prob.l; i++)
        if (target[i] == prob.y[i]) ++total_correct;
    printf("Cross Validation Accuracy = %g%%\n", 100.0 * total_correct / prob.l);
    free(target);
}

int main(int argc, char **argv)
{
    char input_file_name[1024];
    char model_file_name[1024];
    parse_command_line(argc, argv, input_file_name, model_file_name);
    read_problem(input_file_name);
    const char *error_msg = svm_check_parameter(&prob, &param);
    if (error_msg) {
        fprintf(stderr, "ERROR: %s\n", error_msg);
        exit(1);
    }
    if (cross_validation) {
        do_cross_validation();
    } else {
        struct svm_model *model = svm_train(&prob, &param);
        if (model == NULL) {
            fprintf(stderr, "ERROR: training failed\n");
            exit(1);
        }
        if (svm_save_model(model_file_name, model)) {
            fprintf(stderr, "can't save model to file %s\n", model_file_name);
            exit(1);
        }
        svm_free_and_destroy_model(&model);
    }
    svm_destroy_param(&param);
    free(prob.y);
    free(prob.x);
    free(x_space);
    free(line);
    return 0;
}
