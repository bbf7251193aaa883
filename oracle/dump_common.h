// Test infrastructure only: shared by the oracle dump programs (ref_dump.cpp,
// which links the reference's own CPU solver, and oracle_dump.c, which links
// the restatement in svm_oracle.c).  Nothing in the product links this file.
//
// Input format: libsvm sparse text ("label idx:val idx:val ...").  Options are
// the svm-train options (reference svm-train/svm-train.c:162-284) minus -C/-q.
// Output: one record per line, numbers printed with %.17g so doubles round-trip.
#ifndef ORACLE_DUMP_COMMON_H
#define ORACLE_DUMP_COMMON_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int l;
    double *y;
    struct svm_node **x;
    struct svm_node *space;
    int max_index;
} dump_problem;

/* Parse one libsvm text file; the same acceptance rules as the reference's
 * read_problem (svm-train.c:288-389): indices strictly ascending per row. */
static int dump_read_problem(const char *path, dump_problem *out)
{
    FILE *fp = fopen(path, "r");
    if (!fp) return -1;
    size_t cap_rows = 1024, cap_nodes = 1 << 16, nrows = 0, nnodes = 0;
    double *y = (double *)malloc(cap_rows * sizeof(double));
    size_t *start = (size_t *)malloc(cap_rows * sizeof(size_t));
    struct svm_node *space = (struct svm_node *)malloc(cap_nodes * sizeof(struct svm_node));
    int max_index = 0;
    size_t linecap = 1 << 16;
    char *line = (char *)malloc(linecap);
    while (1) {
        size_t len = 0;
        int got = 0;
        for (;;) {
            if (!fgets(line + len, (int)(linecap - len), fp)) break;
            got = 1;
            len += strlen(line + len);
            if (len > 0 && line[len - 1] == '\n') break;
            linecap *= 2;
            line = (char *)realloc(line, linecap);
        }
        if (!got) break;
        char *save = NULL;
        char *tok = strtok_r(line, " \t\n", &save);
        if (!tok) continue;
        if (nrows == cap_rows) {
            cap_rows *= 2;
            y = (double *)realloc(y, cap_rows * sizeof(double));
            start = (size_t *)realloc(start, cap_rows * sizeof(size_t));
        }
        y[nrows] = strtod(tok, NULL);
        start[nrows] = nnodes;
        int last = -1;
        while ((tok = strtok_r(NULL, " \t\n", &save)) != NULL) {
            char *colon = strchr(tok, ':');
            if (!colon) break;
            *colon = 0;
            int idx = (int)strtol(tok, NULL, 10);
            double v = strtod(colon + 1, NULL);
            if (idx <= last) { fclose(fp); return -2; }
            last = idx;
            if (nnodes + 2 > cap_nodes) {
                cap_nodes *= 2;
                space = (struct svm_node *)realloc(space, cap_nodes * sizeof(struct svm_node));
            }
            space[nnodes].index = idx;
            space[nnodes].value = v;
            nnodes++;
            if (idx > max_index) max_index = idx;
        }
        if (nnodes + 1 > cap_nodes) {
            cap_nodes *= 2;
            space = (struct svm_node *)realloc(space, cap_nodes * sizeof(struct svm_node));
        }
        space[nnodes].index = -1;
        space[nnodes].value = 0;
        nnodes++;
        nrows++;
    }
    fclose(fp);
    free(line);
    out->l = (int)nrows;
    out->y = y;
    out->space = space;
    out->x = (struct svm_node **)malloc((nrows ? nrows : 1) * sizeof(struct svm_node *));
    for (size_t i = 0; i < nrows; i++) out->x[i] = space + start[i];
    free(start);
    out->max_index = max_index;
    return 0;
}

/* svm-train defaults and option letters (reference svm-train.c:167-245). */
static int dump_parse_options(int argc, char **argv, struct svm_parameter *param, int *nr_fold, int *first_file)
{
    memset(param, 0, sizeof(*param));
    param->svm_type = C_SVC;
    param->kernel_type = RBF;
    param->degree = 3;
    param->gamma = 0;
    param->coef0 = 0;
    param->nu = 0.5;
    param->cache_size = 100;
    param->C = 1;
    param->eps = 1e-3;
    param->p = 0.1;
    param->shrinking = 1;
    param->probability = 0;
    *nr_fold = 0;
    int i;
    for (i = 1; i < argc; i++) {
        if (argv[i][0] != '-') break;
        if (i + 1 >= argc) return -1;
        const char *v = argv[i + 1];
        switch (argv[i][1]) {
        case 's': param->svm_type = atoi(v); break;
        case 't': param->kernel_type = atoi(v); break;
        case 'd': param->degree = atoi(v); break;
        case 'g': param->gamma = atof(v); break;
        case 'r': param->coef0 = atof(v); break;
        case 'n': param->nu = atof(v); break;
        case 'm': param->cache_size = atof(v); break;
        case 'c': param->C = atof(v); break;
        case 'e': param->eps = atof(v); break;
        case 'p': param->p = atof(v); break;
        case 'h': param->shrinking = atoi(v); break;
        case 'b': param->probability = atoi(v); break;
        case 'v': *nr_fold = atoi(v); break;
        case 'w':
            param->nr_weight++;
            param->weight_label = (int *)realloc(param->weight_label, sizeof(int) * param->nr_weight);
            param->weight = (double *)realloc(param->weight, sizeof(double) * param->nr_weight);
            param->weight_label[param->nr_weight - 1] = atoi(&argv[i][2]);
            param->weight[param->nr_weight - 1] = atof(v);
            break;
        default: return -1;
        }
        i++;
    }
    *first_file = i;
    return 0;
}

static void dump_model(FILE *out, const struct svm_model *m)
{
    int k = m->nr_class;
    int npair = k * (k - 1) / 2;
    fprintf(out, "nr_class %d\n", k);
    fprintf(out, "total_sv %d\n", m->l);
    if (m->label) {
        fprintf(out, "labels");
        for (int i = 0; i < k; i++) fprintf(out, " %d", m->label[i]);
        fprintf(out, "\n");
    }
    if (m->nSV) {
        fprintf(out, "nsv");
        for (int i = 0; i < k; i++) fprintf(out, " %d", m->nSV[i]);
        fprintf(out, "\n");
    }
    fprintf(out, "rho");
    for (int i = 0; i < npair; i++) fprintf(out, " %.17g", m->rho[i]);
    fprintf(out, "\n");
    if (m->probA) {
        fprintf(out, "probA");
        for (int i = 0; i < npair; i++) fprintf(out, " %.17g", m->probA[i]);
        fprintf(out, "\n");
    }
    if (m->probB) {
        fprintf(out, "probB");
        for (int i = 0; i < npair; i++) fprintf(out, " %.17g", m->probB[i]);
        fprintf(out, "\n");
    }
    fprintf(out, "sv_indices");
    for (int i = 0; i < m->l; i++) fprintf(out, " %d", m->sv_indices[i]);
    fprintf(out, "\n");
    for (int j = 0; j < k - 1; j++) {
        fprintf(out, "sv_coef %d", j);
        for (int i = 0; i < m->l; i++) fprintf(out, " %.17g", m->sv_coef[j][i]);
        fprintf(out, "\n");
    }
}

/* The solver reports "#iter = N" and "obj = X, rho = Y" through the print hook
 * (reference svm.cpp:821 and :1739); collect them in call order. */
static char *dump_log = NULL;
static size_t dump_log_len = 0, dump_log_cap = 0;
static void dump_capture(const char *s)
{
    size_t n = strlen(s);
    if (dump_log_len + n + 1 > dump_log_cap) {
        dump_log_cap = (dump_log_len + n + 1) * 2;
        dump_log = (char *)realloc(dump_log, dump_log_cap);
    }
    memcpy(dump_log + dump_log_len, s, n + 1);
    dump_log_len += n;
}

static void dump_solver_log(FILE *out)
{
    if (!dump_log) return;
    int sub = 0;
    const char *p = dump_log;
    while ((p = strstr(p, "#iter = ")) != NULL) {
        p += 8;
        fprintf(out, "iter %d %ld\n", sub++, strtol(p, NULL, 10));
    }
    sub = 0;
    p = dump_log;
    while ((p = strstr(p, "obj = ")) != NULL) {
        p += 6;
        double obj = strtod(p, NULL);
        fprintf(out, "obj %d %.17g\n", sub++, obj);
    }
}

#endif
