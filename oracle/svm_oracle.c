/*
 * svm_oracle.c -- TEST INFRASTRUCTURE ONLY (see svm_oracle.h).
 *
 * CPU restatement of the reference's SMO training path.  Every function names
 * the reference lines it follows (paths relative to the reference project).
 * Floating-point expressions keep the reference's operand order and types so
 * that results are bit-identical with the reference built by oracle/Makefile
 * (x86-64, no FMA contraction).
 *
 * Structure differs from the reference where only speed is affected: kernel
 * rows are cached by ORIGINAL row id in original column order and gathered
 * into position order on request, instead of the reference's position-keyed
 * LRU with column swapping (svm.cpp:71-189).  A cached value is a pure
 * function of the two rows, so the cache policy cannot change any result.
 */
#define _POSIX_C_SOURCE 200809L
#include "svm_oracle.h"

#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifdef ORACLE_QDOUBLE
typedef double qval;
#else
typedef float qval;             /* reference svm.cpp:16 */
#endif

#define ORC_INF HUGE_VAL
#define ORC_TAU 1e-12           /* reference svm.cpp:42 */

enum { ST_LOWER = 0, ST_UPPER = 1, ST_FREE = 2 };   /* reference svm.cpp:425 */

/* ------------------------------------------------------------------ */
/* solve records                                                       */
/* ------------------------------------------------------------------ */
static oracle_solve_info *g_infos = NULL;
static int g_ninfo = 0, g_capinfo = 0;

static void info_reset(void) { g_ninfo = 0; }
static void info_push(const oracle_solve_info *s)
{
    if (g_ninfo == g_capinfo) {
        g_capinfo = g_capinfo ? 2 * g_capinfo : 64;
        g_infos = (oracle_solve_info *)realloc(g_infos, sizeof(*g_infos) * (size_t)g_capinfo);
    }
    g_infos[g_ninfo++] = *s;
}
int oracle_solve_count(void) { return g_ninfo; }
int oracle_solve_get(int k, oracle_solve_info *out)
{
    if (k < 0 || k >= g_ninfo) return -1;
    *out = g_infos[k];
    return 0;
}
int oracle_q_is_double(void) { return (int)(sizeof(qval) == sizeof(double)); }
void oracle_srand(unsigned seed) { srand(seed); }

/* ------------------------------------------------------------------ */
/* kernel functions                                                    */
/* ------------------------------------------------------------------ */

/* reference svm.cpp:30-40 */
static double orc_powi(double base, int times)
{
    double tmp = base, ret = 1.0;
    for (int t = times; t > 0; t /= 2) {
        if (t % 2 == 1) ret *= tmp;
        tmp = tmp * tmp;
    }
    return ret;
}

/* sparse merge dot product, reference svm.cpp:305-325 */
static double orc_dot(const struct svm_node *px, const struct svm_node *py)
{
    double sum = 0;
    while (px->index != -1 && py->index != -1) {
        if (px->index == py->index) {
            sum += px->value * py->value;
            ++px;
            ++py;
        } else if (px->index > py->index) {
            ++py;
        } else {
            ++px;
        }
    }
    return sum;
}

/* prediction-time kernel, reference svm.cpp:327-384 (RBF walks the sparse
 * difference instead of using precomputed squared norms) */
double oracle_k_function(const struct svm_node *x, const struct svm_node *y, const struct svm_parameter *param)
{
    switch (param->kernel_type) {
    case LINEAR:
        return orc_dot(x, y);
    case POLY:
        return orc_powi(param->gamma * orc_dot(x, y) + param->coef0, param->degree);
    case RBF: {
        double sum = 0;
        while (x->index != -1 && y->index != -1) {
            if (x->index == y->index) {
                double d = x->value - y->value;
                sum += d * d;
                ++x;
                ++y;
            } else if (x->index > y->index) {
                sum += y->value * y->value;
                ++y;
            } else {
                sum += x->value * x->value;
                ++x;
            }
        }
        while (x->index != -1) { sum += x->value * x->value; ++x; }
        while (y->index != -1) { sum += y->value * y->value; ++y; }
        return exp(-param->gamma * sum);
    }
    case SIGMOID:
        return tanh(param->gamma * orc_dot(x, y) + param->coef0);
    case PRECOMPUTED:
        return x[(int)(y->value)].value;
    default:
        return 0;
    }
}

/* training-time kernel K(i,j) on original row ids, reference svm.cpp:235-254
 * (RBF uses x_square, computed as dot(x_i,x_i), svm.cpp:282-296). */
typedef struct {
    int l;
    const struct svm_node *const *x;
    double *x_square;
    int kernel_type, degree;
    double gamma, coef0;
} orc_kernel;

static double kernel_eval(const orc_kernel *k, int i, int j)
{
    switch (k->kernel_type) {
    case LINEAR:
        return orc_dot(k->x[i], k->x[j]);
    case POLY:
        return orc_powi(k->gamma * orc_dot(k->x[i], k->x[j]) + k->coef0, k->degree);
    case RBF:
        return exp(-k->gamma * (k->x_square[i] + k->x_square[j] - 2 * orc_dot(k->x[i], k->x[j])));
    case SIGMOID:
        return tanh(k->gamma * orc_dot(k->x[i], k->x[j]) + k->coef0);
    case PRECOMPUTED:
        return k->x[i][(int)(k->x[j][0].value)].value;
    default:
        return 0;
    }
}

/* ------------------------------------------------------------------ */
/* SVC Q matrix (reference SVC_Q, svm.cpp:1313-1365)                   */
/* Q_ij = y_i y_j K(i,j) stored as qval; QD_i = K(i,i) kept in double.  */
/* ------------------------------------------------------------------ */
typedef struct {
    orc_kernel k;
    const signed char *y_orig;  /* labels by original id */
    /* row cache keyed by original id, full rows in original column order */
    qval **row;
    int *lru_prev, *lru_next;   /* doubly linked list over ids with rows; head = l */
    long budget_rows, used_rows;
    qval *gather[2];
    int gather_next;
} orc_qmatrix;

static void qm_unlink(orc_qmatrix *q, int id)
{
    q->lru_next[q->lru_prev[id]] = q->lru_next[id];
    q->lru_prev[q->lru_next[id]] = q->lru_prev[id];
}
static void qm_push_back(orc_qmatrix *q, int id)
{
    int head = q->k.l;
    q->lru_prev[id] = q->lru_prev[head];
    q->lru_next[id] = head;
    q->lru_next[q->lru_prev[head]] = id;
    q->lru_prev[head] = id;
}

static const qval *qm_full_row(orc_qmatrix *q, int id)
{
    int l = q->k.l;
    if (q->row[id]) {
        qm_unlink(q, id);
        qm_push_back(q, id);
        return q->row[id];
    }
    while (q->used_rows >= q->budget_rows) {
        int old = q->lru_next[l];
        qm_unlink(q, old);
        free(q->row[old]);
        q->row[old] = NULL;
        q->used_rows--;
    }
    qval *r = (qval *)malloc(sizeof(qval) * (size_t)l);
    signed char yi = q->y_orig[id];
    for (int j = 0; j < l; j++)
        r[j] = (qval)(yi * q->y_orig[j] * kernel_eval(&q->k, id, j));   /* svm.cpp:1337 */
    q->row[id] = r;
    q->used_rows++;
    qm_push_back(q, id);
    return r;
}

static void qm_init(orc_qmatrix *q, const struct svm_problem *prob, const struct svm_parameter *param,
                    const signed char *y)
{
    int l = prob->l;
    q->k.l = l;
    q->k.x = (const struct svm_node *const *)prob->x;
    q->k.kernel_type = param->kernel_type;
    q->k.degree = param->degree;
    q->k.gamma = param->gamma;
    q->k.coef0 = param->coef0;
    q->k.x_square = NULL;
    if (param->kernel_type == RBF) {
        q->k.x_square = (double *)malloc(sizeof(double) * (size_t)l);
        for (int i = 0; i < l; i++) q->k.x_square[i] = orc_dot(prob->x[i], prob->x[i]);
    }
    q->y_orig = y;
    q->row = (qval **)calloc((size_t)l, sizeof(qval *));
    q->lru_prev = (int *)malloc(sizeof(int) * (size_t)(l + 1));
    q->lru_next = (int *)malloc(sizeof(int) * (size_t)(l + 1));
    q->lru_prev[l] = q->lru_next[l] = l;
    long bytes = (long)(param->cache_size * (1 << 20));
    long rows = bytes / (long)(sizeof(qval) * (size_t)l);
    if (rows < 2) rows = 2;     /* the reference keeps at least two columns, svm.cpp:102 */
    q->budget_rows = rows;
    q->used_rows = 0;
    q->gather[0] = (qval *)malloc(sizeof(qval) * (size_t)l);
    q->gather[1] = (qval *)malloc(sizeof(qval) * (size_t)l);
    q->gather_next = 0;
}

static void qm_free(orc_qmatrix *q)
{
    for (int i = 0; i < q->k.l; i++) free(q->row[i]);
    free(q->row);
    free(q->lru_prev);
    free(q->lru_next);
    free(q->k.x_square);
    free(q->gather[0]);
    free(q->gather[1]);
}

/* ------------------------------------------------------------------ */
/* SMO solver (reference Solver, svm.cpp:404-1049, and Solver_NU,       */
/* svm.cpp:1056-1308).  State is position-indexed and permuted by        */
/* swap_index exactly like the reference; active_set[pos] = original id. */
/* ------------------------------------------------------------------ */
typedef struct {
    int nu;                     /* 0: Solver, 1: Solver_NU */
    int l, active_size;
    signed char *y;
    double *G, *G_bar, *alpha, *p, *QD;
    char *status;
    int *active_set;
    double Cp, Cn, eps;
    int unshrink;
    orc_qmatrix *Q;
    double r;                   /* Solver_NU si->r */
} orc_solver;

/* get_Q(pos, len): Q row of the variable at position `pos`, in position order */
static const qval *s_get_Q(orc_solver *s, int pos, int len)
{
    orc_qmatrix *q = s->Q;
    const qval *full = qm_full_row(q, s->active_set[pos]);
    qval *out = q->gather[q->gather_next];
    q->gather_next ^= 1;
    for (int j = 0; j < len; j++) out[j] = full[s->active_set[j]];
    return out;
}

static double s_get_C(const orc_solver *s, int i) { return (s->y[i] > 0) ? s->Cp : s->Cn; }   /* svm.cpp:437-440 */

static void s_update_status(orc_solver *s, int i)   /* svm.cpp:441-449 */
{
    if (s->alpha[i] >= s_get_C(s, i)) s->status[i] = ST_UPPER;
    else if (s->alpha[i] <= 0) s->status[i] = ST_LOWER;
    else s->status[i] = ST_FREE;
}
#define IS_UP(s, i) ((s)->status[i] == ST_UPPER)
#define IS_LO(s, i) ((s)->status[i] == ST_LOWER)
#define IS_FREE(s, i) ((s)->status[i] == ST_FREE)

#define SWAPT(T, a, b) do { T t_ = (a); (a) = (b); (b) = t_; } while (0)
static void s_swap_index(orc_solver *s, int i, int j)   /* svm.cpp:461-471 */
{
    SWAPT(signed char, s->y[i], s->y[j]);
    SWAPT(double, s->G[i], s->G[j]);
    SWAPT(char, s->status[i], s->status[j]);
    SWAPT(double, s->alpha[i], s->alpha[j]);
    SWAPT(double, s->p[i], s->p[j]);
    SWAPT(int, s->active_set[i], s->active_set[j]);
    SWAPT(double, s->G_bar[i], s->G_bar[j]);
    SWAPT(double, s->QD[i], s->QD[j]);
}

static void s_reconstruct_gradient(orc_solver *s)  /* svm.cpp:473-513 */
{
    int l = s->l, as = s->active_size;
    if (as == l) return;
    int nr_free = 0;
    for (int j = as; j < l; j++) s->G[j] = s->G_bar[j] + s->p[j];
    for (int j = 0; j < as; j++)
        if (IS_FREE(s, j)) nr_free++;
    /* The reference picks one of two loop orders (svm.cpp:492); both add
     * alpha_f * Q[f][e] to G[e] over free f in position order, and Q is
     * symmetric bit for bit, so one order gives identical results. */
    for (int i = 0; i < as; i++)
        if (IS_FREE(s, i)) {
            const qval *Q_i = s_get_Q(s, i, l);
            double alpha_i = s->alpha[i];
            for (int j = as; j < l; j++) s->G[j] += alpha_i * Q_i[j];
        }
}

/* reference Solver::select_working_set, svm.cpp:833-930 */
static int s_select_c(orc_solver *s, int *out_i, int *out_j)
{
    double Gmax = -ORC_INF, Gmax2 = -ORC_INF;
    int Gmax_idx = -1, Gmin_idx = -1;
    double obj_diff_min = ORC_INF;
    int as = s->active_size;
    for (int t = 0; t < as; t++) {
        if (s->y[t] == +1) {
            if (!IS_UP(s, t) && -s->G[t] >= Gmax) { Gmax = -s->G[t]; Gmax_idx = t; }
        } else {
            if (!IS_LO(s, t) && s->G[t] >= Gmax) { Gmax = s->G[t]; Gmax_idx = t; }
        }
    }
    int i = Gmax_idx;
    const qval *Q_i = NULL;
    if (i != -1) Q_i = s_get_Q(s, i, as);
    for (int j = 0; j < as; j++) {
        if (s->y[j] == +1) {
            if (!IS_LO(s, j)) {
                double grad_diff = Gmax + s->G[j];
                if (s->G[j] >= Gmax2) Gmax2 = s->G[j];
                if (grad_diff > 0) {
                    double obj_diff;
                    double quad_coef = s->QD[i] + s->QD[j] - 2.0 * s->y[i] * Q_i[j];
                    if (quad_coef > 0) obj_diff = -(grad_diff * grad_diff) / quad_coef;
                    else obj_diff = -(grad_diff * grad_diff) / ORC_TAU;
                    if (obj_diff <= obj_diff_min) { Gmin_idx = j; obj_diff_min = obj_diff; }
                }
            }
        } else {
            if (!IS_UP(s, j)) {
                double grad_diff = Gmax - s->G[j];
                if (-s->G[j] >= Gmax2) Gmax2 = -s->G[j];
                if (grad_diff > 0) {
                    double obj_diff;
                    double quad_coef = s->QD[i] + s->QD[j] + 2.0 * s->y[i] * Q_i[j];
                    if (quad_coef > 0) obj_diff = -(grad_diff * grad_diff) / quad_coef;
                    else obj_diff = -(grad_diff * grad_diff) / ORC_TAU;
                    if (obj_diff <= obj_diff_min) { Gmin_idx = j; obj_diff_min = obj_diff; }
                }
            }
        }
    }
    if (Gmax + Gmax2 < s->eps) return 1;
    *out_i = Gmax_idx;
    *out_j = Gmin_idx;
    return 0;
}

/* reference Solver_NU::select_working_set, svm.cpp:1076-1186 */
static int s_select_nu(orc_solver *s, int *out_i, int *out_j)
{
    double Gmaxp = -ORC_INF, Gmaxp2 = -ORC_INF, Gmaxn = -ORC_INF, Gmaxn2 = -ORC_INF;
    int Gmaxp_idx = -1, Gmaxn_idx = -1, Gmin_idx = -1;
    double obj_diff_min = ORC_INF;
    int as = s->active_size;
    for (int t = 0; t < as; t++) {
        if (s->y[t] == +1) {
            if (!IS_UP(s, t) && -s->G[t] >= Gmaxp) { Gmaxp = -s->G[t]; Gmaxp_idx = t; }
        } else {
            if (!IS_LO(s, t) && s->G[t] >= Gmaxn) { Gmaxn = s->G[t]; Gmaxn_idx = t; }
        }
    }
    int ip = Gmaxp_idx, in = Gmaxn_idx;
    const qval *Q_ip = NULL, *Q_in = NULL;
    if (ip != -1) Q_ip = s_get_Q(s, ip, as);
    if (in != -1) Q_in = s_get_Q(s, in, as);
    for (int j = 0; j < as; j++) {
        if (s->y[j] == +1) {
            if (!IS_LO(s, j)) {
                double grad_diff = Gmaxp + s->G[j];
                if (s->G[j] >= Gmaxp2) Gmaxp2 = s->G[j];
                if (grad_diff > 0) {
                    double obj_diff;
                    double quad_coef = s->QD[ip] + s->QD[j] - 2 * Q_ip[j];
                    if (quad_coef > 0) obj_diff = -(grad_diff * grad_diff) / quad_coef;
                    else obj_diff = -(grad_diff * grad_diff) / ORC_TAU;
                    if (obj_diff <= obj_diff_min) { Gmin_idx = j; obj_diff_min = obj_diff; }
                }
            }
        } else {
            if (!IS_UP(s, j)) {
                double grad_diff = Gmaxn - s->G[j];
                if (-s->G[j] >= Gmaxn2) Gmaxn2 = -s->G[j];
                if (grad_diff > 0) {
                    double obj_diff;
                    double quad_coef = s->QD[in] + s->QD[j] - 2 * Q_in[j];
                    if (quad_coef > 0) obj_diff = -(grad_diff * grad_diff) / quad_coef;
                    else obj_diff = -(grad_diff * grad_diff) / ORC_TAU;
                    if (obj_diff <= obj_diff_min) { Gmin_idx = j; obj_diff_min = obj_diff; }
                }
            }
        }
    }
    double m1 = Gmaxp + Gmaxp2, m2 = Gmaxn + Gmaxn2;
    if ((m1 > m2 ? m1 : m2) < s->eps) return 1;
    if (s->y[Gmin_idx] == +1) *out_i = Gmaxp_idx;
    else *out_i = Gmaxn_idx;
    *out_j = Gmin_idx;
    return 0;
}

/* reference Solver::be_shrunk / do_shrinking, svm.cpp:932-1011 */
static int s_be_shrunk_c(const orc_solver *s, int i, double Gmax1, double Gmax2)
{
    if (IS_UP(s, i)) {
        if (s->y[i] == +1) return -s->G[i] > Gmax1;
        return -s->G[i] > Gmax2;
    } else if (IS_LO(s, i)) {
        if (s->y[i] == +1) return s->G[i] > Gmax2;
        return s->G[i] > Gmax1;
    }
    return 0;
}

/* reference Solver_NU::be_shrunk, svm.cpp:1188-1206 */
static int s_be_shrunk_nu(const orc_solver *s, int i, double g1, double g2, double g3, double g4)
{
    if (IS_UP(s, i)) {
        if (s->y[i] == +1) return -s->G[i] > g1;
        return -s->G[i] > g4;
    } else if (IS_LO(s, i)) {
        if (s->y[i] == +1) return s->G[i] > g2;
        return s->G[i] > g3;
    }
    return 0;
}

static void s_do_shrinking(orc_solver *s)
{
    int i;
    if (!s->nu) {
        double Gmax1 = -ORC_INF, Gmax2 = -ORC_INF;
        for (i = 0; i < s->active_size; i++) {
            if (s->y[i] == +1) {
                if (!IS_UP(s, i) && -s->G[i] >= Gmax1) Gmax1 = -s->G[i];
                if (!IS_LO(s, i) && s->G[i] >= Gmax2) Gmax2 = s->G[i];
            } else {
                if (!IS_UP(s, i) && -s->G[i] >= Gmax2) Gmax2 = -s->G[i];
                if (!IS_LO(s, i) && s->G[i] >= Gmax1) Gmax1 = s->G[i];
            }
        }
        if (s->unshrink == 0 && Gmax1 + Gmax2 <= s->eps * 10) {
            s->unshrink = 1;
            s_reconstruct_gradient(s);
            s->active_size = s->l;
        }
        for (i = 0; i < s->active_size; i++)
            if (s_be_shrunk_c(s, i, Gmax1, Gmax2)) {
                s->active_size--;
                while (s->active_size > i) {
                    if (!s_be_shrunk_c(s, s->active_size, Gmax1, Gmax2)) {
                        s_swap_index(s, i, s->active_size);
                        break;
                    }
                    s->active_size--;
                }
            }
    } else {
        /* reference Solver_NU::do_shrinking, svm.cpp:1208-1258 */
        double g1 = -ORC_INF, g2 = -ORC_INF, g3 = -ORC_INF, g4 = -ORC_INF;
        for (i = 0; i < s->active_size; i++) {
            if (!IS_UP(s, i)) {
                if (s->y[i] == +1) { if (-s->G[i] > g1) g1 = -s->G[i]; }
                else if (-s->G[i] > g4) g4 = -s->G[i];
            }
            if (!IS_LO(s, i)) {
                if (s->y[i] == +1) { if (s->G[i] > g2) g2 = s->G[i]; }
                else if (s->G[i] > g3) g3 = s->G[i];
            }
        }
        double a = g1 + g2, b = g3 + g4;
        if (s->unshrink == 0 && (a > b ? a : b) <= s->eps * 10) {
            s->unshrink = 1;
            s_reconstruct_gradient(s);
            s->active_size = s->l;
        }
        for (i = 0; i < s->active_size; i++)
            if (s_be_shrunk_nu(s, i, g1, g2, g3, g4)) {
                s->active_size--;
                while (s->active_size > i) {
                    if (!s_be_shrunk_nu(s, s->active_size, g1, g2, g3, g4)) {
                        s_swap_index(s, i, s->active_size);
                        break;
                    }
                    s->active_size--;
                }
            }
    }
}

/* reference Solver::calculate_rho, svm.cpp:1013-1049 */
static double s_rho_c(const orc_solver *s)
{
    int nr_free = 0;
    double ub = ORC_INF, lb = -ORC_INF, sum_free = 0;
    for (int i = 0; i < s->active_size; i++) {
        double yG = s->y[i] * s->G[i];
        if (IS_UP(s, i)) {
            if (s->y[i] == -1) ub = (ub < yG) ? ub : yG;
            else lb = (lb > yG) ? lb : yG;
        } else if (IS_LO(s, i)) {
            if (s->y[i] == +1) ub = (ub < yG) ? ub : yG;
            else lb = (lb > yG) ? lb : yG;
        } else {
            ++nr_free;
            sum_free += yG;
        }
    }
    if (nr_free > 0) return sum_free / nr_free;
    return (ub + lb) / 2;
}

/* reference Solver_NU::calculate_rho, svm.cpp:1260-1308 */
static double s_rho_nu(orc_solver *s)
{
    int nr_free1 = 0, nr_free2 = 0;
    double ub1 = ORC_INF, ub2 = ORC_INF, lb1 = -ORC_INF, lb2 = -ORC_INF;
    double sum_free1 = 0, sum_free2 = 0;
    for (int i = 0; i < s->active_size; i++) {
        if (s->y[i] == +1) {
            if (IS_UP(s, i)) lb1 = (lb1 > s->G[i]) ? lb1 : s->G[i];
            else if (IS_LO(s, i)) ub1 = (ub1 < s->G[i]) ? ub1 : s->G[i];
            else { ++nr_free1; sum_free1 += s->G[i]; }
        } else {
            if (IS_UP(s, i)) lb2 = (lb2 > s->G[i]) ? lb2 : s->G[i];
            else if (IS_LO(s, i)) ub2 = (ub2 < s->G[i]) ? ub2 : s->G[i];
            else { ++nr_free2; sum_free2 += s->G[i]; }
        }
    }
    double r1 = nr_free1 > 0 ? sum_free1 / nr_free1 : (ub1 + lb1) / 2;
    double r2 = nr_free2 > 0 ? sum_free2 / nr_free2 : (ub2 + lb2) / 2;
    s->r = (r1 + r2) / 2;
    return (r1 - r2) / 2;
}

/* reference Solver::Solve, svm.cpp:515-830 (CPU branch). Returns #iter. */
static long long s_solve(orc_solver *s, const double *p_, const signed char *y_, double *alpha_,
                         double *rho_out, double *obj_out, int shrinking)
{
    int l = s->l;
    s->p = (double *)malloc(sizeof(double) * (size_t)l);
    s->y = (signed char *)malloc((size_t)l);
    s->alpha = (double *)malloc(sizeof(double) * (size_t)l);
    memcpy(s->p, p_, sizeof(double) * (size_t)l);
    memcpy(s->y, y_, (size_t)l);
    memcpy(s->alpha, alpha_, sizeof(double) * (size_t)l);
    s->unshrink = 0;
    s->status = (char *)malloc((size_t)l);
    for (int i = 0; i < l; i++) s_update_status(s, i);
    s->active_set = (int *)malloc(sizeof(int) * (size_t)l);
    for (int i = 0; i < l; i++) s->active_set[i] = i;
    s->active_size = l;
    /* QD (svm.cpp:1321-1327): K(i,i) in double, permuted with the rest */
    s->QD = (double *)malloc(sizeof(double) * (size_t)l);
    for (int i = 0; i < l; i++) s->QD[i] = kernel_eval(&s->Q->k, i, i);

    s->G = (double *)malloc(sizeof(double) * (size_t)l);
    s->G_bar = (double *)malloc(sizeof(double) * (size_t)l);
    for (int i = 0; i < l; i++) { s->G[i] = s->p[i]; s->G_bar[i] = 0; }
    for (int i = 0; i < l; i++)     /* svm.cpp:559-570 */
        if (!IS_LO(s, i)) {
            const qval *Q_i = s_get_Q(s, i, l);
            double alpha_i = s->alpha[i];
            for (int j = 0; j < l; j++) s->G[j] += alpha_i * Q_i[j];
            if (IS_UP(s, i))
                for (int j = 0; j < l; j++) s->G_bar[j] += s_get_C(s, i) * Q_i[j];
        }

    long long iter = 0;
    long long max_iter = (l > INT_MAX / 100) ? INT_MAX : 100LL * l;
    if (max_iter < 10000000) max_iter = 10000000;       /* svm.cpp:577 */
    int counter = (l < 1000 ? l : 1000) + 1;

    while (iter < max_iter) {
        if (--counter == 0) {
            counter = l < 1000 ? l : 1000;
            if (shrinking) s_do_shrinking(s);
        }
        int i = -1, j = -1;
        int opt = s->nu ? s_select_nu(s, &i, &j) : s_select_c(s, &i, &j);
        if (opt != 0) {
            s_reconstruct_gradient(s);
            s->active_size = l;
            opt = s->nu ? s_select_nu(s, &i, &j) : s_select_c(s, &i, &j);
            if (opt != 0) break;
            counter = 1;
        }
        ++iter;

        /* two-variable analytic step, svm.cpp:627-721 */
        const qval *Q_i = s_get_Q(s, i, s->active_size);
        const qval *Q_j = s_get_Q(s, j, s->active_size);
        double C_i = s_get_C(s, i), C_j = s_get_C(s, j);
        double old_alpha_i = s->alpha[i], old_alpha_j = s->alpha[j];
        double *alpha = s->alpha;
        if (s->y[i] != s->y[j]) {
            double quad_coef = s->QD[i] + s->QD[j] + 2 * Q_i[j];
            if (quad_coef <= 0) quad_coef = ORC_TAU;
            double delta = (-s->G[i] - s->G[j]) / quad_coef;
            double diff = alpha[i] - alpha[j];
            alpha[i] += delta;
            alpha[j] += delta;
            if (diff > 0) {
                if (alpha[j] < 0) { alpha[j] = 0; alpha[i] = diff; }
            } else {
                if (alpha[i] < 0) { alpha[i] = 0; alpha[j] = -diff; }
            }
            if (diff > C_i - C_j) {
                if (alpha[i] > C_i) { alpha[i] = C_i; alpha[j] = C_i - diff; }
            } else {
                if (alpha[j] > C_j) { alpha[j] = C_j; alpha[i] = C_j + diff; }
            }
        } else {
            double quad_coef = s->QD[i] + s->QD[j] - 2 * Q_i[j];
            if (quad_coef <= 0) quad_coef = ORC_TAU;
            double delta = (s->G[i] - s->G[j]) / quad_coef;
            double sum = alpha[i] + alpha[j];
            alpha[i] -= delta;
            alpha[j] += delta;
            if (sum > C_i) {
                if (alpha[i] > C_i) { alpha[i] = C_i; alpha[j] = sum - C_i; }
            } else {
                if (alpha[j] < 0) { alpha[j] = 0; alpha[i] = sum; }
            }
            if (sum > C_j) {
                if (alpha[j] > C_j) { alpha[j] = C_j; alpha[i] = sum - C_j; }
            } else {
                if (alpha[i] < 0) { alpha[i] = 0; alpha[j] = sum; }
            }
        }

        /* G update over the active set, svm.cpp:729-735 */
        double dai = alpha[i] - old_alpha_i;
        double daj = alpha[j] - old_alpha_j;
        for (int k = 0; k < s->active_size; k++) s->G[k] += Q_i[k] * dai + Q_j[k] * daj;

        /* status + G_bar, svm.cpp:744-769 */
        int ui = IS_UP(s, i), uj = IS_UP(s, j);
        s_update_status(s, i);
        s_update_status(s, j);
        if (ui != IS_UP(s, i)) {
            Q_i = s_get_Q(s, i, l);
            if (ui) for (int k = 0; k < l; k++) s->G_bar[k] -= C_i * Q_i[k];
            else for (int k = 0; k < l; k++) s->G_bar[k] += C_i * Q_i[k];
        }
        if (uj != IS_UP(s, j)) {
            Q_j = s_get_Q(s, j, l);
            if (uj) for (int k = 0; k < l; k++) s->G_bar[k] -= C_j * Q_j[k];
            else for (int k = 0; k < l; k++) s->G_bar[k] += C_j * Q_j[k];
        }
    }

    if (iter >= max_iter) {
        if (s->active_size < l) {
            s_reconstruct_gradient(s);
            s->active_size = l;
        }
        fprintf(stderr, "\nWARNING: reaching max number of iterations\n");
    }
    *rho_out = s->nu ? s_rho_nu(s) : s_rho_c(s);
    double v = 0;
    for (int i = 0; i < l; i++) v += s->alpha[i] * (s->G[i] + s->p[i]);   /* svm.cpp:795-802 */
    *obj_out = v / 2;
    for (int i = 0; i < l; i++) alpha_[s->active_set[i]] = s->alpha[i];

    free(s->p); free(s->y); free(s->alpha); free(s->status); free(s->active_set);
    free(s->QD); free(s->G); free(s->G_bar);
    return iter;
}

/* ------------------------------------------------------------------ */
/* formulations (reference svm.cpp:1500-1588) and svm_train_one         */
/* (svm.cpp:1707-1769)                                                  */
/* ------------------------------------------------------------------ */
static double *train_one(const struct svm_problem *prob, const struct svm_parameter *param,
                         double Cp, double Cn, double *rho_out)
{
    int l = prob->l;
    double *alpha = (double *)malloc(sizeof(double) * (size_t)(l > 0 ? l : 1));
    signed char *y = (signed char *)malloc((size_t)(l > 0 ? l : 1));
    for (int i = 0; i < l; i++) y[i] = (prob->y[i] > 0) ? +1 : -1;
    orc_qmatrix Q;
    qm_init(&Q, prob, param, y);
    orc_solver s;
    memset(&s, 0, sizeof(s));
    s.l = l;
    s.Q = &Q;
    s.eps = param->eps;
    oracle_solve_info rec;
    memset(&rec, 0, sizeof(rec));
    double rho = 0, obj = 0;
    double *p = (double *)malloc(sizeof(double) * (size_t)(l > 0 ? l : 1));
    double upper_p, upper_n;
    if (param->svm_type == NU_SVC) {
        /* solve_nu_svc, svm.cpp:1535-1588 */
        double nu = param->nu;
        double sum_pos = nu * l / 2, sum_neg = nu * l / 2;
        for (int i = 0; i < l; i++) {
            if (y[i] == +1) { alpha[i] = (1.0 < sum_pos) ? 1.0 : sum_pos; sum_pos -= alpha[i]; }
            else { alpha[i] = (1.0 < sum_neg) ? 1.0 : sum_neg; sum_neg -= alpha[i]; }
        }
        for (int i = 0; i < l; i++) p[i] = 0;
        s.nu = 1;
        s.Cp = 1.0;
        s.Cn = 1.0;
        rec.iters = s_solve(&s, p, y, alpha, &rho, &obj, param->shrinking);
        double r = s.r;
        for (int i = 0; i < l; i++) alpha[i] *= y[i] / r;
        rho /= r;
        obj /= (r * r);
        upper_p = 1 / r;
        upper_n = 1 / r;
        rec.r = r;
    } else {
        /* solve_c_svc, svm.cpp:1500-1533 */
        for (int i = 0; i < l; i++) { alpha[i] = 0; p[i] = -1; }
        s.nu = 0;
        s.Cp = Cp;
        s.Cn = Cn;
        rec.iters = s_solve(&s, p, y, alpha, &rho, &obj, param->shrinking);
        for (int i = 0; i < l; i++) alpha[i] *= y[i];
        upper_p = Cp;
        upper_n = Cn;
    }
    rec.obj = obj;
    rec.rho = rho;
    rec.l = l;
    for (int i = 0; i < l; i++) {
        if (fabs(alpha[i]) > 0) {
            rec.nr_sv++;
            double ub = prob->y[i] > 0 ? upper_p : upper_n;
            if (fabs(alpha[i]) < ub) rec.nr_free++;
        }
    }
    info_push(&rec);
    qm_free(&Q);
    free(p);
    free(y);
    *rho_out = rho;
    return alpha;
}

int oracle_solve_binary(const struct svm_problem *prob, const struct svm_parameter *param,
                        double Cp, double Cn, double *alpha_out, oracle_solve_info *out)
{
    info_reset();
    double rho;
    double *a = train_one(prob, param, Cp, Cn, &rho);
    memcpy(alpha_out, a, sizeof(double) * (size_t)prob->l);
    free(a);
    if (out) *out = g_infos[0];
    return 0;
}

/* ------------------------------------------------------------------ */
/* class grouping and one-vs-one training (reference svm.cpp:2081-2404) */
/* ------------------------------------------------------------------ */
static void group_classes(const struct svm_problem *prob, int *nr_class_ret, int **label_ret,
                          int **start_ret, int **count_ret, int *perm)
{
    int l = prob->l, cap = 16, nr_class = 0;
    int *label = (int *)malloc(sizeof(int) * (size_t)cap);
    int *count = (int *)malloc(sizeof(int) * (size_t)cap);
    int *data_label = (int *)malloc(sizeof(int) * (size_t)(l > 0 ? l : 1));
    for (int i = 0; i < l; i++) {
        int this_label = (int)prob->y[i];
        int j;
        for (j = 0; j < nr_class; j++)
            if (this_label == label[j]) { ++count[j]; break; }
        data_label[i] = j;
        if (j == nr_class) {
            if (nr_class == cap) {
                cap *= 2;
                label = (int *)realloc(label, sizeof(int) * (size_t)cap);
                count = (int *)realloc(count, sizeof(int) * (size_t)cap);
            }
            label[nr_class] = this_label;
            count[nr_class] = 1;
            ++nr_class;
        }
    }
    /* -1/+1 with -1 first: swap so that +1 is class 0, svm.cpp:2123-2134 */
    if (nr_class == 2 && label[0] == -1 && label[1] == 1) {
        SWAPT(int, label[0], label[1]);
        SWAPT(int, count[0], count[1]);
        for (int i = 0; i < l; i++) data_label[i] = data_label[i] == 0 ? 1 : 0;
    }
    int *start = (int *)malloc(sizeof(int) * (size_t)(nr_class > 0 ? nr_class : 1));
    start[0] = 0;
    for (int i = 1; i < nr_class; i++) start[i] = start[i - 1] + count[i - 1];
    for (int i = 0; i < l; i++) { perm[start[data_label[i]]] = i; ++start[data_label[i]]; }
    start[0] = 0;
    for (int i = 1; i < nr_class; i++) start[i] = start[i - 1] + count[i - 1];
    *nr_class_ret = nr_class;
    *label_ret = label;
    *start_ret = start;
    *count_ret = count;
    free(data_label);
}

struct svm_model *oracle_svm_train(const struct svm_problem *prob, const struct svm_parameter *param)
{
    info_reset();
    struct svm_model *model = (struct svm_model *)calloc(1, sizeof(struct svm_model));
    model->param = *param;
    model->free_sv = 0;
    int l = prob->l, nr_class;
    int *label = NULL, *start = NULL, *count = NULL;
    int *perm = (int *)malloc(sizeof(int) * (size_t)(l > 0 ? l : 1));
    group_classes(prob, &nr_class, &label, &start, &count, perm);
    struct svm_node **x = (struct svm_node **)malloc(sizeof(*x) * (size_t)(l > 0 ? l : 1));
    for (int i = 0; i < l; i++) x[i] = prob->x[perm[i]];
    double *weighted_C = (double *)malloc(sizeof(double) * (size_t)nr_class);
    for (int i = 0; i < nr_class; i++) weighted_C[i] = param->C;
    for (int i = 0; i < param->nr_weight; i++) {
        int j;
        for (j = 0; j < nr_class; j++)
            if (param->weight_label[i] == label[j]) break;
        if (j < nr_class) weighted_C[j] *= param->weight[i];
    }
    int npair = nr_class * (nr_class - 1) / 2;
    char *nonzero = (char *)calloc((size_t)(l > 0 ? l : 1), 1);
    double **f_alpha = (double **)malloc(sizeof(double *) * (size_t)(npair > 0 ? npair : 1));
    double *f_rho = (double *)malloc(sizeof(double) * (size_t)(npair > 0 ? npair : 1));
    int p = 0;
    for (int i = 0; i < nr_class; i++)
        for (int j = i + 1; j < nr_class; j++) {
            int si = start[i], sj = start[j], ci = count[i], cj = count[j];
            struct svm_problem sub;
            sub.l = ci + cj;
            sub.x = (struct svm_node **)malloc(sizeof(struct svm_node *) * (size_t)sub.l);
            sub.y = (double *)malloc(sizeof(double) * (size_t)sub.l);
            for (int k = 0; k < ci; k++) { sub.x[k] = x[si + k]; sub.y[k] = +1; }
            for (int k = 0; k < cj; k++) { sub.x[ci + k] = x[sj + k]; sub.y[ci + k] = -1; }
            f_alpha[p] = train_one(&sub, param, weighted_C[i], weighted_C[j], &f_rho[p]);
            for (int k = 0; k < ci; k++)
                if (fabs(f_alpha[p][k]) > 0) nonzero[si + k] = 1;
            for (int k = 0; k < cj; k++)
                if (fabs(f_alpha[p][ci + k]) > 0) nonzero[sj + k] = 1;
            free(sub.x);
            free(sub.y);
            ++p;
        }
    model->nr_class = nr_class;
    model->label = (int *)malloc(sizeof(int) * (size_t)nr_class);
    memcpy(model->label, label, sizeof(int) * (size_t)nr_class);
    model->rho = (double *)malloc(sizeof(double) * (size_t)(npair > 0 ? npair : 1));
    for (int i = 0; i < npair; i++) model->rho[i] = f_rho[i];
    model->probA = model->probB = NULL;
    int total_sv = 0;
    int *nz_count = (int *)malloc(sizeof(int) * (size_t)nr_class);
    model->nSV = (int *)malloc(sizeof(int) * (size_t)nr_class);
    for (int i = 0; i < nr_class; i++) {
        int n = 0;
        for (int j = 0; j < count[i]; j++)
            if (nonzero[start[i] + j]) { ++n; ++total_sv; }
        model->nSV[i] = n;
        nz_count[i] = n;
    }
    model->l = total_sv;
    model->SV = (struct svm_node **)malloc(sizeof(struct svm_node *) * (size_t)(total_sv > 0 ? total_sv : 1));
    model->sv_indices = (int *)malloc(sizeof(int) * (size_t)(total_sv > 0 ? total_sv : 1));
    p = 0;
    for (int i = 0; i < l; i++)
        if (nonzero[i]) { model->SV[p] = x[i]; model->sv_indices[p++] = perm[i] + 1; }
    int *nz_start = (int *)malloc(sizeof(int) * (size_t)nr_class);
    nz_start[0] = 0;
    for (int i = 1; i < nr_class; i++) nz_start[i] = nz_start[i - 1] + nz_count[i - 1];
    model->sv_coef = (double **)malloc(sizeof(double *) * (size_t)(nr_class > 1 ? nr_class - 1 : 1));
    for (int i = 0; i < nr_class - 1; i++)
        model->sv_coef[i] = (double *)malloc(sizeof(double) * (size_t)(total_sv > 0 ? total_sv : 1));
    p = 0;
    for (int i = 0; i < nr_class; i++)
        for (int j = i + 1; j < nr_class; j++) {
            int si = start[i], sj = start[j], ci = count[i], cj = count[j];
            int q = nz_start[i];
            for (int k = 0; k < ci; k++)
                if (nonzero[si + k]) model->sv_coef[j - 1][q++] = f_alpha[p][k];
            q = nz_start[j];
            for (int k = 0; k < cj; k++)
                if (nonzero[sj + k]) model->sv_coef[i][q++] = f_alpha[p][ci + k];
            ++p;
        }
    for (int i = 0; i < npair; i++) free(f_alpha[i]);
    free(f_alpha); free(f_rho); free(label); free(count); free(perm); free(start); free(x);
    free(weighted_C); free(nonzero); free(nz_count); free(nz_start);
    return model;
}

void oracle_free_model(struct svm_model *m)
{
    if (!m) return;
    if (m->sv_coef)
        for (int i = 0; i < m->nr_class - 1; i++) free(m->sv_coef[i]);
    free(m->sv_coef); free(m->SV); free(m->rho); free(m->label); free(m->probA);
    free(m->probB); free(m->sv_indices); free(m->nSV);
    free(m);
}

/* reference svm_predict_values, svm.cpp:2569-2643 (classification branch) */
double oracle_predict_values(const struct svm_model *model, const struct svm_node *x, double *dec_values)
{
    int nr_class = model->nr_class, l = model->l;
    double *kvalue = (double *)malloc(sizeof(double) * (size_t)(l > 0 ? l : 1));
    for (int i = 0; i < l; i++) kvalue[i] = oracle_k_function(x, model->SV[i], &model->param);
    int *start = (int *)malloc(sizeof(int) * (size_t)nr_class);
    start[0] = 0;
    for (int i = 1; i < nr_class; i++) start[i] = start[i - 1] + model->nSV[i - 1];
    int *vote = (int *)calloc((size_t)nr_class, sizeof(int));
    int p = 0;
    for (int i = 0; i < nr_class; i++)
        for (int j = i + 1; j < nr_class; j++) {
            double sum = 0;
            int si = start[i], sj = start[j], ci = model->nSV[i], cj = model->nSV[j];
            double *coef1 = model->sv_coef[j - 1];
            double *coef2 = model->sv_coef[i];
            for (int k = 0; k < ci; k++) sum += coef1[si + k] * kvalue[si + k];
            for (int k = 0; k < cj; k++) sum += coef2[sj + k] * kvalue[sj + k];
            sum -= model->rho[p];
            dec_values[p] = sum;
            if (dec_values[p] > 0) ++vote[i];
            else ++vote[j];
            p++;
        }
    int best = 0;
    for (int i = 1; i < nr_class; i++)
        if (vote[i] > vote[best]) best = i;
    double lab = model->label[best];
    free(kvalue); free(start); free(vote);
    return lab;
}

double oracle_predict(const struct svm_model *model, const struct svm_node *x)
{
    int k = model->nr_class;
    double *dec = (double *)malloc(sizeof(double) * (size_t)(k * (k - 1) / 2 > 0 ? k * (k - 1) / 2 : 1));
    double r = oracle_predict_values(model, x, dec);
    free(dec);
    return r;
}

/* reference svm_cross_validation, svm.cpp:2407-2525 (classification, no
 * probability).  Uses the C library rand() exactly like the reference. */
void oracle_cross_validation(const struct svm_problem *prob, const struct svm_parameter *param, int nr_fold, double *target)
{
    int l = prob->l;
    int *perm = (int *)malloc(sizeof(int) * (size_t)(l > 0 ? l : 1));
    if (nr_fold > l) nr_fold = l;
    int *fold_start = (int *)malloc(sizeof(int) * (size_t)(nr_fold + 1));
    if (nr_fold < l) {
        int nr_class, *start = NULL, *label = NULL, *count = NULL;
        group_classes(prob, &nr_class, &label, &start, &count, perm);
        int *fold_count = (int *)malloc(sizeof(int) * (size_t)nr_fold);
        int *index = (int *)malloc(sizeof(int) * (size_t)(l > 0 ? l : 1));
        for (int i = 0; i < l; i++) index[i] = perm[i];
        for (int c = 0; c < nr_class; c++)
            for (int i = 0; i < count[c]; i++) {
                int j = i + rand() % (count[c] - i);
                SWAPT(int, index[start[c] + j], index[start[c] + i]);
            }
        for (int i = 0; i < nr_fold; i++) {
            fold_count[i] = 0;
            for (int c = 0; c < nr_class; c++)
                fold_count[i] += (i + 1) * count[c] / nr_fold - i * count[c] / nr_fold;
        }
        fold_start[0] = 0;
        for (int i = 1; i <= nr_fold; i++) fold_start[i] = fold_start[i - 1] + fold_count[i - 1];
        for (int c = 0; c < nr_class; c++)
            for (int i = 0; i < nr_fold; i++) {
                int begin = start[c] + i * count[c] / nr_fold;
                int end = start[c] + (i + 1) * count[c] / nr_fold;
                for (int j = begin; j < end; j++) { perm[fold_start[i]] = index[j]; fold_start[i]++; }
            }
        fold_start[0] = 0;
        for (int i = 1; i <= nr_fold; i++) fold_start[i] = fold_start[i - 1] + fold_count[i - 1];
        free(start); free(label); free(count); free(index); free(fold_count);
    } else {
        for (int i = 0; i < l; i++) perm[i] = i;
        for (int i = 0; i < l; i++) {
            int j = i + rand() % (l - i);
            SWAPT(int, perm[i], perm[j]);
        }
        for (int i = 0; i <= nr_fold; i++) fold_start[i] = i * l / nr_fold;
    }
    int saved = 0;
    oracle_solve_info *acc = NULL;
    for (int i = 0; i < nr_fold; i++) {
        int begin = fold_start[i], end = fold_start[i + 1];
        struct svm_problem sub;
        sub.l = l - (end - begin);
        sub.x = (struct svm_node **)malloc(sizeof(struct svm_node *) * (size_t)(sub.l > 0 ? sub.l : 1));
        sub.y = (double *)malloc(sizeof(double) * (size_t)(sub.l > 0 ? sub.l : 1));
        int k = 0;
        for (int j = 0; j < begin; j++) { sub.x[k] = prob->x[perm[j]]; sub.y[k] = prob->y[perm[j]]; ++k; }
        for (int j = end; j < l; j++) { sub.x[k] = prob->x[perm[j]]; sub.y[k] = prob->y[perm[j]]; ++k; }
        struct svm_model *m = oracle_svm_train(&sub, param);
        size_t need = (size_t)saved + (size_t)g_ninfo + 1u;
        acc = (oracle_solve_info *)realloc(acc, sizeof(*acc) * need);
        memcpy(acc + saved, g_infos, sizeof(*acc) * (size_t)g_ninfo);
        saved += g_ninfo;
        for (int j = begin; j < end; j++) target[perm[j]] = oracle_predict(m, prob->x[perm[j]]);
        oracle_free_model(m);
        free(sub.x);
        free(sub.y);
    }
    info_reset();
    for (int i = 0; i < saved; i++) info_push(&acc[i]);
    free(acc);
    free(fold_start);
    free(perm);
}
