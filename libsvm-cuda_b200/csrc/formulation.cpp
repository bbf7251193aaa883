// formulation.cpp -- see formulation.hpp.
#include "formulation.hpp"

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>

namespace svmb {

namespace {

void say(std::vector<std::string> &log, const char *fmt, ...)
{
    char buf[256];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    log.emplace_back(buf);
}

}  // namespace

int formulate(int svm_type, const int *rows, const double *y, int l, double Cp, double Cn, double C, double nu,
              double p, SubProblem &sp)
{
    const bool svr = svm_type == EPSILON_SVR || svm_type == NU_SVR;
    const int n = svr ? 2 * l : l;
    sp.rows.resize(n);
    sp.y.resize(n);
    sp.alpha0.assign(n, 0.0);
    sp.p.assign(n, 0.0);
    sp.nu = 0;
    for (int i = 0; i < l; i++) {
        sp.rows[i] = rows[i];
        if (svr) sp.rows[i + l] = rows[i];
    }
    switch (svm_type) {
    case C_SVC:
        for (int i = 0; i < l; i++) {
            sp.y[i] = y[i] > 0 ? +1 : -1;
            sp.p[i] = -1;
        }
        sp.Cp = Cp;
        sp.Cn = Cn;
        break;
    case NU_SVC: {
        // (feasibility, nu*l/2 <= min(#pos, #neg), is svm_check_parameter's
        // to report; like the reference, the solve itself does not refuse)
        for (int i = 0; i < l; i++) sp.y[i] = y[i] > 0 ? +1 : -1;
        // half of nu*l on each side, filled in order up to 1 (svm.cpp:1546-1564)
        double left_pos = nu * l / 2, left_neg = nu * l / 2;
        for (int i = 0; i < l; i++) {
            double &left = sp.y[i] > 0 ? left_pos : left_neg;
            sp.alpha0[i] = std::min(1.0, left);
            left -= sp.alpha0[i];
        }
        sp.nu = 1;
        sp.Cp = sp.Cn = 1.0;
        break;
    }
    case ONE_CLASS: {
        // the first floor(nu*l) points at the bound 1, the next takes the
        // remainder (svm.cpp:1598-1604)
        const int at_bound = (int)(nu * l);
        for (int i = 0; i < l; i++) {
            sp.y[i] = +1;
            sp.alpha0[i] = i < at_bound ? 1.0 : 0.0;
        }
        if (at_bound < l) sp.alpha0[at_bound] = nu * l - at_bound;
        sp.Cp = sp.Cn = 1.0;
        break;
    }
    case EPSILON_SVR:
        // alpha (sign +1) and alpha* (sign -1) of every point, linear terms p -+ y
        for (int i = 0; i < l; i++) {
            sp.y[i] = +1;
            sp.y[i + l] = -1;
            sp.p[i] = p - y[i];
            sp.p[i + l] = p + y[i];
        }
        sp.Cp = sp.Cn = C;
        break;
    case NU_SVR: {
        // C*nu*l/2 spread over the pairs in order, both of a pair equal (svm.cpp:1668-1679)
        double left = C * nu * l / 2;
        for (int i = 0; i < l; i++) {
            const double a = std::min(left, C);
            sp.alpha0[i] = sp.alpha0[i + l] = a;
            left -= a;
            sp.y[i] = +1;
            sp.y[i + l] = -1;
            sp.p[i] = -y[i];
            sp.p[i + l] = y[i];
        }
        sp.nu = 1;
        sp.Cp = sp.Cn = C;
        break;
    }
    default:
        set_error("unknown svm_type");
        return -1;
    }
    return 0;
}

void decide(int svm_type, const SubProblem &sp, const SolveResult &R, const double *y, int l, Decision &f)
{
    f.log.clear();
    f.coef.assign(l, 0.0);
    f.rho = R.out.rho;
    f.obj = R.out.obj;
    f.r = R.out.r;
    double up = sp.Cp, un = sp.Cn;
    say(f.log, "\noptimization finished, #iter = %lld\n", R.out.iters);
    switch (svm_type) {
    case C_SVC: {
        double sum_alpha = 0;
        for (int i = 0; i < l; i++) sum_alpha += R.alpha[i];
        if (sp.Cp == sp.Cn) say(f.log, "nu = %f\n", sum_alpha / (sp.Cp * l));
        for (int i = 0; i < l; i++) f.coef[i] = R.alpha[i] * sp.y[i];
        break;
    }
    case NU_SVC: {
        // scale by 1/r (svm.cpp:1572-1584)
        const double r = R.out.r;
        say(f.log, "C = %f\n", 1 / r);
        for (int i = 0; i < l; i++) f.coef[i] = R.alpha[i] * (sp.y[i] / r);
        f.rho /= r;
        f.obj /= (r * r);
        up = un = 1 / r;
        break;
    }
    case ONE_CLASS:
        for (int i = 0; i < l; i++) f.coef[i] = R.alpha[i];
        break;
    case EPSILON_SVR: {
        double sum_alpha = 0;
        for (int i = 0; i < l; i++) {
            f.coef[i] = R.alpha[i] - R.alpha[i + l];
            sum_alpha += fabs(f.coef[i]);
        }
        say(f.log, "nu = %f\n", sum_alpha / (sp.Cp * l));
        break;
    }
    case NU_SVR:
        say(f.log, "epsilon = %f\n", -R.out.r);
        for (int i = 0; i < l; i++) f.coef[i] = R.alpha[i] - R.alpha[i + l];
        break;
    }
    say(f.log, "obj = %f, rho = %f\n", f.obj, f.rho);
    // bounded SVs are judged by the sign of the point's target (svm.cpp:1744-1760)
    f.nSV = f.nBSV = 0;
    for (int i = 0; i < l; i++)
        if (fabs(f.coef[i]) > 0) {
            ++f.nSV;
            if (fabs(f.coef[i]) >= (y[i] > 0 ? up : un)) ++f.nBSV;
        }
    say(f.log, "nSV = %d, nBSV = %d\n", f.nSV, f.nBSV);
}

}  // namespace svmb
