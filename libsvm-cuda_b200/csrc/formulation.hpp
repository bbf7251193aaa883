// formulation.hpp -- the reference's five binary formulations as engine
// subproblems, and the decision function of a solved one (internal).
//
// Every formulation is one SMO problem over "variables" that address rows of
// a device row set by id:
//   C-SVC     (reference svm.cpp:1500-1533)  l variables, alpha = 0, p = -1
//   nu-SVC    (:1535-1588)                   l variables, Solver_NU, alpha from nu
//   one-class (:1590-1620)                   l variables, y = +1, p = 0, alpha from nu
//   eps-SVR   (:1622-1658)                   2l variables over l rows (SVR_Q,
//   nu-SVR    (:1660-1699)                   :1417-1495): variable k and k+l
//                                            both read row k, signs +1 / -1
// The device solver evaluates Q[a][b] = y_a y_b K(row_a, row_b) for every
// formulation, which is exactly SVC_Q, ONE_CLASS_Q and SVR_Q.
#pragma once
#include <string>
#include <vector>

#include "engine.hpp"
#include "svm.h"

namespace svmb {

// Subproblem of formulation `svm_type` over rows[0..l) with targets y[0..l)
// (class labels as +-1 for the classifiers, regression targets for SVR).
// Cp/Cn: C-SVC bounds (weighted C of the positive / negative class); C, nu, p
// as in svm_parameter.  Returns -1 (error set) for an unknown svm_type.
int formulate(int svm_type, const int *rows, const double *y, int l, double Cp, double Cn, double C, double nu,
              double p, SubProblem &sp);

// The decision function of a solved subproblem (svm_train_one, svm.cpp:1707-1769):
// coefficients per training point (signed; SVR: alpha_i - alpha*_i), rho,
// and the solver's messages, one entry per info() call of the reference.
struct Decision {
    std::vector<double> coef;
    double rho = 0, obj = 0, r = 0;
    int nSV = 0, nBSV = 0;
    std::vector<std::string> log;
};
void decide(int svm_type, const SubProblem &sp, const SolveResult &R, const double *y, int l, Decision &f);

}  // namespace svmb
