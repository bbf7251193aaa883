// capi_internal.hpp -- pieces of the svmb_* C-ABI shared by capi.cpp and
// server.cpp (internal to libsvm_b200.so).
#pragma once
#include "engine.hpp"
#include "svm_b200.h"

namespace svmb {
namespace capi {

int check_params(const svmb_params *p);
SolveParams to_solve_params(const svmb_params &p);
// one problem in the formulation of p.svm_type over the rows with ids rows[0..l)
int make_subproblem(const svmb_params &p, int l, const int *rows, const double *y, int nrows, SubProblem &sp);
// coefficients of the l points (y: their targets) and the statistics of one solve
void finish_instance(const svmb_params &p, const SubProblem &sp, const SolveResult &R, const double *y, int l,
                     double *alpha_out, svmb_solve_stats *stats);
int solve_many(const DeviceRows &rows, int ninst, const int *inst_ptr, const int *inst_rows, const double *inst_y,
               const svmb_params *params, double *alpha_out, svmb_solve_stats *stats);

}  // namespace capi
}  // namespace svmb
