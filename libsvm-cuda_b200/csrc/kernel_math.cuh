// kernel_math.cuh -- kernel values from a dot product (reference
// libsvm/svm.cpp:30-40 powi, :235-254 kernel_linear/poly/rbf/sigmoid), in
// float64 with explicit round-to-nearest operations so that no multiply-add
// is contracted.  Shared by the solver and the kernel-block products.
#pragma once
#include "engine.h"

namespace svmb {

__device__ __forceinline__ double powi_d(double base, int times)
{
    double tmp = base, ret = 1.0;
    for (int t = times; t > 0; t /= 2) {
        if (t % 2 == 1) ret = __dmul_rn(ret, tmp);
        tmp = __dmul_rn(tmp, tmp);
    }
    return ret;
}

__device__ __forceinline__ double kernel_from_dot(const KernelParams &kp, double dot, double xsq_a, double xsq_b)
{
    switch (kp.type) {
    case 0: return dot;
    case 1: return powi_d(__dadd_rn(__dmul_rn(kp.gamma, dot), kp.coef0), kp.degree);
    case 2: return exp(__dmul_rn(-kp.gamma, __dsub_rn(__dadd_rn(xsq_a, xsq_b), __dmul_rn(2.0, dot))));
    case 3: return tanh(__dadd_rn(__dmul_rn(kp.gamma, dot), kp.coef0));
    default: return 0.0;
    }
}

// Q value exactly as the reference stores it: (Qfloat)(y_i*y_j*K)  (svm.cpp:1337)
__device__ __forceinline__ float q_value(const KernelParams &kp, int yy, double dot, double xsq_a, double xsq_b)
{
    return __double2float_rn(__dmul_rn((double)yy, kernel_from_dot(kp, dot, xsq_a, xsq_b)));
}

}  // namespace svmb
