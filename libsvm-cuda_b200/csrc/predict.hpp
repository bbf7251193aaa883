// predict.hpp -- device decision values for svm_predict* (internal).
#pragma once
#include "svm.h"

namespace svmb {

// Decision values and labels of n rows against a trained or loaded model.
// labels[n]; dec (optional) [n][k(k-1)/2] in the reference's pair order.
int predict_batch(const svm_model *model, const svm_node *const *rows, int n, double *labels, double *dec);

// Drop the device copy of a model's support vectors (called when it is freed).
void predict_forget(const svm_model *model);

}  // namespace svmb
