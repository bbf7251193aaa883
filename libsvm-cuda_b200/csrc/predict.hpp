// predict.hpp -- device decision values for svm_predict* (internal).
#pragma once
#include "svm.h"

namespace svmb {

// Decision values and labels of n rows against a trained or loaded model.
// labels[n]; dec (optional) [n][k(k-1)/2] in the reference's pair order.
int predict_batch(const svm_model *model, const svm_node *const *rows, int n, double *labels, double *dec);

// Drop the device copy of a model's support vectors (called when it is freed).
void predict_forget(const svm_model *model);

// Arithmetic form of the kernel values of prediction: FORM_EXACT (default,
// the reference's k_function bit for bit) or a tensor-core form, where
// K(test rows, SVs) is one block product per chunk of test rows.
int predict_set_form(int form);

}  // namespace svmb
