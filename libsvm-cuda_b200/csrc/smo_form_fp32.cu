// smo_form_fp32.cu -- the persistent SMO solver of FORM_FP32 (smo_solver.cuh).
#include "smo_solver.cuh"

namespace svmb {

const void *smo_entry_fp32() { return (const void *)smo_persistent<FORM_FP32>; }

}  // namespace svmb
