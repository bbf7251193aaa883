// smo_form_fp16x3.cu -- the persistent SMO solver of FORM_FP16X3 (smo_solver.cuh).
#include "smo_solver.cuh"

namespace svmb {

const void *smo_entry_fp16x3() { return (const void *)smo_persistent<FORM_FP16X3>; }

}  // namespace svmb
