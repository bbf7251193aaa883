// smo_form_bf16x3.cu -- the persistent SMO solver of FORM_BF16X3 (smo_solver.cuh).
#include "smo_solver.cuh"

namespace svmb {

const void *smo_entry_bf16x3() { return (const void *)smo_persistent<FORM_BF16X3>; }

}  // namespace svmb
