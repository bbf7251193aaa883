// smo_form_tf32.cu -- the persistent SMO solver of FORM_TF32 (smo_solver.cuh).
#include "smo_solver.cuh"

namespace svmb {

const void *smo_entry_tf32() { return (const void *)smo_persistent<FORM_TF32>; }

}  // namespace svmb
