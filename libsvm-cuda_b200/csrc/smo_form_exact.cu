// smo_form_exact.cu -- the persistent SMO solver of FORM_EXACT (smo_solver.cuh).
#include "smo_solver.cuh"

namespace svmb {

const void *smo_entry_exact() { return (const void *)smo_persistent<FORM_EXACT>; }

}  // namespace svmb
