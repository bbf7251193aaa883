// Test infrastructure only (oracle build recipe). Link-time stand-ins for the
// reference's device launchers declared in libsvm/svm_device.h:25-108.
//
// The reference's CPU solver path (svm.cpp Solver/Solver_NU with cuda_flag == 0)
// never calls these; they exist only because svm.cpp and cuda_solver.cpp
// reference them. The reference's own svm_device.cu does not compile under
// CUDA 12.x (legacy texture references), so every entry here aborts loudly.
#include <cstdio>
#include <cstdlib>
#include "svm.h"
#include "svm_device.h"

static void ref_gpu_path_unavailable(const char *what)
{
    std::fprintf(stderr, "oracle/_ref: reference GPU path called (%s); it is not built\n", what);
    std::abort();
}

void launch_cuda_setup_x_square(size_t, size_t, int) { ref_gpu_path_unavailable("setup_x_square"); }
void launch_cuda_setup_QD(size_t, size_t, int) { ref_gpu_path_unavailable("setup_QD"); }
void launch_cuda_compute_obj_diff(size_t, size_t, GradValue_t, CValue_t *, int *, int) { ref_gpu_path_unavailable("compute_obj_diff"); }
void launch_cuda_compute_obj_diff_SVR(size_t, size_t, GradValue_t, CValue_t *, int *, int) { ref_gpu_path_unavailable("compute_obj_diff_SVR"); }
void launch_cuda_update_gradient(size_t, size_t, int) { ref_gpu_path_unavailable("update_gradient"); }
void launch_cuda_update_gradient_SVR(size_t, size_t, int) { ref_gpu_path_unavailable("update_gradient_SVR"); }
void launch_cuda_init_gradient(size_t, size_t, int, int, int) { ref_gpu_path_unavailable("init_gradient"); }
void launch_cuda_prep_gmax(size_t, size_t, GradValue_t *, GradValue_t *, int *, int) { ref_gpu_path_unavailable("prep_gmax"); }
void launch_cuda_compute_alpha(size_t, size_t) { ref_gpu_path_unavailable("compute_alpha"); }
void launch_cuda_update_alpha_status(size_t, size_t) { ref_gpu_path_unavailable("update_alpha_status"); }
void launch_cuda_find_gmax(size_t, size_t, size_t, find_gmax_param, int, bool) { ref_gpu_path_unavailable("find_gmax"); }
void launch_cuda_find_min_idx(size_t, size_t, size_t, CValue_t *, int *, CValue_t *, int *, int) { ref_gpu_path_unavailable("find_min_idx"); }
void launch_cuda_find_nu_gmax(size_t, size_t, size_t, find_nu_gmax_param, int) { ref_gpu_path_unavailable("find_nu_gmax"); }
void launch_cuda_find_nu_min_idx(size_t, size_t, size_t, CValue_t *, int *, CValue_t *, int *, int) { ref_gpu_path_unavailable("find_nu_min_idx"); }
void launch_cuda_compute_nu_obj_diff(size_t, size_t, GradValue_t, GradValue_t, CValue_t *, int *, int) { ref_gpu_path_unavailable("compute_nu_obj_diff"); }
void launch_cuda_compute_nu_obj_diff_SVR(size_t, size_t, GradValue_t, GradValue_t, CValue_t *, int *, int) { ref_gpu_path_unavailable("compute_nu_obj_diff_SVR"); }
void launch_cuda_prep_nu_gmax(size_t, size_t, GradValue_t *, GradValue_t *, GradValue_t *, GradValue_t *, int *, int *, int) { ref_gpu_path_unavailable("prep_nu_gmax"); }
cudaError_t update_solver_variables(SChar_t *, CValue_t *, GradValue_t *, GradValue_t *, char *, double, double) { ref_gpu_path_unavailable("update_solver_variables"); return cudaSuccess; }
cudaError_t update_rbf_variables(CValue_t *) { ref_gpu_path_unavailable("update_rbf_variables"); return cudaSuccess; }
cudaError_t update_param_constants(const svm_parameter &, int *, cuda_svm_node *, size_t, int, uint32_t *, int) { ref_gpu_path_unavailable("update_param_constants"); return cudaSuccess; }
void unbind_texture() { ref_gpu_path_unavailable("unbind_texture"); }
void init_device_gradient(int, int, int, int) { ref_gpu_path_unavailable("init_device_gradient"); }
void show_device_cache_stats() { ref_gpu_path_unavailable("show_device_cache_stats"); }
void setup_device_LRU_cache(CacheNodeBucket *, CValue_t *, int, int) { ref_gpu_path_unavailable("setup_device_LRU_cache"); }
