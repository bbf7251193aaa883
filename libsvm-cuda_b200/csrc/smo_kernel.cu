// smo_kernel.cu -- launchers of the persistent SMO solver (its device code is
// in smo_solver.cuh, instantiated per form in smo_form_*.cu) and the row
// set-up kernels: norms and CSR -> dense rows.
#include "engine.h"

#include <cuda_runtime.h>

namespace svmb {

// the solver kernel of each form (smo_form_*.cu)
const void *smo_entry_exact();
const void *smo_entry_fp32();
const void *smo_entry_bf16x3();
const void *smo_entry_fp16x3();
const void *smo_entry_tf32();

// ---------------------------------------------------------------------------
// setup kernels
// ---------------------------------------------------------------------------
// ||x||^2 per row, in feature order (reference svm.cpp:282-296)
__global__ void xsq_kernel(DevX x, int n, double *out, int form)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        double acc = 0.0;
        float accf = 0.0f;
        if (x.X) {
            const float4 *row = reinterpret_cast<const float4 *>(x.X + (long long)r * x.ld);
            for (int k = 0; k < (x.ld >> 2); k++) {
                const float4 v = __ldg(row + k);
                acc = fma((double)v.x, (double)v.x, acc); acc = fma((double)v.y, (double)v.y, acc);
                acc = fma((double)v.z, (double)v.z, acc); acc = fma((double)v.w, (double)v.w, acc);
                accf = fmaf(v.x, v.x, accf); accf = fmaf(v.y, v.y, accf);
                accf = fmaf(v.z, v.z, accf); accf = fmaf(v.w, v.w, accf);
            }
        } else {
            for (long long e = x.rowptr[r]; e < x.rowptr[r + 1]; e++) {
                const float v = x.val[e];
                acc = fma((double)v, (double)v, acc);
                accf = fmaf(v, v, accf);
            }
        }
        out[r] = form == FORM_EXACT ? acc : (double)accf;
    }
}

// CSR -> dense rows on the device (rows [n][ld] must be zeroed)
__global__ void scatter_dense_kernel(const long long *rowptr, const int *col, const float *val, int n, int ld, float *X)
{
    for (int r = blockIdx.x; r < n; r += gridDim.x)
        for (long long e = rowptr[r] + threadIdx.x; e < rowptr[r + 1]; e += blockDim.x)
            X[(long long)r * ld + col[e]] = val[e];
}

// host-callable launchers ----------------------------------------------------
cudaError_t launch_xsq(const DevX &x, int n, double *out, int form, cudaStream_t s)
{
    int blocks = (n + 255) / 256;
    if (blocks > 148 * 8) blocks = 148 * 8;
    if (blocks < 1) blocks = 1;
    xsq_kernel<<<blocks, 256, 0, s>>>(x, n, out, form);
    return cudaGetLastError();
}

cudaError_t launch_scatter_dense(const long long *rowptr, const int *col, const float *val, int n, int ld, float *X,
                                 cudaStream_t s)
{
    const int blocks = n < 148 * 16 ? (n > 0 ? n : 1) : 148 * 16;
    scatter_dense_kernel<<<blocks, 128, 0, s>>>(rowptr, col, val, n, ld, X);
    return cudaGetLastError();
}

static cudaError_t set_max_dyn_smem(const void *fn)
{
    int dev = 0, optin = 0;
    cudaFuncAttributes a;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, fn);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)a.sharedSizeBytes);
    return e;
}

static const void *smo_fn(int form)
{
    if (form == FORM_EXACT) return smo_entry_exact();
    if (form == FORM_FP32) return smo_entry_fp32();
    if (form == FORM_BF16X3) return smo_entry_bf16x3();
    if (form == FORM_TF32) return smo_entry_tf32();
    return smo_entry_fp16x3();
}

cudaError_t launch_smo(int form, const InstanceDesc *d_insts, const int *d_block_inst, int nblocks,
                       size_t dyn_smem, bool cooperative, cudaStream_t s)
{
    void *args[] = {(void *)&d_insts, (void *)&d_block_inst};
    const void *fn = smo_fn(form);
    // the attribute is set to the largest size any launch may use (the same
    // value from every thread), never lowered to one launch's need
    cudaError_t e = set_max_dyn_smem(fn);
    if (e != cudaSuccess) return e;
    (void)dyn_smem;
    if (cooperative)
        return cudaLaunchCooperativeKernel(fn, dim3(nblocks), dim3(kThreads), args, dyn_smem, s);
    return cudaLaunchKernel(fn, dim3(nblocks), dim3(kThreads), args, dyn_smem, s);
}

cudaError_t smo_max_blocks(int form, size_t dyn_smem, int *blocks_per_sm)
{
    const void *fn = smo_fn(form);
    cudaError_t e = set_max_dyn_smem(fn);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, fn, kThreads, dyn_smem);
}

int smo_static_smem()
{
    int most = 0;
    for (int f = 0; f < kNumForms; f++) {
        cudaFuncAttributes a;
        if (cudaFuncGetAttributes(&a, smo_fn(f)) != cudaSuccess) return 16384;
        most = (int)a.sharedSizeBytes > most ? (int)a.sharedSizeBytes : most;
    }
    return most;
}

}  // namespace svmb
