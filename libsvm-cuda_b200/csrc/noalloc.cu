// noalloc.cu -- a binary C-SVC solve that allocates no memory.
//
// Some callers cannot allocate device memory while they run: code that
// executes inside a fixed device-memory budget set up at start-up (an
// inference server that pins its pool, an embedded host with no allocator
// available on its real-time path, a plugin whose host application owns every
// allocation).  svmb_solve_dense_noalloc serves them: the caller passes the
// rows, the labels and the output buffer, all already in device memory, and
// every piece of solver state (gradient, alpha, bound status, shrinking lists,
// the Q-row cache, the cross-block records and the launch descriptor) is
// carved out of the statically allocated workspace below.  The function calls
// no cudaMalloc, cudaFree or other allocating routine.
//
// The workspace is a file-scope __device__ array, so every GPU that loads the
// library holds it until the process exits.  Its address is looked up once per
// device with cudaGetSymbolAddress (the first call on a device does this, so
// make that first call before any stream capture) and kept for the life of the
// process: after a cudaDeviceReset by the caller the kept address is stale.  All calls share the one
// workspace and it keeps the previous call's contents: each call re-clears
// what the solver needs to start from zero, and two calls whose work overlaps
// on the GPU (different streams, different host threads) race on it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "engine.hpp"
#include "svm_b200.h"

namespace svmb {

// size of the workspace and the largest problem it accepts
constexpr size_t kNoAllocScratchBytes = 8u << 20;   // 8 MiB per device
constexpr int kNoAllocMaxRows = 16384;
constexpr int kNoAllocMaxBlocks = 160;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

std::mutex g_mu;
void *g_scratch_addr[64] = {};   // device address of the workspace, per device

// initial C-SVC state (reference solve_c_svc, svm.cpp:1500-1533): alpha = 0,
// p = -1, labels +-1; positions start in input order.
__global__ void noalloc_init(const double *yin, int n, signed char *y, double *alpha, double *p, int *pos_local,
                             int *pos_row)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        y[i] = yin[i] > 0 ? 1 : -1;
        alpha[i] = 0.0;
        p[i] = -1.0;
        pos_local[i] = i;
        pos_row[i] = i;
    }
}

// signed coefficients y_i * alpha_i (svm.cpp:1531-1532)
__global__ void noalloc_finish(const double *alpha_local, const double *yin, int n, double *out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = yin[i] > 0 ? alpha_local[i] : -alpha_local[i];
}

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

}  // namespace
}  // namespace svmb

extern "C" int svmb_solve_dense_noalloc(int n, int ld, const float *X, const double *y, const svmb_params *params,
                                        double *alpha_out, svmb_solve_stats *stats, void *stream)
{
    using namespace svmb;
    cudaStream_t s = (cudaStream_t)stream;
    if (!params || !X || !y || !alpha_out) { set_error("NULL argument"); return -1; }
    if (n < 2 || n > kNoAllocMaxRows) {
        set_error("svmb_solve_dense_noalloc: n must be in [2, 16384] (the fixed workspace holds at most 16384 rows)");
        return -1;
    }
    if (ld < 4 || ld % 4 != 0) { set_error("svmb_solve_dense_noalloc: ld must be a positive multiple of 4"); return -1; }
    // rows are read as 16-byte pieces (float4 loads, cp.async): a misaligned
    // base would fault inside the kernel, so it is refused before any launch
    if (((uintptr_t)X & 15) != 0) { set_error("svmb_solve_dense_noalloc: X must be 16-byte aligned"); return -1; }
    if (params->svm_type != C_SVC) { set_error("svmb_solve_dense_noalloc: only C_SVC"); return -1; }
    if (params->kernel_type < LINEAR || params->kernel_type > SIGMOID) { set_error("kernel_type must be LINEAR, POLY, RBF or SIGMOID"); return -1; }
    if (params->C_pos <= 0 || params->C_neg <= 0 || params->eps <= 0 || params->gamma < 0 || params->degree < 0) {
        set_error("svmb_solve_dense_noalloc: invalid parameters");
        return -1;
    }
    if (params->form != SVMB_FORM_EXACT && params->form != SVMB_FORM_FP32) { set_error("unknown form"); return -1; }

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) { set_error("no usable CUDA device"); return -1; }
    void *base;
    {
        std::lock_guard<std::mutex> g(g_mu);
        if (!g_scratch_addr[dev]) {
            void *addr = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
            if (e != cudaSuccess || !addr) {
                set_error(std::string("cudaGetSymbolAddress of the workspace failed: ") + cudaGetErrorString(e));
                return -1;
            }
            g_scratch_addr[dev] = addr;
        }
        base = g_scratch_addr[dev];
    }

    // launch geometry (same rules as the allocating path, capped)
    int smem_total = 0, sms = 0;
    if (cudaDeviceGetAttribute(&smem_total, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        set_error("cannot query the device");
        return -1;
    }
    constexpr int kChunkBytes = 3 * 8 + 2 * 4 + 2;
    const long long budget = (long long)smem_total - smo_static_smem() - 1024;
    int stage_cap = (int)std::min<long long>(kSrcBatch, (48LL << 10) / ((long long)ld * 4));
    if (stage_cap < 2) stage_cap = 0;
    // staged source values are float64 in the exact form
    const int elem = params->form == SVMB_FORM_EXACT ? 8 : 4;
    long long stage_bytes = (((long long)stage_cap * ld * elem) + 15) & ~15LL;
    stage_bytes += kAuxBytes;   // transpose tiles (two per warp) / prefetch candidates
    const long long chunk_max = (budget - stage_bytes) / kChunkBytes;
    if (chunk_max < 64) { set_error("not enough shared memory for the solver state"); return -1; }
    int nb = (int)std::max<long long>(1, std::min<long long>(sms, (n + 1499) / 1500));
    nb = (int)std::max<long long>(nb, (n + chunk_max - 1) / chunk_max);
    if (params->blocks > 0) nb = std::max(params->blocks, (int)((n + chunk_max - 1) / chunk_max));
    nb = std::min(nb, std::min(n, kNoAllocMaxBlocks));
    const long long chunk_cap = (n + nb - 1) / nb;
    if (chunk_cap > chunk_max) { set_error("svmb_solve_dense_noalloc: problem does not fit the block layout"); return -1; }
    const size_t dyn_smem = (size_t)(stage_bytes + chunk_cap * kChunkBytes);
    int per_sm = 0;
    if (smo_max_blocks(params->form, dyn_smem, &per_sm) != cudaSuccess || per_sm * sms < nb) {
        set_error("solver blocks do not fit on the device");
        return -1;
    }

    // carve the workspace
    char *w = (char *)base;
    size_t off = 0;
    auto take = [&](size_t bytes) { char *p = w + off; off = align256(off + bytes); return p; };
    InstanceDesc *d_desc = (InstanceDesc *)take(sizeof(InstanceDesc));
    int *d_block_inst = (int *)take(sizeof(int) * kNoAllocMaxBlocks);
    SolveOut *d_out = (SolveOut *)take(sizeof(SolveOut));
    GroupSync *d_sync = (GroupSync *)take(sizeof(GroupSync));
    Partial *d_part = (Partial *)take(sizeof(Partial) * 2 * kNoAllocMaxBlocks);
    double *G = (double *)take(8 * (size_t)n), *G_bar = (double *)take(8 * (size_t)n);
    double *alpha = (double *)take(8 * (size_t)n), *pvec = (double *)take(8 * (size_t)n);
    double *QD = (double *)take(8 * (size_t)n), *alpha_local = (double *)take(8 * (size_t)n);
    double *xsq = (double *)take(8 * (size_t)n);
    signed char *yy = (signed char *)take((size_t)n);
    unsigned char *status = (unsigned char *)take((size_t)n);
    int *pos_local = (int *)take(4 * (size_t)n), *pos_row = (int *)take(4 * (size_t)n);
    int *lists = (int *)take(8 * (size_t)n);
    // cache: whatever remains, at least 4 rows
    const int ways_max = kMaxWays;
    const size_t meta_per_slot = 4 + 4 + 8;
    const size_t left = kNoAllocScratchBytes - off - 3 * 256;
    long long slots = (long long)(left / (meta_per_slot + 4 * (size_t)n));
    slots = std::min<long long>(slots, 2LL * n);
    if (slots < 4) { set_error("svmb_solve_dense_noalloc: workspace too small for the Q-row cache"); return -1; }
    const int ways = (int)std::min<long long>(ways_max, slots);
    const int sets = (int)(slots / ways);
    const size_t nslots = (size_t)sets * ways;
    int *tag = (int *)take(4 * nslots);
    int *epoch = (int *)take(4 * nslots);
    unsigned long long *stamp = (unsigned long long *)take(8 * nslots);
    float *cdata = (float *)take(4 * nslots * (size_t)n);
    if (off > kNoAllocScratchBytes) { set_error("svmb_solve_dense_noalloc: workspace overflow"); return -1; }

    InstanceDesc D;
    memset(&D, 0, sizeof(D));
    D.l = n;
    D.nu = 0;
    D.shrinking = params->shrinking;
    D.form = params->form;
    D.Cp = params->C_pos;
    D.Cn = params->C_neg;
    D.eps = params->eps;
    D.max_iter = std::max<long long>(10000000LL, 100LL * n);
    D.kp.type = params->kernel_type;
    D.kp.degree = params->degree;
    D.kp.gamma = params->gamma;
    D.kp.coef0 = params->coef0;
    D.x.X = X;
    D.x.ld = ld;
    D.x.rowptr = nullptr;
    D.x.col = nullptr;
    D.x.val = nullptr;
    D.x.d = ld;
    D.x.xsq = xsq;
    D.x.Xs = nullptr;
    D.x.nchunk = 0;
    D.x.xinv = nullptr;
    D.G = G; D.G_bar = G_bar; D.alpha = alpha; D.p = pvec; D.QD = QD;
    D.y = yy; D.status = status; D.pos_local = pos_local; D.pos_row = pos_row;
    D.alpha_local = alpha_local; D.out = d_out;
    D.block0 = 0; D.nblocks = nb;
    D.sync = d_sync; D.partials = d_part; D.scratch = lists;
    D.cache.data = cdata; D.cache.tag = tag; D.cache.epoch = epoch; D.cache.stamp = stamp;
    D.cache.nsets = sets; D.cache.nways = ways; D.cache.stride = n;
    D.stage_cap = stage_cap;
    D.stage_lds = ld;
    D.chunk_cap = (int)chunk_cap;
    D.prefetch = stage_cap > 0 ? std::min(kPrefetchMax, stage_cap) : kPrefetchMax;
    if (params->prefetch > 0) D.prefetch = std::min(D.prefetch, params->prefetch);
    D.lazy_gbar = 0;
    D.tc_n = 0;
    D.done_flag = nullptr;
    D.tile_bufs = 2;
    int block_inst[kNoAllocMaxBlocks];
    for (int b = 0; b < nb; b++) block_inst[b] = 0;

#define NA_CK(call)                                                                     \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) {                                                        \
            set_error(std::string("svmb_solve_dense_noalloc: ") + cudaGetErrorString(e_)); \
            return -1;                                                                  \
        }                                                                               \
    } while (0)
    // what must start from zero (the workspace keeps the previous call's contents)
    NA_CK(cudaMemsetAsync(d_sync, 0, sizeof(GroupSync), s));
    NA_CK(cudaMemsetAsync(d_part, 0, sizeof(Partial) * 2 * kNoAllocMaxBlocks, s));
    NA_CK(cudaMemsetAsync(tag, 0xff, 4 * nslots, s));
    NA_CK(cudaMemsetAsync(epoch, 0, 4 * nslots, s));
    NA_CK(cudaMemsetAsync(stamp, 0, 8 * nslots, s));
    NA_CK(xfer_async(d_desc, &D, sizeof(InstanceDesc), cudaMemcpyHostToDevice, s));
    NA_CK(xfer_async(d_block_inst, block_inst, sizeof(int) * nb, cudaMemcpyHostToDevice, s));
    noalloc_init<<<(n + 255) / 256, 256, 0, s>>>(y, n, yy, alpha, pvec, pos_local, pos_row);
    NA_CK(cudaGetLastError());
    count_launch();
    NA_CK(launch_xsq(D.x, n, xsq, params->form, s));
    count_launch();
    NA_CK(launch_smo(params->form, d_desc, d_block_inst, nb, dyn_smem, true, s));
    count_launch();
    noalloc_finish<<<(n + 255) / 256, 256, 0, s>>>(alpha_local, y, n, alpha_out);
    NA_CK(cudaGetLastError());
    count_launch();
    SolveOut o;
    NA_CK(xfer_async(&o, d_out, sizeof(SolveOut), cudaMemcpyDeviceToHost, s));
    NA_CK(cudaStreamSynchronize(s));
#undef NA_CK
    if (o.status < 0) { set_error("svmb_solve_dense_noalloc: solver wait timed out"); return -1; }
    if (stats) {
        memset(stats, 0, sizeof(*stats));
        stats->iters = o.iters;
        stats->obj = o.obj;
        stats->rho = o.rho;
        stats->l = n;
        stats->status = o.status;
        stats->active_size = o.active_size;
        stats->sum_active = o.sum_active;
        stats->q_evals = o.q_evals;
        stats->lookups = o.lookups;
        stats->hits = o.hits;
        for (int k = 0; k < 8; k++) stats->prof_cycles[k] = o.prof[k];
    }
    return 0;
}
